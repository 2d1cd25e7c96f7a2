"""CUDA engine vs the CPU oracle and the golden fixtures (through the C ABI).

Tolerances (see _gpu_helpers): neighbour sets identical
(integer work); per-particle density, k and velocity within 1e-4 relative in
FP32 (relative to the largest magnitude in the scene); outer-iteration count
within +-1; results compared whenever the iteration counts agree, with the
outer count forced to the reference's where it differs, and a floor on the
compared steps of every multi-step test.
"""
import dataclasses
import os

import numpy as np
import pytest
import torch

import _gpu_helpers as H
from oracle import oracle as O
from implicitvelocityprojection_b200 import scenes as S

pytestmark = pytest.mark.gpu

RTOL = H.RTOL


def _engine(scs, **opt):
    from implicitvelocityprojection_b200.engine import Engine, EngineOptions
    return Engine(scs, options=EngineOptions(**opt) if opt else None)


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


def _scene_from_golden(g, x, v):
    return S.Scene(x=np.array(x, np.float32), v=np.array(v, np.float32), is_dynamic=g["is_dynamic"],
                   material=g["material"], density0=g["density0"], particle_radius=float(g["particle_radius"]),
                   domain_size=g["domain_size"], dt=float(g["dt"]))


def _load(golden_dir, name):
    return np.load(os.path.join(golden_dir, name))


@pytest.fixture(scope="module")
def small():
    return S.small_column()


def test_neighbour_sets_density_k(small):
    eng = _engine([small])
    eng.build()
    cnt, ids = eng.neighbours(0)
    st = O.State.from_scene(small)
    st.rebuild()
    dyn = np.where(small.is_dynamic == 1)[0]
    for i in dyn:
        got = set(ids[i, :cnt[i]].tolist())
        assert got == st.neighbour_sets(i), i
    dens = eng.get("density")
    k = eng.get("k")
    np.testing.assert_allclose(dens[dyn], st.density[dyn], rtol=RTOL)
    np.testing.assert_allclose(k[dyn], st.k[dyn], rtol=RTOL)
    assert np.all(k[small.is_dynamic == 0] == 0)
    assert eng.stats(0).overflow_particles == 0


def test_block_solve_vs_golden(golden_dir):
    """One IP solve from the reference's compressed, moving block: lists,
    density, k, outer and CG counts, velocity, density-error history and the
    divergence output against the reference's own run."""
    from implicitvelocityprojection_b200.engine import Engine
    g = _load(golden_dir, "block_solve.npz")
    sc = _scene_from_golden(g, g["x"], g["v0"])
    eng = Engine([sc], divergence=True)
    eng.build()
    dyn = sc.is_dynamic == 1
    cnt, ids = eng.neighbours(0)
    off, gids = g["nbr_offsets"], g["nbr_ids"]
    for i in range(int(dyn.sum())):
        assert set(ids[i, :cnt[i]].tolist()) == set(gids[off[i]:off[i + 1]].tolist())
    np.testing.assert_allclose(eng.get("density")[dyn], g["density"][dyn], rtol=RTOL)
    np.testing.assert_allclose(eng.get("k")[dyn], g["k"][dyn], rtol=RTOL)
    eng.solve()
    s = eng.stats(0)
    assert s.status == 0
    outer = int(g["stats_outer_iters"])
    assert abs(s.stats_outer_iters - outer) <= 1
    np.testing.assert_allclose(s.stats_final_density_error, float(g["stats_final_density_error"]), rtol=1e-3,
                               atol=1e-7)
    if s.stats_outer_iters != outer:
        # an error within rounding of densityErrorTol: the reference's count,
        # forced (fixedOuterIters), then compared
        eng = Engine([dataclasses.replace(sc, fixed_outer_iters=True, max_outer_iters=outer)], divergence=True)
        eng.build()
        eng.solve()
        s = eng.stats(0)
    assert s.stats_outer_iters == outer
    assert s.stats_pcg_iters == g["stats_pcg_iters"].tolist()
    assert _rel(eng.get("v")[dyn], g["v"][dyn]) < RTOL
    np.testing.assert_allclose(s.stats_density_errors, g["stats_density_errors"], rtol=1e-3)
    # ps.divergence = max(J v, 0) (pressure_base.py:449-457)
    assert np.abs(g["divergence"][dyn]).max() > 0
    assert _rel(eng.get("divergence")[dyn], g["divergence"][dyn]) < RTOL


def test_column_steps_vs_golden(golden_dir):
    """Each reference Framework.forward() step, restarted from the reference's
    previous state, on the engine's fused step (gravity, IP, advect, rebuild)."""
    g = _load(golden_dir, "column_steps.npz")
    dyn = g["is_dynamic"] == 1
    steps = g["x"].shape[0]
    mism = 0
    for s in range(steps):
        x_prev = g["x0"] if s == 0 else g["x"][s - 1]
        v_prev = g["v0"] if s == 0 else g["v"][s - 1]
        sc = _scene_from_golden(g, x_prev, v_prev)
        sc.gravity = tuple(float(a) for a in g["gravity"])
        eng = _engine([sc])
        eng.build()
        eng.step(1)
        st = eng.stats(0)
        assert st.status == 0
        if st.stats_outer_iters != int(g["outer"][s]):
            assert abs(st.stats_outer_iters - int(g["outer"][s])) <= 1
            mism += 1
            continue
        assert st.stats_pcg_iters == g["pcg"][g["pcg_off"][s]:g["pcg_off"][s + 1]].tolist()
        assert _rel(eng.get("v")[dyn], g["v"][s][dyn]) < RTOL, s
        assert np.abs(eng.get("x")[dyn] - g["x"][s][dyn]).max() < 1e-6, s
        np.testing.assert_allclose(eng.get("density")[dyn], g["density"][s][dyn], rtol=RTOL)
        np.testing.assert_allclose(eng.get("k")[dyn], g["k"][s][dyn], rtol=RTOL)
    assert mism <= max(1, steps // 10)


def test_small_column_steps_vs_oracle(small):
    """The 8,192-particle column: every fused step restarted from the oracle's
    state (strict per-step parity), then a free run of both."""
    st = O.State.from_scene(small)
    st.rebuild()
    compared = 0
    steps = 12
    for s in range(steps):
        sc = H.with_state(small, st.x, st.v)
        ok, eng, st = H.compare_step(sc)
        compared += ok
    assert compared >= steps - 1, compared


def test_small_column_free_run_vs_oracle(small):
    """20 steps of both in lockstep: the trajectories separate only through
    FP32 summation-order rounding, amplified by the violent first steps."""
    eng = _engine([small])
    eng.build()
    st = O.State.from_scene(small)
    st.rebuild()
    dyn = small.is_dynamic == 1
    for s in range(20):
        eng.step(1)
        st.step(fast=True)
        gs = eng.stats(0)
        assert gs.status == 0 and st.status == 0
        assert abs(gs.stats_outer_iters - st.stats_outer_iters) <= 1, s
    assert np.abs(eng.get("x")[dyn] - st.x[dyn]).max() < 5e-4  # 2.5 % of a spacing


def test_solve_matches_oracle_and_fp64(small):
    """One IP solve from a compressed, moving state: velocity against the
    oracle (1e-4 relative), and the first linear system's FP64 CG solution
    exists (the FP32 path's error against it is stated by
    test_cg_solution_error_vs_fp64_oracle)."""
    sc = S.column_in_box((12, 14, 12), 0.018, (0.4, 0.5, 0.4), seed=5)
    rng = np.random.default_rng(1)
    sc.v[sc.is_dynamic == 1] = rng.normal(0, 0.2, size=(sc.n_dynamic, 3)).astype(np.float32)
    ok, eng, st, _ = H.compare_solve(sc)
    assert ok, "iteration counts differ even with the outer count fixed"
    dyn = sc.is_dynamic == 1
    st2 = O.State.from_scene(sc)
    st2.rebuild()
    d0 = np.zeros((sc.n, 3), np.float32)
    d0[dyn] = np.float32(sc.dt) * sc.v[dyn]
    t, f, dfdt, rhs = st2.system(d0)
    x64, it = st2.cg_f64(dfdt, rhs, rel_tol=1e-12)
    assert it > 0 and np.isfinite(x64).all()


def _error_scene(workload):
    if workload == "small_column":
        return S.small_column()
    if workload == "tall_column_102k":
        return S.tall_column()
    if workload == "dam_break_524k":
        return S.dam_break()
    # the largest scene of the 64-scene batch (a scene's result in the batch
    # is bit-identical to the scene alone)
    return max(S.batch_mix(64), key=lambda sc: sc.n_dynamic)


@pytest.mark.parametrize("workload,row_format,bound", [("small_column", 1, 1e-3), ("small_column", 3, 0.1),
                                                       ("tall_column_102k", 1, 3e-3),
                                                       ("tall_column_102k", 3, 0.1),
                                                       # early in the dam break the constraint is small, so
                                                       # the FP32 rounding of c = rho - rho0 is a larger
                                                       # share of the right-hand side (measured 2.8e-3)
                                                       ("dam_break_524k", 1, 5e-3),
                                                       ("batch64_largest", 1, 3e-3)])
def test_cg_solution_error_vs_fp64_oracle(workload, row_format, bound, record_property):
    """The CG solution of one outer system (the scene after 40 steps, one
    fixed outer update) against the oracle's FP64 CG on the same system run
    for the same number of iterations: the precision error of the FP32 rows
    and of the bf16 gradients, stated per configuration (printed and recorded
    as a test property).  Against the fully converged FP64 solution both are
    about 0.25-0.6 off: the reference's CG stops once |r|^2 < tol_pcg (1e-6,
    absolute, ip.py:319) after two iterations."""
    sc = _error_scene(workload)
    eng = _engine([sc])
    eng.build()
    eng.step(40)
    s1 = dataclasses.replace(sc, x=eng.get("x").copy(), v=eng.get("v").copy(), max_outer_iters=1,
                             fixed_outer_iters=True, viscosity_method=0, viscosity_coeff=0.0,
                             surface_tension_method=0, surface_tension_coeff=0.0)
    dyn = sc.is_dynamic == 1
    st = O.State.from_scene(s1)
    st.rebuild()
    d0 = np.zeros((sc.n, 3), np.float32)
    d0[dyn] = np.float32(sc.dt) * s1.v[dyn]
    t, f, dfdt, rhs = st.system(d0)
    e = _engine([s1], row_format=row_format)
    e.build()
    vb = e.get("v").astype(np.float64)
    e.solve()
    gs = e.stats(0)
    assert gs.status == 0 and gs.stats_outer_iters == 1
    sol = np.float64(sc.dt) * (vb - e.get("v").astype(np.float64))
    xk, _ = st.cg_f64(dfdt, rhs, rel_tol=0.0, max_iter=gs.stats_pcg_iters[0])
    err = np.linalg.norm(sol[dyn] - xk[dyn]) / np.linalg.norm(xk[dyn])
    x64, it = st.cg_f64(dfdt, rhs, rel_tol=1e-14)
    err64 = np.linalg.norm(sol[dyn] - x64[dyn]) / np.linalg.norm(x64[dyn])
    print(f"{workload} rows={'bf16' if row_format == 3 else 'fp32'}: CG iterations {gs.stats_pcg_iters[0]}, "
          f"error vs FP64 CG at equal iterations {err:.3e}, vs converged FP64 ({it} iterations) {err64:.3e}")
    record_property("error_vs_fp64_equal_iterations", float(err))
    record_property("error_vs_fp64_converged", float(err64))
    assert err < bound, err
    assert it > gs.stats_pcg_iters[0]
    assert err64 < 0.8


def test_multi_scene_bitwise_equal_to_alone():
    """Scenes batched in one engine give bit-identical results to each scene
    alone (per-scene reductions never mix scenes)."""
    scs = [S.random_column(2500, 1.5, seed=11), S.random_column(6000, 3.0, seed=12),
           S.small_dam_break(3000, seed=13)]
    eng = _engine(scs)
    eng.build()
    eng.step(5)
    for i, sc in enumerate(scs):
        alone = _engine([sc])
        alone.build()
        alone.step(5)
        assert np.array_equal(eng.get("x", i), alone.get("x", 0)), i
        assert np.array_equal(eng.get("v", i), alone.get("v", 0)), i
        a, b = eng.stats(i), alone.stats(0)
        assert a.stats_density_errors == b.stats_density_errors


def test_deterministic_across_execution_paths(small):
    """Persistent cooperative solve, one launch per phase in conditional
    graphs, and host-driven launches share the tile code and the reduction
    order: results are bit-identical, and repeatable."""
    outs = []
    for use_graphs, persistent in ((True, True), (True, True), (True, False), (False, False), (False, True)):
        eng = _engine([small], use_graphs=use_graphs, persistent=persistent)
        eng.build()
        eng.step(4)
        outs.append((eng.get("x"), eng.get("v"), eng.stats(0).stats_density_errors))
    for o in outs[1:]:
        assert np.array_equal(o[0], outs[0][0])
        assert np.array_equal(o[1], outs[0][1])
        assert o[2] == outs[0][2]


def test_persistent_equals_per_phase_with_many_tiles_per_cta():
    """About 600k fluid particles in 32-particle tiles: every persistent CTA
    walks more than 16 tiles per phase, so it combines its parked per-warp
    tile sums several times within one phase.  The results stay bit-identical
    to one launch per phase."""
    scs = [S.random_column(150_000, 2.0, seed=31 + k) for k in range(4)]
    opts = dict(lanes_per_particle=8, particles_per_block=32)
    n_tiles = sum((sc.n_dynamic + 31) // 32 for sc in scs)
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    assert n_tiles > 16 * 4 * sms  # 256-thread CTAs, at most 4 per SM at 64 registers
    a = _engine(scs, persistent=True, **opts)
    b = _engine(scs, persistent=False, **opts)
    for e in (a, b):
        e.build()
        e.step(2)
    for i in range(len(scs)):
        assert np.array_equal(a.get("x", i), b.get("x", i)), i
        assert np.array_equal(a.get("v", i), b.get("v", i)), i
        assert a.stats(i).stats_pcg_iters == b.stats(i).stats_pcg_iters


def test_read_solve_equals_stats_and_history():
    """ivp_read_solve (one synchronisation) returns what ivp_read_stats and
    ivp_read_history return separately, for every scene of a batch."""
    import ctypes
    from implicitvelocityprojection_b200 import _lib
    scs = [S.random_column(2500, 1.5, seed=41), S.small_dam_break(4000, seed=42)]
    eng = _engine(scs)
    eng.build()
    eng.step(2)
    L, h, st = eng.L, eng._handle, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    cap = 16
    for i in range(len(scs)):
        a = _lib.SolveStats()
        assert L.ivp_read_stats(h, i, st, ctypes.byref(a)) == _lib.OK
        e1, p1 = np.zeros(cap), np.zeros(cap, np.int32)
        n1, m1 = ctypes.c_int32(0), ctypes.c_int32(0)
        assert L.ivp_read_history(h, i, st, e1.ctypes.data_as(ctypes.c_void_p), p1.ctypes.data_as(ctypes.c_void_p),
                                  cap, ctypes.byref(n1), ctypes.byref(m1)) == _lib.OK
        b = _lib.SolveStats()
        e2, p2 = np.full(cap, -1.0), np.full(cap, -1, np.int32)
        n2, m2 = ctypes.c_int32(0), ctypes.c_int32(0)
        assert L.ivp_read_solve(h, i, st, ctypes.byref(b), e2.ctypes.data_as(ctypes.c_void_p),
                                p2.ctypes.data_as(ctypes.c_void_p), cap, ctypes.byref(n2), ctypes.byref(m2)) == _lib.OK
        assert bytes(a) == bytes(b)
        assert (n1.value, m1.value) == (n2.value, m2.value) and n1.value >= 1
        assert np.array_equal(e1[:n1.value], e2[:n2.value]) and np.array_equal(p1[:m1.value], p2[:m2.value])


def test_multi_scene_persistent_equals_per_phase():
    scs = [S.random_column(2500, 1.5, seed=21), S.small_dam_break(4000, seed=22), S.random_column(900, 3.0, seed=23)]
    a = _engine(scs, persistent=True)
    b = _engine(scs, persistent=False)
    for e in (a, b):
        e.build()
        e.step(3)
    for i in range(len(scs)):
        assert np.array_equal(a.get("x", i), b.get("x", i))
        assert np.array_equal(a.get("v", i), b.get("v", i))
        assert a.stats(i).stats_pcg_iters == b.stats(i).stats_pcg_iters


@pytest.mark.parametrize("lanes,ppb", [(1, 128), (2, 128), (4, 64), (8, 32), (2, 64), (4, 32), (8, 16)])
def test_lane_variants_agree(small, lanes, ppb):
    """Every launch shape the autotuner can pick (and one lane per particle)
    gives the same steps within the FP32 tolerance."""
    ref = _engine([small])
    ref.build()
    ref.step(3)
    eng = _engine([small], lanes_per_particle=lanes, particles_per_block=ppb)
    eng.build()
    eng.step(3)
    dyn = small.is_dynamic == 1
    assert np.abs(eng.get("x")[dyn] - ref.get("x")[dyn]).max() < 1e-6
    assert _rel(eng.get("v")[dyn], ref.get("v")[dyn]) < 1e-4


def test_standalone_density_aii_equal_fused(small):
    eng = _engine([small])
    eng.build()
    d1, k1 = eng.get("density"), eng.get("k")
    eng.arrays["density"].zero_()
    eng.arrays["k"].zero_()
    eng.compute_density()
    eng.compute_aii()
    dyn = small.is_dynamic == 1
    np.testing.assert_allclose(eng.get("density")[dyn], d1[dyn], rtol=1e-6)
    np.testing.assert_allclose(eng.get("k")[dyn], k1[dyn], rtol=1e-6)


def test_not_converged_status(small):
    """maxOuterIters = 0 forces the reference's check_converged raise when the
    error is above tolerance."""
    fluid = S.lattice_block([0.2, 0.2, 0.2], (10, 10, 10), 0.014, jitter=0.01, seed=2)
    sc = S.assemble([fluid], [], particle_radius=0.01, domain_size=[0.6, 0.6, 0.6], max_outer_iters=0)
    eng = _engine([sc])
    eng.build()
    v0 = eng.get("v").copy()
    eng.solve()
    s = eng.stats(0)
    assert s.status == 2
    # the reference raises before v = d / dt, so v is unchanged
    assert np.array_equal(eng.get("v"), v0)


# ----------------------------------------------------------- Weiler18 viscosity

def _visc_scene(g, x, v, coeff):
    sc = _scene_from_golden(g, x, v)
    sc.viscosity_method = 1
    sc.viscosity_coeff = float(coeff)
    return sc


def test_viscosity_solve_vs_golden(golden_dir):
    g = _load(golden_dir, "visc_solve.npz")
    sc = _visc_scene(g, g["x"], g["v0"], g["coeff"])
    eng = _engine([sc])
    eng.build()
    dyn = sc.is_dynamic == 1
    np.testing.assert_allclose(eng.get("density")[dyn], g["density"][dyn], rtol=RTOL)
    eng.viscosity_solve()
    v = eng.get("v")
    assert _rel(v[dyn], g["v"][dyn]) < RTOL
    assert _rel(v[dyn] - g["v0"][dyn], g["dv"][dyn]) < 1e-3


@pytest.mark.parametrize("persistent", [True, False])
def test_column_visc_steps_vs_golden(golden_dir, persistent):
    g = _load(golden_dir, "column_visc_steps.npz")
    dyn = g["is_dynamic"] == 1
    steps = g["x"].shape[0]
    compared = 0
    for s in range(steps):
        x_prev = g["x0"] if s == 0 else g["x"][s - 1]
        v_prev = g["v0"] if s == 0 else g["v"][s - 1]
        sc = _visc_scene(g, x_prev, v_prev, g["viscosity"])
        sc.gravity = tuple(float(a) for a in g["gravity"])
        eng = _engine([sc], persistent=persistent)
        eng.build()
        eng.step(1)
        st = eng.stats(0)
        assert st.status == 0
        assert abs(st.stats_outer_iters - int(g["outer"][s])) <= 1
        if st.stats_outer_iters != int(g["outer"][s]):
            continue
        compared += 1
        assert _rel(eng.get("v")[dyn], g["v"][s][dyn]) < RTOL, s
        assert np.abs(eng.get("x")[dyn] - g["x"][s][dyn]).max() < 1e-6, s
    assert compared >= steps - 1, compared


def test_viscous_column_vs_oracle_and_paths():
    """The tall-column physics (Weiler18 nu = 1e-3) on a smaller column: each
    step restarted from the oracle's state, and persistent vs per-phase paths
    bit-identical."""
    sc = S.column_in_box((12, 24, 12), 0.02, (0.4, 1.0, 0.4), seed=4, viscosity_method=1, viscosity_coeff=1e-3)
    st = O.State.from_scene(sc)
    st.rebuild()
    compared = 0
    steps = 6
    for s in range(steps):
        cur = H.with_state(sc, st.x, st.v)
        b = _engine([cur], persistent=False)
        b.build()
        b.step(1)
        ok, a, st = H.compare_step(cur, persistent=True)
        compared += ok
        if ok:  # the same (unforced) solve on both paths
            assert np.array_equal(a.get("v"), b.get("v"))
    assert compared >= steps - 1, compared


@pytest.mark.parametrize("persistent", [True, False])
def test_row_formats_bitwise_equal(persistent):
    """Full rows {J, j} and compact rows {j, w} (J rebuilt from the positions
    with the same products) give bit-identical steps, with and without
    viscosity, and identical exported neighbour lists."""
    scs = [S.random_column(3000, 2.0, seed=31),
           S.column_in_box((10, 20, 10), 0.02, (0.4, 0.9, 0.4), seed=32, viscosity_method=1, viscosity_coeff=1e-3)]
    full = _engine(scs, row_format=1, persistent=persistent)
    comp = _engine(scs, row_format=2, persistent=persistent)
    for e in (full, comp):
        e.build()
        e.step(4)
    for i in range(len(scs)):
        assert np.array_equal(full.get("x", i), comp.get("x", i)), i
        assert np.array_equal(full.get("v", i), comp.get("v", i)), i
        assert np.array_equal(full.get("density", i), comp.get("density", i)), i
        assert np.array_equal(full.get("k", i), comp.get("k", i)), i
        a, b = full.stats(i), comp.stats(i)
        assert a.stats_pcg_iters == b.stats_pcg_iters and a.stats_density_errors == b.stats_density_errors
        ca, ia = full.neighbours(i)
        cb, ib = comp.neighbours(i)
        assert np.array_equal(ca, cb) and np.array_equal(ia, ib)


# ---------------------------------------------------- Jeske23 surface tension

def _st_scene(g, x, v, sigma, visc=0.0):
    sc = _scene_from_golden(g, x, v)
    sc.surface_tension_method = 1
    sc.surface_tension_coeff = float(sigma)
    if visc > 0:
        sc.viscosity_method = 1
        sc.viscosity_coeff = float(visc)
    return sc


@pytest.mark.parametrize("persistent", [True, False])
def test_surface_tension_solve_vs_golden(golden_dir, persistent):
    g = _load(golden_dir, "st_solve.npz")
    sc = _st_scene(g, g["x"], g["v0"], g["sigma"])
    eng = _engine([sc], persistent=persistent)
    eng.build()
    dyn = sc.is_dynamic == 1
    eng.surface_tension_solve()
    v = eng.get("v")
    assert _rel(v[dyn], g["v"][dyn]) < RTOL
    assert _rel(v[dyn] - g["v0"][dyn], g["dv"][dyn]) < 5e-3  # the correction, relative to its own size
    assert eng.raw_stats(0).sum_st_iters >= 1


@pytest.mark.parametrize("persistent", [True, False])
def test_column_st_steps_vs_golden(golden_dir, persistent):
    """Steps with surface tension, viscosity and IP, each restarted from the
    reference's previous state."""
    g = _load(golden_dir, "column_st_steps.npz")
    dyn = g["is_dynamic"] == 1
    compared = 0
    for s in range(g["x"].shape[0]):
        x_prev = g["x0"] if s == 0 else g["x"][s - 1]
        v_prev = g["v0"] if s == 0 else g["v"][s - 1]
        sc = _st_scene(g, x_prev, v_prev, g["sigma"], float(g["viscosity"]))
        sc.gravity = tuple(float(a) for a in g["gravity"])
        eng = _engine([sc], persistent=persistent)
        eng.build()
        eng.step(1)
        st = eng.stats(0)
        assert st.status == 0
        raw = eng.raw_stats(0)
        assert raw.sum_st_iters >= 1 and raw.sum_visc_iters >= 1
        if st.stats_outer_iters != int(g["outer"][s]):
            continue
        compared += 1
        assert _rel(eng.get("v")[dyn], g["v"][s][dyn]) < RTOL, s
        assert np.abs(eng.get("x")[dyn] - g["x"][s][dyn]).max() < 1e-6, s
    assert compared >= g["x"].shape[0] - 1


def test_surface_tension_paths_and_batch_bitwise():
    """Surface tension + viscosity scenes: persistent and per-phase paths, and
    a scene in a batch with other scenes, give identical bits."""
    a = S.column_in_box((10, 18, 10), 0.02, (0.4, 0.8, 0.4), seed=51, viscosity_method=1, viscosity_coeff=1e-3,
                        surface_tension_method=1, surface_tension_coeff=0.05)
    b = S.small_dam_break(3000, seed=52)
    c = S.random_column(2000, 2.0, seed=53, surface_tension_method=1, surface_tension_coeff=0.05)
    p = _engine([a, b, c], persistent=True)
    q = _engine([a, b, c], persistent=False)
    for e in (p, q):
        e.build()
        e.step(3)
    for i in range(3):
        assert np.array_equal(p.get("v", i), q.get("v", i)), i
        assert np.array_equal(p.get("x", i), q.get("x", i)), i
    alone = _engine([a])
    alone.build()
    alone.step(3)
    assert np.array_equal(alone.get("v"), p.get("v", 0))
    assert p.raw_stats(0).sum_st_iters > 0 and p.raw_stats(1).sum_st_iters == 0


def test_surface_tension_free_run_vs_oracle():
    """A small surface-tension column stepped on the GPU and by the oracle."""
    sc = S.column_in_box((8, 14, 8), 0.02, (0.3, 0.5, 0.3), seed=61, surface_tension_method=1,
                         surface_tension_coeff=0.05)
    eng = _engine([sc])
    eng.build()
    st = O.State.from_scene(sc)
    st.rebuild()
    dyn = sc.is_dynamic == 1
    for s in range(5):
        eng.step(1)
        st.step(fast=True)
    assert np.abs(eng.get("x")[dyn] - st.x[dyn]).max() < 5e-4


def test_bf16_gradient_variant_close_to_fp32():
    """The reduced-precision row format (gradients rounded to bf16, relative
    error 2^-9): identical neighbour sets, every step converged to the
    density tolerance, positions within 5 % of a particle spacing of the FP32
    rows after 5 steps."""
    sc = S.column_in_box((12, 24, 12), 0.02, (0.4, 1.0, 0.4), seed=71, viscosity_method=1, viscosity_coeff=1e-3,
                         surface_tension_method=1, surface_tension_coeff=0.05)
    full = _engine([sc], row_format=1)
    half = _engine([sc], row_format=3)
    for e in (full, half):
        e.build()
    ca, ia = full.neighbours(0)
    cb, ib = half.neighbours(0)
    assert np.array_equal(ca, cb) and np.array_equal(ia, ib)
    dyn = sc.is_dynamic == 1
    for _ in range(5):
        for e in (full, half):
            e.step(1)
        st = half.stats(0)
        assert st.status == 0 and st.stats_final_density_error < sc.density_error_tol
    assert np.abs(half.get("x")[dyn] - full.get("x")[dyn]).max() < 0.05 * 0.02
    assert np.abs(half.get("density")[dyn] - full.get("density")[dyn]).max() / 1000.0 < 1e-2


# --------------------------------------------------------- PRJ (projected Jacobi)

def _prj_scene(g, x, v):
    sc = _scene_from_golden(g, x, v)
    sc.pressure_method = 0
    sc.omega = 0.5  # PRJ's relaxation (prj.py:127)
    return sc


@pytest.mark.parametrize("persistent", [True, False])
def test_prj_solve_vs_golden(golden_dir, persistent):
    g = _load(golden_dir, "prj_solve.npz")
    sc = _prj_scene(g, g["x"], g["v0"])
    eng = _engine([sc], persistent=persistent)
    eng.build()
    eng.prj_solve()
    st = eng.stats(0)
    dyn = sc.is_dynamic == 1
    passes = int(g["stats_outer_iters"])
    assert st.status == 0
    assert abs(st.stats_outer_iters - passes) <= 1
    if st.stats_outer_iters != passes:
        # the reference's pass count, forced (fixedOuterIters), then compared
        eng = _engine([dataclasses.replace(sc, fixed_outer_iters=True, max_outer_iters=passes)],
                      persistent=persistent)
        eng.build()
        eng.prj_solve()
        st = eng.stats(0)
    assert st.stats_outer_iters == passes
    assert _rel(eng.get("v")[dyn], g["v"][dyn]) < RTOL
    np.testing.assert_allclose(st.stats_density_errors, g["stats_density_errors"], rtol=1e-3, atol=1e-8)


@pytest.mark.parametrize("persistent", [True, False])
def test_column_prj_steps_vs_golden(golden_dir, persistent):
    g = _load(golden_dir, "column_prj_steps.npz")
    dyn = g["is_dynamic"] == 1
    compared = 0
    for s in range(g["x"].shape[0]):
        x_prev = g["x0"] if s == 0 else g["x"][s - 1]
        v_prev = g["v0"] if s == 0 else g["v"][s - 1]
        sc = _prj_scene(g, x_prev, v_prev)
        sc.gravity = tuple(float(a) for a in g["gravity"])
        eng = _engine([sc], persistent=persistent)
        eng.build()
        eng.step(1)
        st = eng.stats(0)
        assert st.status == 0
        assert abs(st.stats_outer_iters - int(g["outer"][s])) <= 1
        if st.stats_outer_iters != int(g["outer"][s]):
            continue
        compared += 1
        assert _rel(eng.get("v")[dyn], g["v"][s][dyn]) < RTOL, s
        assert np.abs(eng.get("x")[dyn] - g["x"][s][dyn]).max() < 1e-6, s
    assert compared >= g["x"].shape[0] - 2


def test_prj_paths_and_mixed_batch_bitwise():
    """PRJ and IP scenes in one engine: every path gives the same bits, and
    each scene equals the scene run alone."""
    a = S.random_column(2500, 2.0, seed=81, pressure_method=0, omega=0.5)
    b = S.random_column(3000, 1.5, seed=82)
    c = S.small_dam_break(2000, seed=83, pressure_method=0, omega=0.5)
    outs = []
    for use_graphs, persistent in ((True, True), (True, False), (False, False)):
        e = _engine([a, b, c], use_graphs=use_graphs, persistent=persistent)
        e.build()
        e.step(3)
        outs.append([(e.get("x", i), e.get("v", i)) for i in range(3)])
        assert all(e.stats(i).status == 0 for i in range(3))
    for o in outs[1:]:
        for i in range(3):
            assert np.array_equal(o[i][0], outs[0][i][0]) and np.array_equal(o[i][1], outs[0][i][1]), i
    for i, sc in enumerate((a, b, c)):
        alone = _engine([sc])
        alone.build()
        alone.step(3)
        assert np.array_equal(alone.get("x"), outs[0][i][0]), i


def test_prj_framework_dropin():
    """Framework with pressureMethod 0 builds the PRJ class and steps."""
    from implicitvelocityprojection_b200.config import SimConfig
    from implicitvelocityprojection_b200.framework import Framework
    from implicitvelocityprojection_b200.neighbour_search import NeighbourSearch
    from implicitvelocityprojection_b200.prj import PRJ
    from implicitvelocityprojection_b200.simulation_data import SimulationData
    sc = S.random_column(2000, 2.0, seed=84, pressure_method=0)
    cfg = SimConfig.from_scene(sc)
    ps = SimulationData.from_scene(sc, cfg)
    ns = NeighbourSearch(cfg.domain_size, cfg.support_radius, ps)
    fw = Framework(ps, ns, cfg)
    assert isinstance(fw.pressure, PRJ) and fw.pressure.omega == 0.5
    fw.initialize()
    for _ in range(3):
        fw.forward()
    assert fw.pressure.stats_outer_iters >= 1
    assert fw.pressure.stats_final_density_error < cfg.get_cfg("densityErrorTol", 1e-3)


def test_autotuner_picks_a_candidate_and_caches():
    """The autotuner times every candidate on the actual scenes, picks the
    fastest, and answers the same scene set again from its cache; the engine
    built with the choice steps to the same result as the default shape
    within the FP32 tolerance."""
    from implicitvelocityprojection_b200 import autotune
    scs = [S.random_column(6000, 2.0, seed=101), S.random_column(3000, 1.5, seed=102)]
    opts, res = autotune.tuned_options(scs, force=True)
    assert not res["cached"] and len(res["table"]) == len(autotune.candidates())
    best = min(res["table"], key=lambda r: r["ms_per_step"])
    assert best["shape"].startswith(f"{opts.lanes_per_particle}x{opts.particles_per_block}/")
    bm = res["build_ms"]
    assert set(bm) == {"thread per particle", "warp per cell"} and all(v > 0 for v in bm.values())
    assert {1: "thread per particle", 2: "warp per cell"}[opts.build_kernel] == min(bm, key=bm.get)
    again = autotune.tune(scs)
    assert again["cached"] and again["choice"] == res["choice"]
    a = _engine(scs, lanes_per_particle=opts.lanes_per_particle, particles_per_block=opts.particles_per_block,
                persistent=opts.persistent, row_format=opts.row_format, build_kernel=opts.build_kernel)
    b = _engine(scs)
    for e in (a, b):
        e.build()
        e.step(3)
    for i in range(len(scs)):
        dyn = scs[i].is_dynamic == 1
        assert _rel(a.get("v", i)[dyn], b.get("v", i)[dyn]) < 1e-4


@pytest.mark.parametrize("scene", ["column", "dam", "overflow"])
def test_build_kernels_same_lists(golden_dir, scene):
    """The thread-per-particle build and the warp-per-cell build walk the
    candidates in the same order: identical neighbour lists entry for entry
    (also with truncated lists), density and k equal up to their summation
    order, and steps equal within the FP32 tolerance."""
    if scene == "column":
        sc = S.column_in_box((12, 24, 12), 0.02, (0.4, 1.0, 0.4), seed=4, viscosity_method=1, viscosity_coeff=1e-3)
    elif scene == "dam":
        sc = S.small_dam_break(6000, seed=7)
    else:
        g = _load(golden_dir, "overflow_solve.npz")
        sc = dataclasses.replace(_scene_from_golden(g, g["x"], g["v0"]), max_outer_iters=2, fixed_outer_iters=True)
    a = _engine([sc], build_kernel=1)
    b = _engine([sc], build_kernel=2)
    for e in (a, b):
        e.build()
    ca, ia = a.neighbours(0)
    cb, ib = b.neighbours(0)
    dyn = sc.is_dynamic == 1
    assert np.array_equal(ca, cb) and np.array_equal(ia, ib)
    np.testing.assert_allclose(a.get("density")[dyn], b.get("density")[dyn], rtol=1e-6)
    np.testing.assert_allclose(a.get("k")[dyn], b.get("k")[dyn], rtol=1e-5)
    if scene == "overflow":
        # the truncated block flies apart (tens of m/s within three steps):
        # its steps amplify the summation-order differences of density; the
        # build outputs above are the comparison
        return
    for e in (a, b):
        e.step(3)
    assert _rel(a.get("v")[dyn], b.get("v")[dyn]) < RTOL

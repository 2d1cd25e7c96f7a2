"""Pins the CPU oracle (oracle/ivp_oracle.c) to fixtures produced by executing
the reference's own source (tests/golden/make_golden.py) and to analytic known
answers.  No GPU needed."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from implicitvelocityprojection_b200 import scenes as S

RTOL = 1e-4  # per-particle FP32 tolerance for velocity correction and density


def _load(golden_dir, name):
    return np.load(os.path.join(golden_dir, name))


def _state_from(g, x, v):
    sc = S.Scene(x=x.copy(), v=v.copy(), is_dynamic=g["is_dynamic"], material=g["material"],
                 density0=g["density0"], particle_radius=float(g["particle_radius"]),
                 domain_size=g["domain_size"], dt=float(g["dt"]))
    return O.State.from_scene(sc)


def _rel(a, b, scale=None):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    s = np.abs(b).max() if scale is None else scale
    return np.abs(a - b).max() / max(s, 1e-30)


def test_kernels_bitexact(golden_dir):
    g = _load(golden_dir, "kernels.npz")
    h = float(g["h"])
    W = np.array([O.cubic_kernel(r, h) for r in g["r"]], np.float32)
    assert np.array_equal(W, g["W"]), np.abs(W - g["W"]).max()
    G = np.stack([O.spiky_grad(v, h) for v in g["vecs"]])
    np.testing.assert_allclose(G, g["gradW"], rtol=2e-6, atol=0)


@pytest.mark.parametrize("fast", [False, True])
def test_block_solve(golden_dir, fast):
    g = _load(golden_dir, "block_solve.npz")
    st = _state_from(g, g["x"], g["v0"])
    st.rebuild(only_dynamic=True)
    dyn = st.is_dynamic == 1
    nd = int(dyn.sum())
    assert np.array_equal(st.m, g["m"]) and np.array_equal(st.m_inv, g["m_inv"])
    # neighbour sets identical (integer work: bit-exact as sets)
    off, ids = g["nbr_offsets"], g["nbr_ids"]
    for i in range(nd):
        assert st.neighbour_sets(i) == set(ids[off[i]:off[i + 1]].tolist()), i
    np.testing.assert_allclose(st.density[dyn], g["density"][dyn], rtol=RTOL)
    np.testing.assert_allclose(st.k[dyn], g["k"][dyn], rtol=RTOL)
    d = st.solve(fast=fast, return_d=True)
    assert st.status == O.OK
    assert st.stats_outer_iters == int(g["stats_outer_iters"])
    assert st.stats_pcg_iters == g["stats_pcg_iters"].tolist()
    assert _rel(st.v[dyn], g["v"][dyn]) < RTOL
    assert _rel(d[dyn], g["d"][dyn]) < RTOL
    np.testing.assert_allclose(st.stats_density_errors, g["stats_density_errors"], rtol=1e-3)
    np.testing.assert_allclose(st.stats_final_density_error, float(g["stats_final_density_error"]),
                               rtol=1e-3, atol=1e-7)


@pytest.mark.parametrize("fast", [False, True])
def test_column_steps_one_step_parity(golden_dir, fast):
    """Each reference step, restarted from the reference's previous state."""
    g = _load(golden_dir, "column_steps.npz")
    steps = g["x"].shape[0]
    dyn = g["is_dynamic"] == 1
    mism = 0
    for s in range(steps):
        x_prev = g["x0"] if s == 0 else g["x"][s - 1]
        v_prev = g["v0"] if s == 0 else g["v"][s - 1]
        st = _state_from(g, x_prev, v_prev)
        st.rebuild()
        st.step(fast=fast)
        assert st.status == O.OK
        go = int(g["outer"][s])
        assert abs(st.stats_outer_iters - go) <= 1
        if st.stats_outer_iters != go:
            mism += 1
            continue
        pcg = g["pcg"][g["pcg_off"][s]:g["pcg_off"][s + 1]].tolist()
        assert st.stats_pcg_iters == pcg
        # velocity after the step carries the IP correction d/dt
        assert _rel(st.v[dyn], g["v"][s][dyn]) < RTOL, s
        assert _rel(st.x[dyn], g["x"][s][dyn], scale=1.0) < 1e-6, s
        np.testing.assert_allclose(st.density[dyn], g["density"][s][dyn], rtol=RTOL)
        np.testing.assert_allclose(st.k[dyn], g["k"][s][dyn], rtol=RTOL)
        ref_sets = g["nbr_ids"][g["nbr_ids_off"][s]:g["nbr_ids_off"][s + 1]]
        off = g["nbr_offsets"][s]
        bad = sum(st.neighbour_sets(i) != set(ref_sets[off[i]:off[i + 1]].tolist()) for i in range(int(dyn.sum())))
        # positions agree to ~1e-7 m, so only pairs within rounding of r = h can differ
        assert bad <= 2, (s, bad)
    assert mism <= max(1, steps // 10)


def test_column_trajectory(golden_dir):
    """Free run of the oracle against the reference's trajectory."""
    g = _load(golden_dir, "column_steps.npz")
    dyn = g["is_dynamic"] == 1
    st = _state_from(g, g["x0"], g["v0"])
    st.rebuild()
    for s in range(g["x"].shape[0]):
        st.step(fast=True)
        assert abs(st.stats_outer_iters - int(g["outer"][s])) <= 1
    # chaotic growth of rounding differences stays far below a particle spacing
    assert np.abs(st.x[dyn] - g["x"][-1][dyn]).max() < 1e-4


# ---------------------------------------------------------------- analytic KATs

def _overflow_state(g):
    sc = S.Scene(x=g["x"].copy(), v=g["v0"].copy(), is_dynamic=g["is_dynamic"], material=g["material"],
                 density0=g["density0"], particle_radius=float(g["particle_radius"]),
                 domain_size=g["domain_size"], dt=float(g["dt"]), max_outer_iters=int(g["max_outer_iters"]),
                 fixed_outer_iters=True)
    return O.State.from_scene(sc)


@pytest.mark.parametrize("fast", [False, True])
def test_overflow_solve(golden_dir, fast):
    """Truncated lists (neighbour_search.py:38-51: the first neighborCacheSize
    hits of the hash-grid walk) and the IP solve whose J^T is the scatter form
    over the truncated rows (ip.py:110-121), against the reference's own run.
    FAST mode switches to the scatter form when a list is full."""
    g = _load(golden_dir, "overflow_solve.npz")
    st = _overflow_state(g)
    st.rebuild(only_dynamic=True)
    dyn = st.is_dynamic == 1
    nd = int(dyn.sum())
    assert st.overflow > 0 and int((g["nbr_count"] >= int(g["cache_size"])).sum()) > 0
    off, ids = g["nbr_offsets"], g["nbr_ids"]
    for i in range(nd):
        assert st.neighbour_sets(i) == set(ids[off[i]:off[i + 1]].tolist()), i
    np.testing.assert_allclose(st.density[dyn], g["density"][dyn], rtol=RTOL)
    np.testing.assert_allclose(st.k[dyn], g["k"][dyn], rtol=RTOL)
    st.solve(fast=fast)
    assert st.status == O.OK
    assert st.stats_outer_iters == int(g["stats_outer_iters"])
    assert st.stats_pcg_iters == g["stats_pcg_iters"].tolist()
    assert _rel(st.v[dyn], g["v"][dyn]) < RTOL


def test_overflow_truncation_order():
    """The kept hits of a truncated list are the neighborCacheSize smallest
    (linear cell index with x fastest, particle index) keys over cells of size
    h from the domain origin, the order of the reference's hash-grid walk."""
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "overflow_solve.npz"))
    st = _overflow_state(g)
    st.rebuild(only_dynamic=True)
    x = st.x.astype(np.float32)
    h = np.float32(st.h)
    inv = np.float32(1.0) / h
    dims = np.ceil(st.domain_size.astype(np.float64) / np.float64(h)).astype(np.int64)
    cell = np.clip(np.floor(x * inv).astype(np.int64), 0, dims - 1)
    lin = (cell[:, 2] * dims[1] + cell[:, 1]) * dims[0] + cell[:, 0]
    full = np.where((st.count >= st.cache_size) & (st.is_dynamic == 1))[0]
    assert len(full) > 0
    for i in full[:40]:
        r = x[i] - x
        d2 = ((r[:, 0] * r[:, 0]).astype(np.float32) + (r[:, 1] * r[:, 1]).astype(np.float32)).astype(np.float32)
        d2 = (d2 + (r[:, 2] * r[:, 2]).astype(np.float32)).astype(np.float32)
        hits = np.where((np.sqrt(d2) < h) & (np.arange(st.n) != i))[0]
        assert len(hits) > st.cache_size
        order = np.lexsort((hits, lin[hits]))
        assert set(hits[order][:st.cache_size].tolist()) == st.neighbour_sets(i), i


def test_rest_lattice_density_and_counts():
    """Exact lattice, h = 2d: interior density is 800 kg/m^3 (sum W d^3 = 1 and
    m = 0.8 d^3 rho0).  Lattice offsets with |o|^2 in {1, 2, 3} (6 + 12 + 8 = 26)
    lie strictly inside h; the 6 axis neighbours at exactly 2d sit on the strict
    `< h` boundary and FP32 rounding of the positions admits some of them."""
    sc = S.assemble([S.lattice_block([0.2, 0.2, 0.2], (12, 12, 12), 0.02)], [], particle_radius=0.01,
                    domain_size=[0.7, 0.7, 0.7])
    st = O.State.from_scene(sc)
    st.rebuild()
    x = sc.x
    interior = np.all((x > 0.2 + 0.05) & (x < 0.2 + 11 * 0.02 - 0.05), axis=1)
    assert interior.sum() > 50
    cnt = st.count[interior]
    assert np.all((cnt >= 26) & (cnt <= 32)), np.unique(cnt)
    for i in np.where(interior)[0][:40]:
        near = {j for j in st.neighbour_sets(i)
                if np.sum((x[j] - x[i]) ** 2) < (1.9 * 0.02) ** 2}
        assert len(near) == 26
    # W(2d) = 0, so the boundary neighbours add nothing to the density
    np.testing.assert_allclose(st.density[interior], 800.0, rtol=2e-4)


def test_gradient_antisymmetry():
    rng = np.random.default_rng(0)
    for _ in range(200):
        r = rng.uniform(-0.04, 0.04, 3).astype(np.float32)
        a = O.spiky_grad(r, 0.04)
        b = O.spiky_grad(-r, 0.04)
        assert np.array_equal(a, -b)


def _random_system(seed=0):
    g = S.assemble([S.lattice_block([0.2, 0.2, 0.2], (6, 6, 6), 0.018, jitter=0.05, seed=seed)],
                   [S.cube_shell([0.26, 0.26, 0.26], [0.16, 0.16, 0.16], 0.02)], particle_radius=0.01,
                   domain_size=[0.6, 0.6, 0.6])
    st = O.State.from_scene(g)
    st.rebuild()
    rng = np.random.default_rng(seed)
    d = np.zeros((st.n, 3), np.float32)
    d[st.is_dynamic == 1] = rng.normal(0, 1e-4, size=(int(st.is_dynamic.sum()), 3))
    t, f, dfdt, rhs = st.system(d)
    return st, dfdt, rhs


def test_operator_symmetric_positive_definite():
    st, dfdt, _ = _random_system(1)
    dyn = st.is_dynamic == 1
    rng = np.random.default_rng(2)
    u = np.zeros((st.n, 3))
    w = np.zeros((st.n, 3))
    u[dyn] = rng.normal(size=(int(dyn.sum()), 3))
    w[dyn] = rng.normal(size=(int(dyn.sum()), 3))
    Au, Aw = st.apply_A_f64(dfdt, u), st.apply_A_f64(dfdt, w)
    lhs, rhs = float((w * Au).sum()), float((u * Aw).sum())
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), abs(rhs))
    assert float((u * Au).sum()) > 0.0


def test_fp64_cg_matches_dense_solve():
    st, dfdt, rhs = _random_system(3)
    dyn = np.where(st.is_dynamic == 1)[0]
    nd = dyn.size
    A = np.zeros((3 * nd, 3 * nd))
    for col in range(3 * nd):
        e = np.zeros((st.n, 3))
        e[dyn[col // 3], col % 3] = 1.0
        A[:, col] = st.apply_A_f64(dfdt, e)[dyn].ravel()
    x_dense = np.linalg.solve(A, rhs[dyn].astype(np.float64).ravel())
    x_cg, it = st.cg_f64(dfdt, rhs, rel_tol=1e-14)
    assert it > 0
    np.testing.assert_allclose(x_cg[dyn].ravel(), x_dense, rtol=1e-8, atol=1e-12 * np.abs(x_dense).max())


# ----------------------------------------------------------- Weiler18 viscosity

def _visc_state(g, x, v, visc):
    sc = S.Scene(x=np.array(x, np.float32), v=np.array(v, np.float32), is_dynamic=g["is_dynamic"],
                 material=g["material"], density0=g["density0"], particle_radius=float(g["particle_radius"]),
                 domain_size=g["domain_size"], dt=float(g["dt"]), viscosity_method=1, viscosity_coeff=visc)
    return O.State.from_scene(sc)


@pytest.mark.parametrize("fast", [False, True])
def test_viscosity_solve_golden(golden_dir, fast):
    g = _load(golden_dir, "visc_solve.npz")
    st = _visc_state(g, g["x"], g["v0"], float(g["coeff"]))
    st.rebuild()
    dyn = st.is_dynamic == 1
    np.testing.assert_allclose(st.density[dyn], g["density"][dyn], rtol=RTOL)
    it = st.viscosity_solve(float(g["coeff"]), fast=fast)
    assert it >= 2
    assert _rel(st.v[dyn], g["v"][dyn]) < RTOL
    dv = st.v[dyn] - g["v0"][dyn]
    assert _rel(dv, g["dv"][dyn]) < 1e-3  # the correction itself, relative to its own size


def test_column_visc_steps_one_step_parity(golden_dir):
    g = _load(golden_dir, "column_visc_steps.npz")
    dyn = g["is_dynamic"] == 1
    visc = float(g["viscosity"])
    for s in range(g["x"].shape[0]):
        x_prev = g["x0"] if s == 0 else g["x"][s - 1]
        v_prev = g["v0"] if s == 0 else g["v"][s - 1]
        st = _visc_state(g, x_prev, v_prev, visc)
        st.rebuild()
        st.step(fast=True)
        assert st.status == O.OK
        if st.stats_outer_iters != int(g["outer"][s]):
            continue
        assert _rel(st.v[dyn], g["v"][s][dyn]) < RTOL, s
        assert np.abs(st.x[dyn] - g["x"][s][dyn]).max() < 1e-6, s


# ---------------------------------------------------- Jeske23 surface tension

def _st_state(g, x, v, sigma, visc=0.0):
    sc = S.Scene(x=np.array(x, np.float32), v=np.array(v, np.float32), is_dynamic=g["is_dynamic"],
                 material=g["material"], density0=g["density0"], particle_radius=float(g["particle_radius"]),
                 domain_size=g["domain_size"], dt=float(g["dt"]), viscosity_method=1 if visc > 0 else 0,
                 viscosity_coeff=visc, surface_tension_method=1, surface_tension_coeff=sigma)
    return O.State.from_scene(sc)


@pytest.mark.parametrize("fast", [False, True])
def test_surface_tension_solve_golden(golden_dir, fast):
    g = _load(golden_dir, "st_solve.npz")
    st = _st_state(g, g["x"], g["v0"], float(g["sigma"]))
    st.rebuild()
    dyn = st.is_dynamic == 1
    it, div, b = st.surface_tension_solve(float(g["sigma"]), fast=fast, particle_radius=float(g["particle_radius"]))
    assert it >= 1
    assert _rel(div[dyn], g["div"][dyn]) < 1e-5
    assert _rel(b[dyn], g["b"][dyn]) < 1e-4
    assert _rel(st.v[dyn], g["v"][dyn]) < RTOL
    assert _rel(st.v[dyn] - g["v0"][dyn], g["dv"][dyn]) < 2e-3  # the correction, relative to its own size


def test_column_st_steps_one_step_parity(golden_dir):
    """Steps with surface tension then viscosity then IP (framework.py:417-421)."""
    g = _load(golden_dir, "column_st_steps.npz")
    dyn = g["is_dynamic"] == 1
    sigma, visc = float(g["sigma"]), float(g["viscosity"])
    compared = 0
    for s in range(g["x"].shape[0]):
        x_prev = g["x0"] if s == 0 else g["x"][s - 1]
        v_prev = g["v0"] if s == 0 else g["v"][s - 1]
        st = _st_state(g, x_prev, v_prev, sigma, visc)
        st.rebuild()
        st.step(fast=True)
        assert st.status == O.OK
        if st.stats_outer_iters != int(g["outer"][s]):
            continue
        compared += 1
        assert _rel(st.v[dyn], g["v"][s][dyn]) < RTOL, s
        assert np.abs(st.x[dyn] - g["x"][s][dyn]).max() < 1e-6, s
    assert compared >= g["x"].shape[0] - 1


# --------------------------------------------------------- PRJ (projected Jacobi)

@pytest.mark.parametrize("fast", [False, True])
def test_prj_solve_golden(golden_dir, fast):
    g = _load(golden_dir, "prj_solve.npz")
    st = _state_from(g, g["x"], g["v0"])
    st.rebuild()
    dyn = st.is_dynamic == 1
    assert st.prj_solve(fast=fast, omega=float(g["omega"])) == O.OK
    assert st.stats_outer_iters == int(g["stats_outer_iters"])
    assert _rel(st.v[dyn], g["v"][dyn]) < RTOL
    np.testing.assert_allclose(st.stats_density_errors, g["stats_density_errors"], rtol=1e-4, atol=1e-9)
    assert abs(st.stats_final_density_error - float(g["stats_final_density_error"])) < 1e-7


def test_column_prj_steps_one_step_parity(golden_dir):
    g = _load(golden_dir, "column_prj_steps.npz")
    dyn = g["is_dynamic"] == 1
    for s in range(g["x"].shape[0]):
        x_prev = g["x0"] if s == 0 else g["x"][s - 1]
        v_prev = g["v0"] if s == 0 else g["v"][s - 1]
        st = _state_from(g, x_prev, v_prev)
        st.pressure_method = 0
        st.rebuild()
        st.step(fast=True)
        assert st.status == O.OK
        assert abs(st.stats_outer_iters - int(g["outer"][s])) <= 1
        if st.stats_outer_iters != int(g["outer"][s]):
            continue
        assert _rel(st.v[dyn], g["v"][s][dyn]) < RTOL, s
        assert np.abs(st.x[dyn] - g["x"][s][dyn]).max() < 1e-6, s

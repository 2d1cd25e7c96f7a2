"""Parity at the benchmarked configurations, through the C ABI, against the
oracle (the C restatement of the reference's step, pinned to the golden
fixtures by tests/test_oracle_golden.py).

* the 102,400-particle viscous tall column (the headline workload): neighbour
  sets of every dynamic particle, density and k, at the initial state and
  after 250 steps; restarted steps early and late in the collapse;
* the 524,288-particle dam break (viscosity, surface tension and IP): one
  restarted step from a moving state;
* four scenes of the 64-scene batch, stepped inside the batch;
* the divergence output, the non-positive-definite stop and the bounded
  grid-barrier waits.

Tolerances are those of _gpu_helpers: identical neighbour sets, density, k
and velocity within 1e-4 relative, outer count within +-1, results compared
whenever the iteration counts agree (else re-run with the outer count fixed),
and a floor on the compared steps of every test.
"""
import dataclasses

import numpy as np
import pytest

import _gpu_helpers as H
from oracle import oracle as O
from implicitvelocityprojection_b200 import scenes as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def column():
    return S.tall_column()


@pytest.fixture(scope="module")
def column_runs(column):
    """GPU states of the tall column after 20 and 250 steps."""
    eng = H.engine([column])
    eng.build()
    out = {}
    done = 0
    for k in (20, 250):
        eng.step(k - done)
        done = k
        assert eng.stats(0).status == 0
        out[k] = (eng.get("x").copy(), eng.get("v").copy())
    return out


@pytest.mark.parametrize("at", [0, 250])
def test_tall_column_lists_density_k(column, column_runs, at):
    sc = column if at == 0 else H.with_state(column, *column_runs[at])
    eng = H.engine([sc])
    eng.build()
    st = O.State.from_scene(sc)
    st.rebuild()
    H.check_build(eng, st, sc)
    assert eng.stats(0).overflow_particles == 0 and st.overflow == 0


@pytest.mark.parametrize("at", [20, 250])
def test_tall_column_restarted_steps(column, column_runs, at):
    """Three Framework.forward() steps (viscosity, IP, advection, rebuild),
    each restarted from the oracle's previous state, from the GPU's state
    `at` steps into the collapse."""
    x, v = column_runs[at]
    compared = 0
    for _ in range(3):
        sc = H.with_state(column, x, v)
        ok, eng, st = H.compare_step(sc)
        compared += ok
        x, v = st.x, st.v
    assert compared >= 2, compared


def test_dam_break_restarted_step():
    """The dam break (524,288 fluid particles, Weiler18 viscosity, Jeske23
    surface tension, IP, dt = 0.5 ms): lists, density and k, then restarted
    steps from the GPU's state after ten steps."""
    dam = S.dam_break()
    eng = H.engine([dam])
    eng.build()
    eng.step(10)
    assert eng.stats(0).status == 0
    x, v = eng.get("x").copy(), eng.get("v").copy()
    del eng
    sc = H.with_state(dam, x, v)
    e = H.engine([sc])
    e.build()
    st = O.State.from_scene(sc)
    st.rebuild()
    H.check_build(e, st, sc)
    del e
    compared = 0
    for _ in range(2):
        sc = H.with_state(dam, x, v)
        ok, eng, st = H.compare_step(sc)
        compared += ok
        raw = eng.raw_stats(0)
        assert raw.sum_visc_iters >= 1 and raw.sum_st_iters >= 1
        x, v = st.x, st.v
        del eng
    assert compared >= 1, compared


def test_batch64_scenes_inside_the_batch():
    """Four scenes of the 64-scene batch, each stepped inside the batch, against
    the oracle stepping that scene alone from the same state: lists, density
    and k before the step, then velocity, positions and counts."""
    scs = S.batch_mix(64)
    eng = H.engine(scs)
    eng.build()
    eng.step(3)
    picks = [0, 21, 42, 63]
    pre = {i: (eng.get("x", i).copy(), eng.get("v", i).copy(), eng.get("density", i).copy(), eng.get("k", i).copy())
           for i in picks}
    states = {}
    for i in picks:
        st = O.State.from_scene(H.with_state(scs[i], *pre[i][:2]))
        st.rebuild()
        H.check_build(eng, st, scs[i], scene=i)
        H.same_build_inputs(st, pre[i][2], pre[i][3], scs[i].is_dynamic == 1)
        states[i] = st
    eng.step(1)
    compared = 0
    for i in picks:
        sc = H.with_state(scs[i], *pre[i][:2])
        st = states[i]
        st.step(fast=True)
        gs = eng.stats(i)
        assert gs.status == 0 and st.status == 0
        assert abs(gs.stats_outer_iters - st.stats_outer_iters) <= 1
        if gs.stats_outer_iters != st.stats_outer_iters or gs.stats_pcg_iters != st.stats_pcg_iters:
            continue
        compared += 1
        dyn = sc.is_dynamic == 1
        assert H.rel(eng.get("v", i)[dyn], st.v[dyn]) < H.RTOL, i
        tol = H.XTOL + float(sc.dt) * H.RTOL * float(np.abs(st.v[dyn]).max())
        assert np.abs(eng.get("x", i)[dyn] - st.x[dyn]).max() < tol, i
    assert compared >= 3, compared


def test_divergence_vs_oracle():
    """ps.divergence = max(J v, 0) after the solve (pressure_base.py:449-457)."""
    sc = S.column_in_box((12, 14, 12), 0.018, (0.4, 0.5, 0.4), seed=5)
    rng = np.random.default_rng(2)
    sc.v[sc.is_dynamic == 1] = rng.normal(0, 0.2, size=(sc.n_dynamic, 3)).astype(np.float32)
    ok, eng, st, div = H.compare_solve(sc, divergence=True)
    assert ok
    dyn = sc.is_dynamic == 1
    got = eng.get("divergence")
    assert np.abs(div[dyn]).max() > 0
    assert H.rel(got[dyn], div[dyn]) < H.RTOL
    assert np.all(got[dyn] >= 0)


def test_not_spd_status_and_message():
    """A negative omega makes p^T A p < 0 at the first CG iteration: the solve
    stops with NOT_SPD, leaves v unchanged, and the IP plugin raises the
    reference's message with the iteration and pAp (ip.py:306-309).  The
    oracle stops the same way."""
    from implicitvelocityprojection_b200.config import SimConfig
    from implicitvelocityprojection_b200.framework import Framework
    from implicitvelocityprojection_b200.neighbour_search import NeighbourSearch
    from implicitvelocityprojection_b200.simulation_data import SimulationData
    sc = S.column_in_box((8, 10, 8), 0.018, (0.3, 0.4, 0.3), seed=7, omega=-1.0e4)
    rng = np.random.default_rng(3)
    sc.v[sc.is_dynamic == 1] = rng.normal(0, 0.3, size=(sc.n_dynamic, 3)).astype(np.float32)
    eng = H.engine([sc])
    eng.build()
    v0 = eng.get("v").copy()
    eng.solve()
    s = eng.stats(0)
    assert s.status == 1 and s.last_pap < 0.0 and s.last_cg_iter == 0
    assert np.array_equal(eng.get("v"), v0)
    st = O.State.from_scene(sc)
    st.rebuild()
    st.solve(fast=True)
    assert st.status == O.NOT_SPD
    cfg = SimConfig.from_scene(sc)
    ps = SimulationData.from_scene(sc, cfg)
    ns = NeighbourSearch(cfg.domain_size, cfg.support_radius, ps)
    fw = Framework(ps, ns, cfg)
    fw.initialize()
    fw.pressure.omega = -1.0e4
    with pytest.raises(RuntimeError, match=r"\[IP\] non-positive definite matrix at PCG iter 0 \(pAp=-"):
        fw.pressure.solve(sc.dt)


@pytest.mark.parametrize("n_scenes", [1, 3])
def test_barrier_wait_limit_times_out_then_recovers(golden_dir, n_scenes):
    """Every wait of the persistent solve on a grid barrier is bounded.  With
    the limit set to 1 ns the waits give up at once: the kernel returns, the
    solve reports IVP_ERR_TIMEOUT and the device stays usable.  After
    ivp_reset_counters and the default limit, the same engine solves again
    and matches a fresh engine bit for bit and the reference's fixture.  One
    scene exercises the barrier in which every CTA reduces, three scenes the
    barrier in which the last CTA to arrive reduces."""
    import os
    from implicitvelocityprojection_b200 import _lib
    g = np.load(os.path.join(golden_dir, "block_solve.npz"))
    outer = int(g["stats_outer_iters"])
    # the reference's outer count, fixed, so the fixture comparison below
    # always runs
    base = S.Scene(x=np.array(g["x"], np.float32), v=np.array(g["v0"], np.float32), is_dynamic=g["is_dynamic"],
                   material=g["material"], density0=g["density0"], particle_radius=float(g["particle_radius"]),
                   domain_size=g["domain_size"], dt=float(g["dt"]), max_outer_iters=outer, fixed_outer_iters=True)
    scs = [base] + [S.random_column(3000, 2.0, seed=90 + k) for k in range(n_scenes - 1)]
    eng = H.engine(scs, persistent=True)
    eng.build()
    eng.set_wait_limit(1)
    eng.solve()
    assert eng.raw_stats(0).status == _lib.TIMEOUT
    eng.set_wait_limit(0)
    eng.reset_counters()
    eng.solve()
    s = eng.stats(0)
    assert s.status == 0
    fresh = H.engine(scs, persistent=True)
    fresh.build()
    fresh.solve()
    for i in range(n_scenes):
        assert np.array_equal(eng.get("v", i), fresh.get("v", i)), i
    dyn = base.is_dynamic == 1
    assert s.stats_outer_iters == outer
    assert s.stats_pcg_iters == g["stats_pcg_iters"].tolist()
    assert H.rel(eng.get("v", 0)[dyn], g["v"][dyn]) < H.RTOL


def _overflow_scene(g):
    return S.Scene(x=np.array(g["x"], np.float32), v=np.array(g["v0"], np.float32), is_dynamic=g["is_dynamic"],
                   material=g["material"], density0=g["density0"], particle_radius=float(g["particle_radius"]),
                   domain_size=g["domain_size"], dt=float(g["dt"]), max_outer_iters=int(g["max_outer_iters"]),
                   fixed_outer_iters=True)


@pytest.mark.parametrize("persistent", [True, False])
def test_overflow_lists_and_solve_vs_golden(golden_dir, persistent):
    """A block compressed to 0.7 d: the inner particles have about 96
    neighbours within h, more than neighborCacheSize = 60.  The engine keeps
    the reference's first 60 hits (neighbour_search.py:38-51) and applies the
    exact transpose of the truncated J (the reference's scatter form,
    ip.py:110-121) through its correction list: lists, density, k, CG counts
    and velocity against the reference's own run."""
    import os
    from implicitvelocityprojection_b200.engine import Engine, EngineOptions
    g = np.load(os.path.join(golden_dir, "overflow_solve.npz"))
    sc = _overflow_scene(g)
    eng = Engine([sc], options=EngineOptions(persistent=persistent))
    eng.build()
    dyn = np.where(sc.is_dynamic == 1)[0]
    cnt, ids = eng.neighbours(0)
    off, gids = g["nbr_offsets"], g["nbr_ids"]
    for i in dyn:
        assert set(ids[i, :cnt[i]].tolist()) == set(gids[off[i]:off[i + 1]].tolist()), i
    np.testing.assert_allclose(eng.get("density")[dyn], g["density"][dyn], rtol=H.RTOL)
    np.testing.assert_allclose(eng.get("k")[dyn], g["k"][dyn], rtol=H.RTOL)
    eng.solve()
    s = eng.stats(0)
    raw = eng.raw_stats(0)
    assert s.status == 0 and s.overflow_particles > 0 and raw.fixup_entries > 0
    assert s.stats_outer_iters == int(g["stats_outer_iters"])
    assert s.stats_pcg_iters == g["stats_pcg_iters"].tolist()
    assert H.rel(eng.get("v")[dyn], g["v"][dyn]) < H.RTOL


def test_overflow_paths_and_batch_bitwise(golden_dir):
    """With truncated lists the persistent, per-phase and host-driven paths
    give the same bits over fused steps, and so does the scene inside a batch
    (the corrections are summed in a fixed order)."""
    import os
    g = np.load(os.path.join(golden_dir, "overflow_solve.npz"))
    sc = _overflow_scene(g)
    other = S.random_column(3000, 2.0, seed=95)
    outs = []
    for use_graphs, persistent in ((True, True), (True, False), (False, False), (False, True)):
        e = H.engine([sc], use_graphs=use_graphs, persistent=persistent)
        e.build()
        e.step(3)
        assert e.stats(0).status == 0
        outs.append((e.get("x"), e.get("v")))
    for o in outs[1:]:
        assert np.array_equal(o[0], outs[0][0]) and np.array_equal(o[1], outs[0][1])
    b = H.engine([other, sc])
    b.build()
    b.step(3)
    assert np.array_equal(b.get("v", 1), outs[0][1]) and np.array_equal(b.get("x", 1), outs[0][0])


def test_overflow_step_vs_oracle(golden_dir):
    """Fused steps of the truncated block, each restarted from the oracle's
    state (the oracle's FAST mode switches to the scatter form of J^T when a
    list is full)."""
    import os
    g = np.load(os.path.join(golden_dir, "overflow_solve.npz"))
    base = dataclasses.replace(_overflow_scene(g), max_outer_iters=1000, fixed_outer_iters=False)
    st = O.State.from_scene(base)
    st.rebuild()
    compared = 0
    for _ in range(3):
        ok, eng, st = H.compare_step(H.with_state(base, st.x, st.v))
        compared += ok
    assert compared >= 2, compared


def _walls_only():
    """A one-layer box with no fluid (a scene with no dynamic particle)."""
    d = 0.02
    box = (0.3, 0.3, 0.3)
    margin = 4 * d
    center = [margin + 0.5 * b for b in box]
    shell = S.cube_shell(center, box, d, layers=1)
    return S.assemble([], [shell], particle_radius=0.5 * d, domain_size=[b + 2 * margin for b in box])


@pytest.mark.parametrize("persistent", [True, False])
def test_edge_scenes_in_a_batch(persistent):
    """Empty and ragged inputs in one batch: a scene with no fluid particle,
    a single fluid particle, 65 fluid particles (one full tile and one
    particle), and an ordinary column.  Every scene steps with status OK and
    equals the scene run alone bit for bit; the fluid-free scene runs no
    outer iteration and nothing in it moves; the others match the oracle
    step by step."""
    scs = [_walls_only(),
           S.column_in_box((1, 1, 1), 0.02, (0.2, 0.2, 0.2), seed=3),
           S.column_in_box((5, 13, 1), 0.02, (0.2, 0.4, 0.1), seed=4),
           S.column_in_box((8, 12, 8), 0.02, (0.3, 0.4, 0.3), seed=1)]
    assert [sc.n_dynamic for sc in scs] == [0, 1, 65, 768]
    eng = H.engine(scs, persistent=persistent)
    eng.build()
    eng.step(3)
    for i, sc in enumerate(scs):
        assert eng.stats(i).status == 0, i
        alone = H.engine([sc], persistent=persistent)
        alone.build()
        alone.step(3)
        assert np.array_equal(eng.get("x", i), alone.get("x", 0)), i
        assert np.array_equal(eng.get("v", i), alone.get("v", 0)), i
    empty = eng.stats(0)
    assert empty.stats_outer_iters == 0 and list(empty.stats_pcg_iters) == []
    assert np.array_equal(eng.get("x", 0), scs[0].x) and not np.any(eng.get("v", 0))
    compared = 0
    for sc in scs[1:]:
        state = sc
        for _ in range(2):
            ok, e, st = H.compare_step(state, persistent=persistent)
            compared += ok
            state = H.with_state(sc, e.get("x"), e.get("v"))
    assert compared >= 5, compared

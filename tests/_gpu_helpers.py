"""Helpers of the GPU parity tests: the engine and the oracle stepped from the
same state, and the comparisons the tolerances below define.

Tolerances: neighbour sets identical (integer work);
per-particle density, k and velocity within 1e-4 relative in FP32 (relative
to the largest magnitude in the scene); outer-iteration count within +-1;
results compared whenever the iteration counts agree.  When they do not (an
error or residual within rounding of its tolerance), both sides are re-run
with the outer-iteration count fixed at the engine's (the reference's
fixedOuterIters, ip.py:364-370) and compared if their CG counts then agree.
Every caller puts a floor on the number of compared steps, so a test can
never pass while comparing nothing.

A step is compared in two parts.  The build (neighbour sets, density, k) is
checked against the oracle's rebuild of the same positions; the solve then
starts, on both sides, from the engine's density and k.  The reason: the
constraint t = rho - rho0 + J d is a small difference of large numbers
(rho ~ 1000 kg/m^3 carries about 4e-4 kg/m^3 of FP32 rounding that depends on
the summation order), and the reference's derivative switch
dfdt = (t >= 1e-6) (ip.py:166) is discontinuous.  On a column of 102,400
particles a few constraints sit within that rounding of the switch, so two
valid FP32 evaluations of the reference's own algorithm can disagree on them
and change their operator rows; handing both sides the same density removes
that ambiguity while every other quantity is still computed independently.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from oracle import oracle as O

RTOL = 1e-4
XTOL = 1e-6  # metres: positions after one step (x = x_old + dt v, FP32)


def engine(scs, **opt):
    from implicitvelocityprojection_b200.engine import Engine, EngineOptions
    return Engine(list(scs), options=EngineOptions(**opt) if opt else None)


def rel(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def with_state(sc, x, v, **over):
    return dataclasses.replace(sc, x=np.array(x, np.float32), v=np.array(v, np.float32), **over)


def sets_equal(cnt_a, ids_a, cnt_b, ids_b, rows) -> np.ndarray:
    """Per row of `rows`: do the two neighbour lists hold the same set?
    ids_* are (n, cache) arrays, cnt_* the list lengths."""
    cache = ids_a.shape[1]
    assert ids_b.shape[1] == cache
    big = np.iinfo(np.int32).max
    k = np.arange(cache)[None, :]
    a = np.where(k < cnt_a[rows][:, None], ids_a[rows], big)
    b = np.where(k < cnt_b[rows][:, None], ids_b[rows], big)
    return (cnt_a[rows] == cnt_b[rows]) & np.all(np.sort(a, axis=1) == np.sort(b, axis=1), axis=1)


def oracle_lists(st):
    """(count, ids as (n, cache)) of an oracle state, counts capped at the cache."""
    c = st.cache_size
    return np.minimum(st.count, c), st.ids.reshape(st.n, c)


def check_build(eng, st, sc, scene=0):
    """Neighbour sets, density and k of a freshly built engine scene against
    the oracle's rebuild of the same positions."""
    dyn = np.where(sc.is_dynamic == 1)[0]
    cnt, ids = eng.neighbours(scene)
    oc, oi = oracle_lists(st)
    same = sets_equal(cnt, ids, oc, oi, dyn)
    assert same.all(), f"{int((~same).sum())} of {len(dyn)} neighbour sets differ, first {dyn[~same][:5]}"
    np.testing.assert_allclose(eng.get("density", scene)[dyn], st.density[dyn], rtol=RTOL)
    np.testing.assert_allclose(eng.get("k", scene)[dyn], st.k[dyn], rtol=RTOL)


def _counts(gs, raw, st) -> bool:
    return (gs.stats_outer_iters == st.stats_outer_iters and gs.stats_pcg_iters == st.stats_pcg_iters
            and int(raw.sum_visc_iters) == st.visc_iters and int(raw.sum_st_iters) == st.st_iters)


def same_build_inputs(st, density, k, dyn):
    """The oracle state continues from the engine's density and k (checked
    against the oracle's own by check_build)."""
    st.density[dyn] = density[dyn]
    st.k[dyn] = k[dyn]


def _step_both(sc, opts):
    eng = engine([sc], **opts)
    eng.build()
    st = O.State.from_scene(sc)
    st.rebuild()
    check_build(eng, st, sc)
    dyn = sc.is_dynamic == 1
    same_build_inputs(st, eng.get("density"), eng.get("k"), dyn)
    eng.step(1)
    gs, raw = eng.stats(0), eng.raw_stats(0)
    st.step(fast=True)
    return eng, gs, raw, st


def compare_step(sc, check_x=True, **opts):
    """One Framework.forward() step of `sc` on the engine and on the oracle
    from the same state.  Returns (compared, engine, oracle state)."""
    eng, gs, raw, st = _step_both(sc, opts)
    assert gs.status == 0 and st.status == 0, (gs.status, st.status)
    assert abs(gs.stats_outer_iters - st.stats_outer_iters) <= 1, (gs.stats_outer_iters, st.stats_outer_iters)
    if not _counts(gs, raw, st):
        fixed = dataclasses.replace(sc, fixed_outer_iters=True, max_outer_iters=gs.stats_outer_iters)
        eng, gs, raw, st = _step_both(fixed, opts)
        assert gs.status == 0 and st.status == 0
        if not _counts(gs, raw, st):
            return False, eng, st
    dyn = sc.is_dynamic == 1
    ev = rel(eng.get("v")[dyn], st.v[dyn])
    assert ev < RTOL, f"velocity off by {ev:.3e} relative"
    if check_x:
        # x = x_old + dt v: the velocity tolerance carried into the positions
        tol = XTOL + float(sc.dt) * RTOL * float(np.abs(st.v[dyn]).max())
        ex = float(np.abs(eng.get("x")[dyn] - st.x[dyn]).max())
        assert ex < tol, f"positions off by {ex:.3e} m (tolerance {tol:.3e})"
    # the step's own rebuild (density, k) ran on the two sides' slightly
    # different new positions; the build is compared from identical positions
    # at the start of every restarted step (check_build), where a truncated
    # list's kept hits do not depend on which cell a particle just moved into
    return True, eng, st


def compare_solve(sc, divergence=False, **opts):
    """One IP.solve of `sc` (lists built from its positions) on the engine and
    on the oracle.  Returns (compared, engine, oracle state, oracle divergence)."""

    def both(s):
        from implicitvelocityprojection_b200.engine import Engine, EngineOptions
        e = Engine([s], options=EngineOptions(**opts) if opts else None, divergence=divergence)
        e.build()
        o = O.State.from_scene(s)
        o.rebuild()
        check_build(e, o, s)
        same_build_inputs(o, e.get("density"), e.get("k"), s.is_dynamic == 1)
        e.solve()
        div = o.solve(fast=True, divergence=divergence)
        return e, e.stats(0), o, div

    eng, gs, st, div = both(sc)
    assert gs.status == 0 and st.status == 0, (gs.status, st.status)
    assert abs(gs.stats_outer_iters - st.stats_outer_iters) <= 1
    if gs.stats_outer_iters != st.stats_outer_iters or gs.stats_pcg_iters != st.stats_pcg_iters:
        fixed = dataclasses.replace(sc, fixed_outer_iters=True, max_outer_iters=gs.stats_outer_iters)
        eng, gs, st, div = both(fixed)
        if gs.stats_outer_iters != st.stats_outer_iters or gs.stats_pcg_iters != st.stats_pcg_iters:
            return False, eng, st, div
    dyn = sc.is_dynamic == 1
    ev = rel(eng.get("v")[dyn], st.v[dyn])
    assert ev < RTOL, f"velocity off by {ev:.3e} relative"
    return True, eng, st, div

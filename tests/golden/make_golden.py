"""Generate golden fixtures by executing the reference's own source.

Runs the reference's Python modules (`scripts/framework.py`,
`scripts/sim/forces/pressure/ip.py`, `pressure_base.py`, `neighbour_search.py`,
`sph_kernel.py`, `math_utils.py`, `simulation_data.py`, `boundary.py`) on the
NumPy FP32 stand-in for the Warp runtime in `wpshim/`, and stores the results
as small `.npz` fixtures next to this script.  It needs a checkout of the
reference, given as `--reference PATH` or in the environment variable
IVP_REFERENCE, and only runs where that checkout exists; the fixtures it
writes are committed and are all that the tests read.

Fixtures
--------
kernels.npz       cubic_kernel / spiky_kernel_derivative at sampled radii;
visc_solve.npz    one Weiler18 implicit-viscosity solve (weiler18.py:371-401) on
                  the moving block;
column_visc_steps.npz  Framework.forward() steps with Weiler18 viscosity on;
prj_solve.npz     one PRJ solve (prj.py:296-340) on the moving block;
column_prj_steps.npz  Framework.forward() steps with PRJ as the pressure solver;
scene_ingest.npz  the reference scene loader's particles for scene_blocks.json;
st_solve.npz      one Jeske23 implicit surface-tension solve (jeske23.py:585-655)
                  on the moving block;
column_st_steps.npz  Framework.forward() steps with Jeske23 surface tension and
                  Weiler18 viscosity on (surface tension runs first,
                  framework.py:417-421);
overflow_solve.npz  the reference's neighbour build, density, Aii and one IP
                  solve (two fixed outer updates) on a block compressed to
                  0.7 d, whose inner lists are truncated at neighborCacheSize;
block_solve.npz   one IP solve (ip.py:331-404) from a compressed, moving block
                  inside a static box, after the reference's neighbour build,
                  density and Aii;
column_steps.npz  successive Framework.forward() steps (framework.py:423-544)
                  of a small column collapse with IP and no viscosity or
                  surface tension (their solver objects are replaced by no-ops,
                  which is what "off" means for these configurations).

Usage:  python tests/golden/make_golden.py --reference PATH [--steps N]
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _setup(reference: str):
    sys.path.insert(0, os.path.join(HERE, "wpshim"))
    sys.path.insert(0, reference)
    sys.path.insert(0, REPO)


def _scene_block():
    from implicitvelocityprojection_b200 import scenes as S
    d = 0.02
    rng = np.random.default_rng(7)
    # 5 x 6 x 5 fluid block at 0.9 d spacing (compressed), moving down and sideways
    lower = [0.12, 0.10, 0.12]
    fluid = S.lattice_block(lower, (5, 6, 5), 0.9 * d, jitter=0.01, seed=11)
    box = (0.28, 0.30, 0.28)
    center = [0.08 + 0.5 * b for b in box]
    shell = S.cube_shell(center, box, d, layers=1)
    domain = [b + 0.16 for b in box]
    sc = S.assemble([fluid], [shell], particle_radius=0.5 * d, domain_size=domain, name="block")
    nf = fluid.shape[0]
    sc.v[:nf] = (rng.uniform(-0.05, 0.05, size=(nf, 3)) + np.array([0.1, -0.6, 0.0])).astype(np.float32)
    return sc


def _scene_column():
    from implicitvelocityprojection_b200 import scenes as S
    return S.column_in_box((5, 9, 5), 0.02, (0.2, 0.26, 0.2), jitter=0.01, seed=3, name="column")


class _Cfg:
    """Stand-in for config_builder.SimConfig with the keys the hot path reads."""


def _make_objects(sc, viscosity_method=0, viscosity_coeff=0.0, st_method=0, st_coeff=0.0, pressure_method=1):
    from scripts.io.config_builder import SimConfig
    from scripts.sim.simulation_data import SimulationData
    from scripts.sim.neighbour_search import NeighbourSearch

    conf = sc.config()
    conf["pressureMethod"] = pressure_method
    cfg = SimConfig(domain_size=tuple(float(s) for s in sc.domain_size), domain_start=(0.0, 0.0, 0.0),
                    particle_radius=sc.particle_radius, dt=sc.dt, density0=1000.0,
                    gravity=tuple(sc.gravity), viscosity_method=viscosity_method, surface_tension_method=st_method,
                    viscosity_coeff=viscosity_coeff, surface_tension_coeff=st_coeff,
                    scene_data={"Configuration": conf})
    ps = SimulationData(cfg)
    ps.allocate(sc.n)
    nf = sc.n_dynamic
    color = np.zeros((sc.n, 3), np.int32)
    # fluid block then static shell, as the scene loader populates them
    ps.add_particles(0, nf, sc.x[:nf], sc.v[:nf], sc.density0[:nf], sc.material[:nf], sc.is_dynamic[:nf],
                     color[:nf])
    ps.add_particles(1, sc.n - nf, sc.x[nf:], sc.v[nf:], sc.density0[nf:], sc.material[nf:],
                     sc.is_dynamic[nf:], color[nf:])
    ns = NeighbourSearch(tuple(float(s) for s in sc.domain_size), ps.support_radius)
    return cfg, ps, ns


def _lists(ps, n_dyn):
    cnt = ps.neighbor_count.numpy()[:n_dyn].astype(np.int32)
    ids = ps.neighbor_ids.numpy().reshape(-1, ps.cache_size)[:n_dyn]
    off = np.zeros(n_dyn + 1, np.int64)
    off[1:] = np.cumsum(np.minimum(cnt, ps.cache_size))
    flat = np.concatenate([np.sort(ids[i, :min(cnt[i], ps.cache_size)]) for i in range(n_dyn)]).astype(np.int32)
    return cnt, off, flat


def make_kernels(out):
    from scripts.sim import sph_kernel as K
    import warp as wp
    h = np.float32(0.04)
    r = np.linspace(0.0, 0.045, 91, dtype=np.float32)
    W = np.array([K.cubic_kernel(np.float32(ri), h) for ri in r], dtype=np.float32)
    rng = np.random.default_rng(1)
    vecs = rng.uniform(-0.04, 0.04, size=(64, 3)).astype(np.float32)
    vecs[0] = 0.0
    G = np.stack([K.spiky_kernel_derivative(wp.vec3(*v), h) for v in vecs]).astype(np.float32)
    np.savez_compressed(out, h=h, r=r, W=W, vecs=vecs, gradW=G)


def make_block_solve(out):
    from scripts.sim.forces.pressure.ip import IP
    sc = _scene_block()
    cfg, ps, ns = _make_objects(sc)
    solver = IP(ps, ns, cfg)
    t0 = time.time()
    ns.build(ps.x, ps.particle_num)
    ns.build_cache(ps.x, ps.particle_num, int(ps.cache_size), ps.neighbor_count, ps.neighbor_ids,
                   ps.neighbor_gradW)
    solver.compute_density()
    solver.compute_Aii()
    nd = sc.n_dynamic
    cnt, off, flat = _lists(ps, nd)
    density = ps.density.numpy().copy()
    k = solver.k.numpy().copy()
    solver.solve(sc.dt)
    print(f"block_solve: {time.time() - t0:.1f}s outer={solver.stats_outer_iters} pcg={solver.stats_pcg_iters}")
    np.savez_compressed(
        out, x=sc.x, v0=sc.v, is_dynamic=sc.is_dynamic, material=sc.material, density0=sc.density0,
        particle_radius=np.float64(sc.particle_radius), domain_size=sc.domain_size, dt=np.float64(sc.dt),
        nbr_count=cnt, nbr_offsets=off, nbr_ids=flat, density=density, k=k,
        v=ps.v.numpy().copy(), d=solver.dx.numpy().copy(), m=ps.m.numpy().copy(), m_inv=ps.m_inv.numpy().copy(),
        divergence=ps.divergence.numpy().copy(),
        stats_density_errors=np.array(solver.stats_density_errors, np.float64),
        stats_pcg_iters=np.array(solver.stats_pcg_iters, np.int32),
        stats_outer_iters=np.int32(solver.stats_outer_iters),
        stats_final_density_error=np.float64(solver.stats_final_density_error))


def _scene_overflow():
    """A 7 x 7 x 7 fluid block at 0.7 d spacing, moving, inside a static box:
    about 96 neighbours within h at the centre, so the lists of the inner
    particles are truncated at neighborCacheSize = 60."""
    from implicitvelocityprojection_b200 import scenes as S
    d = 0.02
    rng = np.random.default_rng(17)
    fluid = S.lattice_block([0.14, 0.12, 0.14], (7, 7, 7), 0.7 * d, jitter=0.01, seed=19)
    box = (0.3, 0.3, 0.3)
    center = [0.08 + 0.5 * b for b in box]
    shell = S.cube_shell(center, box, d, layers=1)
    domain = [b + 0.16 for b in box]
    sc = S.assemble([fluid], [shell], particle_radius=0.5 * d, domain_size=domain, name="overflow_block",
                    max_outer_iters=2, fixed_outer_iters=True)
    nf = fluid.shape[0]
    sc.v[:nf] = (rng.uniform(-0.05, 0.05, size=(nf, 3)) + np.array([0.0, -0.3, 0.1])).astype(np.float32)
    return sc


def make_overflow_solve(out):
    """The reference's neighbour build, density, Aii and one IP solve (two
    fixed outer updates) on a block whose inner lists are truncated at
    neighborCacheSize: the reference keeps the first 60 hits of its hash-grid
    walk and applies J^T in scatter form over the truncated rows
    (ip.py:110-121)."""
    from scripts.sim.forces.pressure.ip import IP
    sc = _scene_overflow()
    cfg, ps, ns = _make_objects(sc)
    solver = IP(ps, ns, cfg)
    t0 = time.time()
    ns.build(ps.x, ps.particle_num)
    ns.build_cache(ps.x, ps.particle_num, int(ps.cache_size), ps.neighbor_count, ps.neighbor_ids,
                   ps.neighbor_gradW)
    solver.compute_density()
    solver.compute_Aii()
    nd = sc.n_dynamic
    cnt, off, flat = _lists(ps, nd)
    full = int((cnt >= ps.cache_size).sum())
    density = ps.density.numpy().copy()
    k = solver.k.numpy().copy()
    solver.solve(sc.dt)
    print(f"overflow_solve: {time.time() - t0:.1f}s full rows={full} outer={solver.stats_outer_iters} "
          f"pcg={solver.stats_pcg_iters}")
    np.savez_compressed(
        out, x=sc.x, v0=sc.v, is_dynamic=sc.is_dynamic, material=sc.material, density0=sc.density0,
        particle_radius=np.float64(sc.particle_radius), domain_size=sc.domain_size, dt=np.float64(sc.dt),
        max_outer_iters=np.int32(sc.max_outer_iters), cache_size=np.int32(ps.cache_size),
        nbr_count=cnt, nbr_offsets=off, nbr_ids=flat, density=density, k=k,
        v=ps.v.numpy().copy(), m=ps.m.numpy().copy(),
        stats_density_errors=np.array(solver.stats_density_errors, np.float64),
        stats_pcg_iters=np.array(solver.stats_pcg_iters, np.int32),
        stats_outer_iters=np.int32(solver.stats_outer_iters),
        stats_final_density_error=np.float64(solver.stats_final_density_error))


class _NoForce:
    def solve(self, *a, **k):
        pass

    def reset(self):
        pass


def make_visc_solve(out, coeff=0.05):
    """One Weiler18.solve (weiler18.py:371-401) on the moving block."""
    from scripts.sim.forces.pressure.ip import IP
    from scripts.sim.forces.non_pressure.viscosity.weiler18 import Weiler18
    sc = _scene_block()
    cfg, ps, ns = _make_objects(sc, 1, coeff)
    solver = IP(ps, ns, cfg)
    ns.build(ps.x, ps.particle_num)
    ns.build_cache(ps.x, ps.particle_num, int(ps.cache_size), ps.neighbor_count, ps.neighbor_ids,
                   ps.neighbor_gradW)
    solver.compute_density()
    visc = Weiler18(ps, ns, cfg)
    v_before = ps.v.numpy().copy()
    t0 = time.time()
    visc.solve(coeff, sc.dt)
    print(f"visc_solve: {time.time() - t0:.1f}s")
    np.savez_compressed(
        out, x=sc.x, v0=v_before, is_dynamic=sc.is_dynamic, material=sc.material, density0=sc.density0,
        particle_radius=np.float64(sc.particle_radius), domain_size=sc.domain_size, dt=np.float64(sc.dt),
        coeff=np.float64(coeff), density=ps.density.numpy().copy(), v=ps.v.numpy().copy(),
        dv=visc.dv.numpy().copy())


def make_st_solve(out, sigma=0.05):
    """One Jeske23.solve (jeske23.py:585-655) on the moving block."""
    from scripts.sim.forces.pressure.ip import IP
    from scripts.sim.forces.non_pressure.surface_tension.jeske23 import Jeske23
    sc = _scene_block()
    cfg, ps, ns = _make_objects(sc, 0, 0.0, 1, sigma)
    solver = IP(ps, ns, cfg)
    ns.build(ps.x, ps.particle_num)
    ns.build_cache(ps.x, ps.particle_num, int(ps.cache_size), ps.neighbor_count, ps.neighbor_ids,
                   ps.neighbor_gradW)
    solver.compute_density()
    st = Jeske23(ps, ns, cfg)
    v_before = ps.v.numpy().copy()
    t0 = time.time()
    st.solve(sigma, sigma, sc.dt)
    print(f"st_solve: {time.time() - t0:.1f}s")
    np.savez_compressed(
        out, x=sc.x, v0=v_before, is_dynamic=sc.is_dynamic, material=sc.material, density0=sc.density0,
        particle_radius=np.float64(sc.particle_radius), domain_size=sc.domain_size, dt=np.float64(sc.dt),
        sigma=np.float64(sigma), density=ps.density.numpy().copy(), v=ps.v.numpy().copy(),
        dv=st.dv.numpy().copy(), div=st.div_arr.numpy().copy(), b=st.b_st.numpy().copy())


def make_prj_solve(out):
    """One PRJ.solve (prj.py:296-340) on the moving block, after the
    reference's neighbour build, density and Aii."""
    from scripts.sim.forces.pressure.prj import PRJ
    sc = _scene_block()
    cfg, ps, ns = _make_objects(sc)
    solver = PRJ(ps, ns, cfg)
    ns.build(ps.x, ps.particle_num)
    ns.build_cache(ps.x, ps.particle_num, int(ps.cache_size), ps.neighbor_count, ps.neighbor_ids,
                   ps.neighbor_gradW)
    solver.compute_density()
    solver.compute_Aii()
    t0 = time.time()
    solver.solve(sc.dt)
    print(f"prj_solve: {time.time() - t0:.1f}s passes={solver.stats_outer_iters}")
    np.savez_compressed(
        out, x=sc.x, v0=sc.v, is_dynamic=sc.is_dynamic, material=sc.material, density0=sc.density0,
        particle_radius=np.float64(sc.particle_radius), domain_size=sc.domain_size, dt=np.float64(sc.dt),
        v=ps.v.numpy().copy(), omega=np.float64(solver.omega),
        stats_density_errors=np.array(solver.stats_density_errors, np.float64),
        stats_outer_iters=np.int32(solver.stats_outer_iters),
        stats_final_density_error=np.float64(solver.stats_final_density_error))


def make_scene_ingest(out):
    """The reference's scene loader (scene_loader.py:70-545) on
    scene_blocks.json: fluid blocks, a generated cube body, boundary walls."""
    from scripts.io.config_builder import SimConfig
    from scripts.io.scene_loader import SceneLoader
    from scripts.sim.simulation_data import SimulationData
    cfg = SimConfig.from_json(os.path.join(HERE, "scene_blocks.json"))
    loader = SceneLoader(cfg)
    data = loader.prepare_scene()
    ps = SimulationData(cfg)
    loader.populate_scene(ps, data)
    n = int(ps.particle_num)
    np.savez_compressed(
        out, x=ps.x.numpy()[:n].copy(), v=ps.v.numpy()[:n].copy(), is_dynamic=ps.is_dynamic.numpy()[:n].copy(),
        material=ps.material.numpy()[:n].copy(), density0=ps.density0.numpy()[:n].copy(),
        m=ps.m.numpy()[:n].copy(), object_id=ps.object_id.numpy()[:n].copy(),
        domain_size=np.asarray(cfg.domain_size, np.float32), particle_radius=np.float64(cfg.particle_radius))


def make_column_steps(out, steps, viscosity=0.0, sigma=0.0, pressure_method=1):
    from scripts.framework import Framework
    sc = _scene_column()
    cfg, ps, ns = _make_objects(sc, 1 if viscosity > 0 else 0, viscosity, 1 if sigma > 0 else 0, sigma,
                                pressure_method)
    fw = Framework(ps, ns, cfg)
    if viscosity <= 0:
        fw.viscosity = _NoForce()
    if sigma <= 0:
        fw.surface_tension = _NoForce()
    fw.initialize()
    nd = sc.n_dynamic
    rec = {k: [] for k in ("x", "v", "density", "k", "err", "pcg", "outer", "final_err", "cnt", "off", "ids")}
    t0 = time.time()
    for s in range(steps):
        fw.forward()
        p = fw.pressure
        cnt, off, flat = _lists(ps, nd)
        rec["x"].append(ps.x.numpy().copy())
        rec["v"].append(ps.v.numpy().copy())
        rec["density"].append(ps.density.numpy().copy())
        rec["k"].append(p.k.numpy().copy())
        rec["err"].append(np.array(p.stats_density_errors, np.float64))
        rec["pcg"].append(np.array(getattr(p, "stats_pcg_iters", []), np.int32))
        rec["outer"].append(p.stats_outer_iters)
        rec["final_err"].append(p.stats_final_density_error)
        rec["cnt"].append(cnt)
        rec["off"].append(off)
        rec["ids"].append(flat)
        print(f"  step {s}: outer={p.stats_outer_iters} pcg={getattr(p, 'stats_pcg_iters', [])} "
              f"err={['%.2e' % e for e in p.stats_density_errors]} ({time.time() - t0:.0f}s)")

    def ragged(lst, dt):
        off = np.zeros(len(lst) + 1, np.int64)
        off[1:] = np.cumsum([len(a) for a in lst])
        return np.concatenate(lst).astype(dt) if lst else np.zeros(0, dt), off

    err, err_off = ragged(rec["err"], np.float64)
    pcg, pcg_off = ragged(rec["pcg"], np.int32)
    ids, ids_off = ragged(rec["ids"], np.int32)
    np.savez_compressed(
        out, x0=sc.x, v0=sc.v, is_dynamic=sc.is_dynamic, material=sc.material, density0=sc.density0,
        particle_radius=np.float64(sc.particle_radius), domain_size=sc.domain_size, dt=np.float64(sc.dt),
        gravity=np.asarray(sc.gravity, np.float32), viscosity=np.float64(viscosity), sigma=np.float64(sigma),
        x=np.stack(rec["x"]), v=np.stack(rec["v"]), density=np.stack(rec["density"]), k=np.stack(rec["k"]),
        err=err, err_off=err_off, pcg=pcg, pcg_off=pcg_off, outer=np.array(rec["outer"], np.int32),
        final_err=np.array(rec["final_err"], np.float64), nbr_count=np.stack(rec["cnt"]),
        nbr_offsets=np.stack(rec["off"]), nbr_ids=ids, nbr_ids_off=ids_off)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("IVP_REFERENCE"),
                    help="checkout of the reference (default: $IVP_REFERENCE)")
    ap.add_argument("--steps", type=int, default=12)
    ap.add_argument("--only", default=None)
    a = ap.parse_args()
    if not a.reference:
        sys.exit("give the reference checkout with --reference PATH or IVP_REFERENCE")
    if not os.path.isdir(os.path.join(a.reference, "scripts")):
        sys.exit(f"reference checkout not found at {a.reference}")
    _setup(a.reference)
    jobs = {"kernels": lambda: make_kernels(os.path.join(HERE, "kernels.npz")),
            "block_solve": lambda: make_block_solve(os.path.join(HERE, "block_solve.npz")),
            "overflow_solve": lambda: make_overflow_solve(os.path.join(HERE, "overflow_solve.npz")),
            "column_steps": lambda: make_column_steps(os.path.join(HERE, "column_steps.npz"), a.steps),
            "visc_solve": lambda: make_visc_solve(os.path.join(HERE, "visc_solve.npz")),
            "column_visc_steps": lambda: make_column_steps(os.path.join(HERE, "column_visc_steps.npz"), 10,
                                                           viscosity=0.01),
            "st_solve": lambda: make_st_solve(os.path.join(HERE, "st_solve.npz")),
            "scene_ingest": lambda: make_scene_ingest(os.path.join(HERE, "scene_ingest.npz")),
            "prj_solve": lambda: make_prj_solve(os.path.join(HERE, "prj_solve.npz")),
            "column_prj_steps": lambda: make_column_steps(os.path.join(HERE, "column_prj_steps.npz"), 6,
                                                          pressure_method=0),
            "column_st_steps": lambda: make_column_steps(os.path.join(HERE, "column_st_steps.npz"), 8,
                                                         viscosity=0.01, sigma=0.05)}
    for name, job in jobs.items():
        if a.only and name != a.only:
            continue
        job()
        print("wrote", name)


if __name__ == "__main__":
    main()

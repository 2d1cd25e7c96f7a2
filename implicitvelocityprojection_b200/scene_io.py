"""Scene ingestion: the reference's JSON scene format to a `scenes.Scene`.

Restates `SceneLoader.prepare_scene` / `populate_scene`
(scripts/io/scene_loader.py:70-429) and its generators for the parts that need
no mesh library:

- `Configuration`: particleRadius, timeStepSize, gravitation, domainStart /
  domainEnd, density0, densityErrorTol, omega, tol_pcg, maxOuterIters,
  neighborCacheSize, viscosity and surface-tension method / coefficient
  (config_builder.py:10-157, pressure_base.py:314-317);
- `FluidBlocks`: lattice blocks with translation and scale
  (scene_loader.py:89-102, 319-336; SimulationData.add_cube,
  simulation_data.py:290-358);
- `GeneratedBodies` of type "cube": hollow box shells, edges repeated on every
  face (scene_loader.py:447-492);
- `Configuration.boundaryLayers`: particle walls on the domain faces
  (scene_loader.py:494-545).

Particles are appended in the reference's order (fluid blocks, generated
bodies, boundary walls), with its dtypes at every step, so positions are
bit-identical to the reference loader's.  `RigidBodies` / `FluidBodies` are
OBJ meshes voxelised with trimesh, which this package does not use: an entry
must then carry its points already voxelised (`"voxelizedPoints"`, world
coordinates) or loading raises.  `SolidBodies` and `ScheduledSpawns` belong to
the elasticity and spawn systems, which are out of this path's scope.
"""
from __future__ import annotations

import json
from typing import Union

import numpy as np

from .scenes import MATERIAL_FLUID, MATERIAL_RIGID, Scene


def _cube_block(lower, size, diameter: float) -> np.ndarray:
    """SimulationData.add_cube positions (simulation_data.py:316-328)."""
    axes = [np.arange(lower[i], lower[i] + size[i], diameter) for i in range(3)]
    g = np.array(np.meshgrid(*axes, sparse=False, indexing="ij"), dtype=np.float32)
    return g.reshape(-1, int(np.prod(g.shape[1:]))).transpose()


def _shell(start, end, diameter: float, layers: int) -> np.ndarray:
    """Six faces per layer, offset outwards by one diameter per layer: the
    generated cube body (scene_loader.py:467-490) and the domain walls
    (scene_loader.py:505-541) share this construction."""
    out = []
    for layer in range(layers):
        off = layer * diameter
        s = start - off
        e = end + off
        xs = np.arange(s[0], e[0] + diameter * 0.5, diameter)
        ys = np.arange(s[1], e[1] + diameter * 0.5, diameter)
        zs = np.arange(s[2], e[2] + diameter * 0.5, diameter)
        gx, gz = np.meshgrid(xs, zs, indexing="ij")
        out.append(np.stack([gx.ravel(), np.full(gx.size, s[1]), gz.ravel()], axis=1))
        out.append(np.stack([gx.ravel(), np.full(gx.size, e[1]), gz.ravel()], axis=1))
        gy, gz2 = np.meshgrid(ys, zs, indexing="ij")
        out.append(np.stack([np.full(gy.size, s[0]), gy.ravel(), gz2.ravel()], axis=1))
        out.append(np.stack([np.full(gy.size, e[0]), gy.ravel(), gz2.ravel()], axis=1))
        gx2, gy2 = np.meshgrid(xs, ys, indexing="ij")
        out.append(np.stack([gx2.ravel(), gy2.ravel(), np.full(gx2.size, s[2])], axis=1))
        out.append(np.stack([gx2.ravel(), gy2.ravel(), np.full(gx2.size, e[2])], axis=1))
    return np.concatenate(out, axis=0).astype(np.float32)


def load_scene(src: Union[str, dict], name: str = None) -> Scene:
    """A `Scene` from a scene file path or its parsed dict."""
    if isinstance(src, str):
        with open(src, "r") as f:
            data = json.load(f)
        if name is None:
            import pathlib
            name = pathlib.Path(src).stem
    else:
        data = src
    conf = data.get("Configuration", {})
    unsupported = [k for k in ("SolidBodies", "ScheduledSpawns") if data.get(k)]
    if unsupported:
        raise NotImplementedError(f"{', '.join(unsupported)}: elasticity and scheduled spawns are outside this package")
    radius = float(conf.get("particleRadius", 0.01))
    diameter = 2.0 * radius  # config_builder.py:46-52
    rho0 = float(conf.get("density0", 1000.0))
    start = np.array(conf.get("domainStart", [0.0, 0.0, 0.0]), dtype=np.float32)
    end_cfg = conf.get("domainEnd", [1.0, 1.0, 1.0])
    domain_size = tuple(e - s for s, e in zip(conf.get("domainStart", [0.0, 0.0, 0.0]), end_cfg))

    xs, vs, rhos, mats, dyns = [], [], [], [], []

    def add(x, v, rho, mat, dyn):
        n = x.shape[0]
        xs.append(np.asarray(x, np.float32))
        vs.append(np.ascontiguousarray(np.broadcast_to(np.asarray(v, np.float32), (n, 3)), dtype=np.float32))
        rhos.append(np.full(n, rho, np.float32))
        mats.append(np.full(n, mat, np.int32))
        dyns.append(np.full(n, dyn, np.int32))

    # fluid blocks (scene_loader.py:89-102, 319-336)
    for fb in data.get("FluidBlocks", []) or []:
        t = np.array(fb.get("translation", [0, 0, 0]), dtype=np.float32)
        s = np.array(fb.get("scale", [1, 1, 1]), dtype=np.float32)
        lo = np.array(fb["start"], dtype=np.float32) + t
        size = (np.array(fb["end"], dtype=np.float32) - np.array(fb["start"], dtype=np.float32)) * s
        hi = lo + size
        x = _cube_block(tuple(lo), tuple(hi - lo), diameter)
        add(x, fb.get("velocity", [0.0, 0.0, 0.0]), float(fb.get("density", 1000.0)), MATERIAL_FLUID, 1)
    # mesh bodies, pre-voxelised (scene_loader.py:104-122, 338-387)
    for key, mat in (("FluidBodies", MATERIAL_FLUID), ("RigidBodies", MATERIAL_RIGID)):
        for body in data.get(key, []) or []:
            pts = body.get("voxelizedPoints")
            if pts is None:
                raise NotImplementedError(f"{key} entry {body.get('objectId')}: OBJ voxelisation needs trimesh; "
                                          "pass the body's points as 'voxelizedPoints'")
            pts = np.asarray(pts, dtype=np.float32).reshape(-1, 3)
            if mat == MATERIAL_FLUID:
                add(pts, body.get("velocity", [0.0, 0.0, 0.0]), float(body.get("density", 1000.0)), mat, 1)
            else:
                dyn = int(bool(body.get("isDynamic", False)))
                v = body.get("velocity", [0.0, 0.0, 0.0]) if dyn else [0.0, 0.0, 0.0]
                add(pts, v, float(body.get("density", 1000.0)), mat, dyn)
    # generated bodies (scene_loader.py:447-492, 389-405)
    for gb in data.get("GeneratedBodies", []) or []:
        if gb.get("type", "cube") != "cube":
            raise ValueError(f"Unknown generated body type: {gb.get('type')}")
        tr = np.array(gb.get("translation", [0, 0, 0]), dtype=np.float32)
        size = np.array(gb.get("size", [1, 1, 1]), dtype=np.float32)
        half = size / 2.0
        x = _shell(tr - half, tr + half, diameter, int(gb.get("layers", 2)))
        add(x, [0.0, 0.0, 0.0], float(gb.get("density", 1000.0)), MATERIAL_RIGID, int(bool(gb.get("isDynamic", False))))
    # boundary walls (scene_loader.py:494-545, 407-425)
    layers = int(conf.get("boundaryLayers", 0))
    if layers > 0:
        end = start + np.array(domain_size, dtype=np.float32)
        add(_shell(start, end, diameter, layers), [0.0, 0.0, 0.0], rho0, MATERIAL_RIGID, 0)

    if not xs:
        raise ValueError("scene has no particles")
    x = np.concatenate(xs)
    dyn = np.concatenate(dyns)
    kw = dict(
        dt=float(conf.get("timeStepSize", 0.0016)),
        gravity=tuple(float(g) for g in conf.get("gravitation", [0.0, -9.8, 0.0])),
        omega=float(conf.get("omega", 10.0)), tol_pcg=float(conf.get("tol_pcg", 1e-6)),
        density_error_tol=float(conf.get("densityErrorTol", 1e-3)),
        max_outer_iters=int(conf.get("maxOuterIters", 1000)),
        fixed_outer_iters=bool(conf.get("fixedOuterIters", False)),
        cache_size=int(conf.get("neighborCacheSize", 60)),
        viscosity_method=int(conf.get("viscosityMethod", 0)),
        viscosity_coeff=float(conf.get("viscosityCoeff", 0.01)),
        surface_tension_method=int(conf.get("surfaceTensionMethod", 0)),
        surface_tension_coeff=float(conf.get("surfaceTensionCoeff", 0.01)),
        pressure_method=int(conf.get("pressureMethod", 1)),
    )
    return Scene(x=np.ascontiguousarray(x), v=np.ascontiguousarray(np.concatenate(vs)), is_dynamic=dyn, material=np.concatenate(mats),
                 density0=np.concatenate(rhos), particle_radius=radius,
                 domain_size=np.asarray(domain_size, dtype=np.float32), name=name or "scene", **kw)


class SceneLoader:
    """The reference's loader interface (scene_loader.py:41-216) over
    `load_scene`: `prepare_scene()` parses and counts, `populate_scene(ps,
    data)` allocates the SimulationData and appends the particles."""

    def __init__(self, config):
        self.cfg = config
        self.dim = 3
        self.particle_diameter = config.particle_diameter

    def get_scene_name(self, scene_file_path: str) -> str:
        import pathlib
        return pathlib.Path(scene_file_path).stem if scene_file_path else "scene"

    def prepare_scene(self) -> dict:
        sc = load_scene(self.cfg.scene_data or {"Configuration": {}})
        nf = int(sc.is_dynamic.sum())
        return {"scene": sc, "particle_max_num": int(sc.n), "fluid_particle_num": nf,
                "rigid_particle_num": int(sc.n - nf), "solid_particle_num": 0, "num_objects": 1,
                "num_rigid_bodies": 0}

    def populate_scene(self, ps, scene_data: dict):
        sc = scene_data["scene"]
        ps.allocate(particle_max_num=scene_data["particle_max_num"], num_objects=scene_data["num_objects"],
                    num_rigid_bodies=scene_data["num_rigid_bodies"])
        ps.rigid_particle_num = scene_data["rigid_particle_num"]
        color = np.where(sc.material[:, None] == MATERIAL_FLUID, np.array([10, 100, 200], np.float32),
                         np.array([200, 200, 200], np.float32))
        ps.add_particles(0, sc.n, sc.x, sc.v, sc.density0, sc.material, sc.is_dynamic, color)

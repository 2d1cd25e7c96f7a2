"""Synthetic scene builders (host side, NumPy).

The reference loads scenes from JSON (`scripts/io/config_builder.py:54-115`,
`scripts/io/scene_loader.py:70-429`).  The workloads this package is measured on
are synthetic restatements of the reference's column / dam-break scenes, so
this module builds the particle arrays directly:

* fluid blocks on a cubic lattice (the reference's `SimulationData.add_cube`,
  `scripts/sim/simulation_data.py:290-356`) with an optional seeded uniform
  jitter of +-`jitter` x spacing per coordinate (the reference has no jitter);
* a one-layer (or multi-layer) hollow box of static boundary particles, the
  reference's `GeneratedBodies` "cube" shell (`scene_loader.py:447-492`), which
  keeps the duplicated edge rows of that generator so particle counts agree;
* the domain-wall generator (`scene_loader.py:494-545`), also with duplicated
  edges;
* a Fibonacci-sampled sphere surface for the dam-break obstacle (the
  reference only voxelises OBJ meshes, which needs trimesh).

Per-particle mass follows the reference's rule (`simulation_data.py:40-57`):
m = 0.8 d^3 rho, 1/m for dynamic particles, and static particles get m x 10
with m_inv = 0.  All arithmetic that the reference does in FP32 is done in
FP32 here, in the same order.

The reference is y-up (gravity [0, -9.81, 0]); a box written as
(width, depth, height) maps to (x = width, y = height, z = depth).
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional, Sequence

import numpy as np

MATERIAL_RIGID = 0
MATERIAL_FLUID = 1


@dataclasses.dataclass
class Scene:
    """One independent scene: particle arrays in the reference's layout and
    the configuration keys the IP pressure step reads."""

    x: np.ndarray            # (N, 3) float32 positions
    v: np.ndarray            # (N, 3) float32 velocities
    is_dynamic: np.ndarray   # (N,) int32
    material: np.ndarray     # (N,) int32 (0 rigid, 1 fluid)
    density0: np.ndarray     # (N,) float32 rest density per particle
    particle_radius: float
    domain_size: np.ndarray  # (3,) float32, domain starts at the origin
    dt: float = 1e-3
    gravity: tuple = (0.0, -9.81, 0.0)
    # IP solver keys (`ip.py:228`, `pressure_base.py:314-317`)
    omega: float = 10.0
    tol_pcg: float = 1e-6
    density_error_tol: float = 1e-3
    max_outer_iters: int = 1000
    fixed_outer_iters: bool = False
    max_iteration_pcg: int = 1000
    cache_size: int = 60
    # non-pressure forces (`framework.py:400-421`); 0 disables
    viscosity_method: int = 0
    viscosity_coeff: float = 0.0
    surface_tension_method: int = 0
    surface_tension_coeff: float = 0.0
    # pressureMethod (framework.py:168-174): 1 IP, 0 PRJ
    pressure_method: int = 1
    name: str = "scene"

    @property
    def particle_diameter(self) -> float:
        return 2.0 * self.particle_radius

    @property
    def support_radius(self) -> float:
        # config_builder.py:51-52: d = 2r, h = 4r
        return 4.0 * self.particle_radius

    @property
    def n(self) -> int:
        return int(self.x.shape[0])

    @property
    def n_dynamic(self) -> int:
        return int(self.is_dynamic.sum())

    def masses(self):
        """(m, m_inv) in FP32 following `simulation_data.py:40-57`."""
        d = self.particle_diameter
        m_v0 = np.float32(0.8 * d ** 3)
        m = (m_v0 * self.density0.astype(np.float32)).astype(np.float32)
        dyn = self.is_dynamic == 1
        m_inv = np.zeros_like(m)
        m_inv[dyn] = np.float32(1.0) / m[dyn]
        m[~dyn] = m[~dyn] * np.float32(10.0)
        return m, m_inv

    def config(self) -> dict:
        """The scene's `Configuration` dict in the reference's JSON key names."""
        return {
            "particleRadius": self.particle_radius,
            "timeStepSize": self.dt,
            "gravitation": list(self.gravity),
            "domainStart": [0.0, 0.0, 0.0],
            "domainEnd": [float(s) for s in self.domain_size],
            "pressureMethod": self.pressure_method,
            "omega": self.omega,
            "tol_pcg": self.tol_pcg,
            "densityErrorTol": self.density_error_tol,
            "maxOuterIters": self.max_outer_iters,
            "fixedOuterIters": self.fixed_outer_iters,
            "neighborCacheSize": self.cache_size,
            "viscosityMethod": self.viscosity_method,
            "viscosityCoeff": self.viscosity_coeff,
            "surfaceTensionMethod": self.surface_tension_method,
            "surfaceTensionCoeff": self.surface_tension_coeff,
        }


# ---------------------------------------------------------------------------
# generators
# ---------------------------------------------------------------------------

def lattice_block(lower, counts, spacing, jitter=0.0, seed=0) -> np.ndarray:
    """counts[0] x counts[1] x counts[2] lattice starting at `lower`, x slowest
    (the reference's meshgrid 'ij' order, simulation_data.py:316-328), plus a
    seeded uniform jitter of +-jitter*spacing on every coordinate."""
    axes = [np.float64(lower[a]) + spacing * np.arange(int(counts[a]), dtype=np.float64)
            for a in range(3)]
    g = np.meshgrid(*axes, indexing="ij")
    pts = np.stack([c.ravel() for c in g], axis=1)
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        pts = pts + rng.uniform(-jitter * spacing, jitter * spacing, size=pts.shape)
    return pts.astype(np.float32)


def _face_grid(a, b):
    ga, gb = np.meshgrid(a, b, indexing="ij")
    return ga.ravel(), gb.ravel()


def cube_shell(center, size, diameter, layers=1) -> np.ndarray:
    """Hollow box of boundary particles, six faces per layer, edges and corners
    repeated on every face that contains them (the reference's cube generator,
    scene_loader.py:447-492)."""
    c = np.asarray(center, dtype=np.float32)
    half = np.asarray(size, dtype=np.float32) / np.float32(2.0)
    lo0, hi0 = c - half, c + half
    d = np.float32(diameter)
    out = []
    for layer in range(int(layers)):
        off = np.float32(layer) * d
        lo, hi = lo0 - off, hi0 + off
        xs, ys, zs = (np.arange(lo[a], hi[a] + d * np.float32(0.5), d) for a in range(3))
        u, w = _face_grid(xs, zs)
        for y in (lo[1], hi[1]):
            out.append(np.stack([u, np.full(u.size, y), w], axis=1))
        u, w = _face_grid(ys, zs)
        for xv in (lo[0], hi[0]):
            out.append(np.stack([np.full(u.size, xv), u, w], axis=1))
        u, w = _face_grid(xs, ys)
        for zv in (lo[2], hi[2]):
            out.append(np.stack([u, w, np.full(u.size, zv)], axis=1))
    return np.concatenate(out, axis=0).astype(np.float32)


def domain_walls(domain_size, diameter, layers=1) -> np.ndarray:
    """Boundary particles on the domain faces (scene_loader.py:494-545)."""
    size = np.asarray(domain_size, dtype=np.float32)
    return cube_shell(size / np.float32(2.0), size, diameter, layers)


def sphere_surface(center, radius, spacing) -> np.ndarray:
    """Fibonacci-lattice samples of a sphere surface, about 4 pi R^2 / d^2 points."""
    n = max(12, int(round(4.0 * math.pi * radius * radius / (spacing * spacing))))
    k = np.arange(n, dtype=np.float64) + 0.5
    phi = np.arccos(1.0 - 2.0 * k / n)
    theta = math.pi * (1.0 + 5.0 ** 0.5) * k
    pts = np.stack([np.cos(theta) * np.sin(phi), np.cos(phi), np.sin(theta) * np.sin(phi)], axis=1)
    return (np.asarray(center, dtype=np.float64) + radius * pts).astype(np.float32)


def assemble(fluid: Sequence[np.ndarray], static: Sequence[np.ndarray], particle_radius: float,
             domain_size, rho0: float = 1000.0, fluid_velocity=None, **kw) -> Scene:
    """Fluid blocks first, then static bodies (the reference's population order,
    scene_loader.py:217-429)."""
    xf = np.concatenate(list(fluid), axis=0) if fluid else np.zeros((0, 3), np.float32)
    xs = np.concatenate(list(static), axis=0) if static else np.zeros((0, 3), np.float32)
    nf, ns = xf.shape[0], xs.shape[0]
    x = np.concatenate([xf, xs], axis=0).astype(np.float32)
    v = np.zeros_like(x)
    if fluid_velocity is not None:
        v[:nf] = np.asarray(fluid_velocity, dtype=np.float32)
    dyn = np.concatenate([np.ones(nf, np.int32), np.zeros(ns, np.int32)])
    mat = np.concatenate([np.full(nf, MATERIAL_FLUID, np.int32), np.full(ns, MATERIAL_RIGID, np.int32)])
    rho = np.full(nf + ns, rho0, np.float32)
    return Scene(x=x, v=v, is_dynamic=dyn, material=mat, density0=rho,
                 particle_radius=float(particle_radius),
                 domain_size=np.asarray(domain_size, dtype=np.float32), **kw)


def column_in_box(counts_xyz, spacing, box_xyz, *, jitter=0.01, seed=0, corner=True,
                  margin=None, **kw) -> Scene:
    """A fluid column on a cubic lattice resting on the floor of a one-layer
    static box.  The box is a cube shell placed inside a domain padded by more
    than h on every side, so the reference's domain clamp (padding = h) never
    touches the fluid while the box holds it (boundary.py:27-91).  Box edges
    shorter than the fluid extent + 2 spacings are widened to that length."""
    d = float(spacing)
    h = 2.0 * d
    counts = [int(c) for c in counts_xyz]
    extent = [(c - 1) * d for c in counts]
    box = [max(float(b), e + 2.0 * d) for b, e in zip(box_xyz, extent)]
    margin = 2.0 * h if margin is None else float(margin)
    domain = [b + 2.0 * margin for b in box]
    lo_box = [margin, margin, margin]
    if corner:
        lower = [lo_box[0] + d, lo_box[1] + d, lo_box[2] + d]
    else:
        lower = [lo_box[0] + 0.5 * (box[0] - extent[0]), lo_box[1] + d,
                 lo_box[2] + 0.5 * (box[2] - extent[2])]
    fluid = lattice_block(lower, counts, d, jitter, seed)
    center = [lo_box[a] + 0.5 * box[a] for a in range(3)]
    shell = cube_shell(center, box, d, layers=1)
    return assemble([fluid], [shell], particle_radius=0.5 * d, domain_size=domain, **kw)


# ---------------------------------------------------------------------------
# the measured workloads
# ---------------------------------------------------------------------------

def small_column(seed=0, **kw) -> Scene:
    """8,192 fluid particles (16 x 32 x 16, y tall) at d = 0.02 m with +-1 %
    jitter, in a 0.64 x 1.28 x 0.64 m one-layer box; IP only, dt = 1 ms,
    densityErrorTol 1e-3, maxOuterIters 100."""
    kw.setdefault("max_outer_iters", 100)
    return column_in_box((16, 32, 16), 0.02, (0.64, 1.28, 0.64), seed=seed,
                         name="small_column_8k", **kw)


def tall_column(seed=0, viscosity=True, **kw) -> Scene:
    """102,400 fluid particles (40 x 64 x 40, y tall) at d = 0.02 m with +-1 %
    jitter, in a 0.8 x 3.0 x 0.8 m one-layer box; implicit viscosity
    (Weiler 2018, nu = 1e-3 m^2/s) when `viscosity`; dt = 1 ms."""
    if viscosity:
        kw.setdefault("viscosity_method", 1)
        kw.setdefault("viscosity_coeff", 1e-3)
    return column_in_box((40, 64, 40), 0.02, (0.8, 3.0, 0.8), seed=seed,
                         name="tall_column_102k", **kw)


def dam_break(seed=0, **kw) -> Scene:
    """524,288 fluid particles (128 x 64 x 64) at d = 0.01 m against the x-min
    end of a 3.2 x 1.28 x 0.64 m tank, with a static sphere (R = 0.15 m)
    sampled on its surface at the tank centre; dt = 0.5 ms."""
    d = 0.01
    h = 2.0 * d
    counts = (128, 64, 64)
    box = [3.2, 1.28, 0.64]
    extent = [(c - 1) * d for c in counts]
    box = [max(b, e + 2.0 * d) for b, e in zip(box, extent)]
    margin = 2.0 * h
    domain = [b + 2.0 * margin for b in box]
    lower = [margin + d, margin + d, margin + d]
    fluid = lattice_block(lower, counts, d, 0.01, seed)
    center = [margin + 0.5 * b for b in box]
    shell = cube_shell(center, box, d, layers=1)
    sphere = sphere_surface(center, 0.15, d)
    kw.setdefault("dt", 5e-4)
    kw.setdefault("viscosity_method", 1)
    kw.setdefault("viscosity_coeff", 1e-3)
    kw.setdefault("surface_tension_method", 1)
    kw.setdefault("surface_tension_coeff", 0.05)
    return assemble([fluid], [shell, sphere], particle_radius=0.5 * d, domain_size=domain,
                    name="dam_break_524k", **kw)


def random_column(n_target, aspect, spacing=0.02, seed=0, **kw) -> Scene:
    """A column of about `n_target` fluid particles with height/width `aspect`
    in a box whose horizontal sides are twice the column's."""
    nw = max(2, int(round((n_target / aspect) ** (1.0 / 3.0))))
    nh = max(2, int(round(n_target / (nw * nw))))
    d = spacing
    side = 2.0 * nw * d
    height = 1.25 * nh * d + 2.0 * d
    return column_in_box((nw, nh, nw), d, (side, height, side), seed=seed,
                         name=f"column_{nw}x{nh}x{nw}", **kw)


def batch_mix(n_scenes=64, lo=4096, hi=65536, seed=0, **kw) -> List[Scene]:
    """`n_scenes` column-collapse scenes with fluid counts log-uniform in
    [lo, hi] and aspect ratios uniform in [1, 4], all from one seed."""
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(math.log(lo), math.log(hi), size=n_scenes))
    aspects = rng.uniform(1.0, 4.0, size=n_scenes)
    return [random_column(float(c), float(a), seed=seed + 1 + i, **kw)
            for i, (c, a) in enumerate(zip(counts, aspects))]


def small_dam_break(n_target, spacing=0.02, seed=0, **kw) -> Scene:
    """A dam-break block of about `n_target` particles (2:1:1) against one end
    of a tank 2.5x as long as the block, no obstacle."""
    n1 = max(2, int(round((n_target / 2.0) ** (1.0 / 3.0))))
    counts = (2 * n1, n1, n1)
    d = spacing
    box = (2.5 * 2 * n1 * d, 2.0 * n1 * d, n1 * d + 2.0 * d)
    return column_in_box(counts, d, box, seed=seed, name=f"dambreak_{2*n1}x{n1}x{n1}", **kw)


@dataclasses.dataclass
class Request:
    arrival_s: float
    scene: Scene
    steps: int


def request_stream(rate=4.0, duration_s=120.0, lo=2048, hi=262144, steps_lo=100, steps_hi=2000,
                   seed=0, max_requests: Optional[int] = None) -> List[Request]:
    """Poisson arrivals (mean `rate`/s over `duration_s`), each a column
    collapse or a dam break (50/50) with a log-uniform fluid count and a
    uniform number of steps."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out: List[Request] = []
    i = 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration_s or (max_requests is not None and len(out) >= max_requests):
            break
        n = float(math.exp(rng.uniform(math.log(lo), math.log(hi))))
        steps = int(rng.integers(steps_lo, steps_hi + 1))
        if rng.uniform() < 0.5:
            sc = random_column(n, float(rng.uniform(1.0, 4.0)), seed=seed + 1000 + i)
        else:
            sc = small_dam_break(n, seed=seed + 1000 + i)
        out.append(Request(arrival_s=t, scene=sc, steps=steps))
        i += 1
    return out

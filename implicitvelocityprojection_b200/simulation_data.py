"""SimulationData: particle state in the reference's layout
(`scripts/sim/simulation_data.py:113-356`), held in PyTorch device tensors.

Arrays are sized `particle_max_num` and the first `particle_num` rows are
live, as in the reference.  The CUDA engine (`engine.Engine`) is created
lazily over the live rows and shared by `NeighbourSearch` and the pressure
solver; its neighbour lists are internal (cell-ordered, compact), and
`neighbour_cache()` exports them in the reference's cache layout.
"""
from __future__ import annotations

import dataclasses
from functools import reduce
from typing import Optional

import numpy as np
import torch


@dataclasses.dataclass
class SceneSpec:
    """What the engine needs to know about one scene."""

    n: int
    n_dynamic: int
    particle_radius: float
    domain_size: tuple
    dt: float
    gravity: tuple
    omega: float = 10.0
    tol_pcg: float = 1e-6
    density_error_tol: float = 1e-3
    max_outer_iters: int = 1000
    max_iteration_pcg: int = 1000
    fixed_outer_iters: bool = False
    cache_size: int = 60
    viscosity_coeff: float = 0.0
    viscosity_method: int = 0
    surface_tension_coeff: float = 0.0
    surface_tension_method: int = 0
    pressure_method: int = 1  # 1 IP, 0 PRJ


class SimulationData:
    def __init__(self, config, device: str = "cuda"):
        self.cfg = config
        self.dim = 3
        self.device = torch.device(device)
        self.domain_size = np.array(config.domain_size[:3], dtype=np.float32)
        self.material_rigid = 0
        self.material_fluid = 1
        self.particle_radius = config.particle_radius
        self.particle_diameter = config.particle_diameter
        self.support_radius = config.support_radius
        self.padding = self.support_radius
        self.m_V0_init = 0.8 * self.particle_diameter ** self.dim  # simulation_data.py:137
        self.num_objects = 1
        self.num_rigid_bodies = 0
        self.rigid_particle_num = 0
        self.particle_num = 0
        self.particle_max_num = 0
        self.num_deformable = 0
        self.cache_size = int(config.get_cfg("neighborCacheSize", 60))
        self.allocated = False
        self._engine = None
        self._engine_key = None
        self._n_dynamic = 0

    # ------------------------------------------------------------ storage
    def allocate(self, particle_max_num: int, num_objects: int = 1, num_rigid_bodies: int = 0):
        """simulation_data.py:165-212 (device tensors instead of Warp arrays)."""
        n = int(particle_max_num)
        self.particle_max_num = n
        self.num_objects = int(max(num_objects, 1))
        self.num_rigid_bodies = int(num_rigid_bodies)
        z3 = lambda: torch.zeros((n, 3), dtype=torch.float32, device=self.device)
        z1 = lambda: torch.zeros(n, dtype=torch.float32, device=self.device)
        zi = lambda: torch.zeros(n, dtype=torch.int32, device=self.device)
        self.object_id = zi()
        self.x, self.x_old, self.x0, self.v, self.v0 = z3(), z3(), z3(), z3(), z3()
        self.m, self.m_inv = z1(), z1()
        self.n = z3()
        self.density, self.density0, self.divergence = z1(), z1(), z1()
        self.material = zi()
        self.color = torch.zeros((n, 4), dtype=torch.float32, device=self.device)
        self.is_dynamic = zi()
        self.is_fixed = zi()
        self.is_kinematic = zi()
        self.k = z1()  # shared with the pressure solver (PressureBase.k)
        self.allocated = True
        self._engine = None

    def add_particles(self, object_id, new_particles_num, new_particles_positions, new_particles_velocity,
                      new_particle_density, new_particles_material, new_particles_is_dynamic, new_particles_color,
                      m_V0: Optional[float] = None):
        """simulation_data.py:214-287 with the per-particle rule of add_particle
        (simulation_data.py:14-59) evaluated in FP32 on the host."""
        if not self.allocated:
            raise RuntimeError("Must call allocate() before adding particles")
        n = int(new_particles_num)
        if self.particle_num + n > self.particle_max_num:
            print(f"Warning: Cannot add {n} particles. "
                  f"Only {self.particle_max_num - self.particle_num} slots available.")
            return
        s = slice(self.particle_num, self.particle_num + n)
        x = np.asarray(new_particles_positions, dtype=np.float32).reshape(n, 3)
        v = np.asarray(new_particles_velocity, dtype=np.float32).reshape(n, 3)
        rho = np.asarray(new_particle_density, dtype=np.float32).reshape(n)
        dyn = np.asarray(new_particles_is_dynamic, dtype=np.int32).reshape(n)
        mv0 = np.float32(self.m_V0_init if m_V0 is None else float(m_V0))
        m = (mv0 * rho).astype(np.float32)
        m_inv = np.zeros(n, np.float32)
        m_inv[dyn == 1] = np.float32(1.0) / m[dyn == 1]
        m[dyn != 1] = m[dyn != 1] * np.float32(10.0)  # static particles: x10 mass
        col = np.asarray(new_particles_color, dtype=np.float32)
        if col.ndim == 2 and col.shape[1] == 3:
            col = np.hstack([col, np.full((n, 1), 255.0, np.float32)])
        put = lambda t, a: t[s].copy_(torch.from_numpy(np.ascontiguousarray(a)).to(self.device))
        put(self.object_id, np.full(n, int(object_id), np.int32))
        for t in (self.x, self.x_old, self.x0):
            put(t, x)
        put(self.v, v)
        put(self.v0, v)
        put(self.density0, rho)
        put(self.density, rho)
        put(self.m, m)
        put(self.m_inv, m_inv)
        put(self.material, np.asarray(new_particles_material, dtype=np.int32).reshape(n))
        put(self.is_dynamic, dyn)
        put(self.color, col.reshape(n, 4))
        self.particle_num += n
        self._n_dynamic += int((dyn == 1).sum())
        self._engine = None

    def add_cube(self, object_id, lower_corner, cube_size, material, is_dynamic, color=(0, 0, 0), density=None,
                 velocity=None):
        """simulation_data.py:290-356: lattice with np.arange per axis."""
        axes = [np.arange(lower_corner[i], lower_corner[i] + cube_size[i], self.particle_diameter)
                for i in range(self.dim)]
        num = reduce(lambda a, b: a * b, [len(a) for a in axes])
        pos = np.array(np.meshgrid(*axes, sparse=False, indexing="ij"), dtype=np.float32)
        pos = pos.reshape(self.dim, -1).transpose()
        vel = np.zeros_like(pos) if velocity is None else np.tile(np.asarray(velocity, np.float32), (num, 1))
        self.add_particles(object_id, num, pos, vel,
                           np.full(num, 1000.0 if density is None else density, np.float32),
                           np.full(num, material, np.int32), np.full(num, is_dynamic, np.int32),
                           np.tile(np.asarray(color, np.float32), (num, 1)))

    @classmethod
    def from_scene(cls, sc, config=None, device: str = "cuda") -> "SimulationData":
        """SimulationData holding a synthetic `scenes.Scene`."""
        from .config import SimConfig
        cfg = config or SimConfig.from_scene(sc)
        ps = cls(cfg, device=device)
        ps.allocate(sc.n)
        ps.add_particles(0, sc.n, sc.x, sc.v, sc.density0, sc.material, sc.is_dynamic,
                         np.zeros((sc.n, 3), np.float32))
        return ps

    # ------------------------------------------------------------ engine
    def spec(self, solver=None, dt: Optional[float] = None) -> SceneSpec:
        n = self.particle_num
        n_dyn = self._n_dynamic
        cfg = self.cfg
        g = cfg.gravity
        sp = SceneSpec(n=n, n_dynamic=n_dyn, particle_radius=float(self.particle_radius),
                       domain_size=tuple(float(a) for a in self.domain_size),
                       dt=float(cfg.dt if dt is None else dt), gravity=tuple(float(a) for a in g),
                       cache_size=self.cache_size,
                       viscosity_coeff=float(cfg.viscosity_coeff) if int(cfg.viscosity_method) == 1 else 0.0,
                       viscosity_method=int(cfg.viscosity_method) if float(cfg.viscosity_coeff) > 0 else 0,
                       surface_tension_coeff=float(cfg.surface_tension_coeff)
                       if int(cfg.surface_tension_method) == 1 else 0.0,
                       surface_tension_method=int(cfg.surface_tension_method)
                       if float(cfg.surface_tension_coeff) > 0 else 0)
        if solver is not None:
            sp.pressure_method = int(getattr(solver, "pressure_method", 1))
            sp.omega = float(solver.omega)
            sp.tol_pcg = float(getattr(solver, "tol_pcg", 1e-6))
            sp.density_error_tol = float(solver.tol_opt)
            sp.max_outer_iters = int(solver.max_iteration_opt)
            sp.max_iteration_pcg = int(getattr(solver, "max_iteration_pcg", 1000))
            sp.fixed_outer_iters = bool(solver.use_fixed_iters)
        return sp

    def live(self) -> dict:
        n = self.particle_num
        return {"x": self.x[:n], "v": self.v[:n], "m": self.m[:n], "density0": self.density0[:n],
                "is_dynamic": self.is_dynamic[:n], "material": self.material[:n], "density": self.density[:n],
                "k": self.k[:n], "divergence": self.divergence[:n]}

    def engine(self, solver=None, dt: Optional[float] = None):
        """The engine over the live particles (created on first use, recreated
        when the particle count changes); run-time parameters are refreshed
        from `solver` / `dt` when they changed."""
        from .engine import Engine
        sp = self.spec(solver, dt)
        # solver choice and enabled forces fix the engine's plan (launches and
        # buffers): a change rebuilds the engine
        key = (sp.n, sp.n_dynamic, self.x.data_ptr() if self.allocated else 0, sp.pressure_method,
               sp.viscosity_method == 1 and sp.viscosity_coeff > 0,
               sp.surface_tension_method == 1 and sp.surface_tension_coeff > 0)
        if self._engine is None or self._engine_key != key:
            self._engine = Engine([sp], device=str(self.device), arrays=self.live())
            self._engine_key = key
            self._engine_spec = sp
        elif sp != self._engine_spec:  # field-wise dataclass comparison
            self._engine.update_scene(0, sp)
            self._engine_spec = sp
        return self._engine

    def neighbour_cache(self):
        """(neighbor_count[N], neighbor_ids[N, cache_size]) in the reference
        layout (simulation_data.py:206-209); rows of static particles are 0."""
        return self.engine().neighbours(0, self.cache_size)

"""Framework: the time-step orchestrator with the reference's interface
(`scripts/framework.py:143-544`) for the IP pressure method.

`forward()` runs one whole step -- gravity, implicit surface tension and
implicit viscosity where enabled, the IP solve, advect + boundary clamp, neighbour rebuild, density
and Aii (framework.py:423-544) -- as one CUDA graph launch of the engine, then
reads the solve statistics once (the reference synchronises many times per
step).  `forward_many(n)` queues n steps and checks them once at the end.
"""
from __future__ import annotations

import math
import time

import torch

from .ip import IP
from .prj import PRJ


class Framework:
    def __init__(self, simulation_data, neighbour_search, config):
        self.ps = simulation_data
        self.ns = neighbour_search
        if getattr(neighbour_search, "ps", None) is None and hasattr(neighbour_search, "attach"):
            neighbour_search.attach(simulation_data)
        self.cfg = config
        self.dt = config.dt
        self.dt_default = config.dt
        self.use_cfl = bool(config.get_cfg("useCFL", False))
        self.cfl_factor = float(config.get_cfg("cflFactor", 0.4))
        self.cfl_min_dt = float(config.get_cfg("cflMinDt", 1e-4))
        self.time = 0.0
        self.initial_particle_num = simulation_data.particle_num
        self.stats_pressure_ms = 0.0
        self.stats_elasticity_ms = 0.0
        # framework.py:168-174: IP (1) and PRJ (0) are built here; SISPH (3)
        # and PBF (5) are position-based solvers outside this engine
        pressure_method = int(config.get_cfg("pressureMethod", 1))
        if pressure_method not in (0, 1):
            raise NotImplementedError(f"pressureMethod {pressure_method}: only PRJ (0) and IP (1) are implemented "
                                      "on this engine")
        self.pressure = (IP if pressure_method == 1 else PRJ)(simulation_data, neighbour_search, config)
        # non-pressure forces (framework.py:176-187): Jeske 2023 implicit
        # surface tension and Weiler 2018 implicit viscosity run inside the
        # engine's step; the explicit forms (Akinci 2013 surface tension,
        # XSPH-style viscosity) are not built, so they must be disabled
        if int(config.viscosity_method) != 1 and float(config.viscosity_coeff) != 0.0:
            raise NotImplementedError("explicit viscosity (viscosityMethod 0) is not implemented; set "
                                      "viscosityCoeff 0 or viscosityMethod 1")
        if int(config.surface_tension_method) != 1 and float(config.surface_tension_coeff) != 0.0:
            raise NotImplementedError("explicit surface tension (surfaceTensionMethod 0) is not implemented; set "
                                      "surfaceTensionCoeff 0 or surfaceTensionMethod 1")
        self.elasticity = None
        self.pressure_enabled = bool(config.get_cfg("pressureEnabled", True))
        self._events = None

    def engine(self):
        return self.ps.engine(self.pressure, self.dt)

    def initialize(self):
        """framework.py:282-290 / 323-330: neighbour rebuild, density, Aii."""
        self.ns.build(self.ps.x, self.ps.particle_num)
        self.ns.build_cache(self.ps.x, self.ps.particle_num, self.ps.cache_size, solver=self.pressure)

    def reset(self):
        """framework.py:227-280 for the state this engine owns."""
        ps = self.ps
        ps.particle_num = self.initial_particle_num
        n = ps.particle_num
        ps.x[:n].copy_(ps.x0[:n])
        ps.x_old[:n].copy_(ps.x0[:n])
        ps.v[:n].copy_(ps.v0[:n])
        ps.density.copy_(ps.density0)
        ps.k.zero_()
        self.time = 0.0
        self.initialize()

    def _cfl(self):
        """framework.py:426-440 (one host read-back, as in the reference)."""
        n = self.ps.particle_num
        dyn = self.ps.is_dynamic[:n] == 1
        v = self.ps.v[:n][dyn]
        v_max_sq = float((v * v).sum(dim=1).max().item()) if v.numel() else 0.0
        if math.isfinite(v_max_sq) and v_max_sq > 1e-16:
            self.dt = min(self.dt_default, self.cfl_factor * self.ps.support_radius / v_max_sq ** 0.5)
        else:
            self.dt = self.dt_default
        self.dt = max(self.dt, self.cfl_min_dt)

    def forward(self):
        """One time step (framework.py:423-544)."""
        if self.use_cfl:
            self._cfl()
        if not self.pressure_enabled:
            raise NotImplementedError("pressureEnabled = false is not supported by the fused step")
        t0 = time.perf_counter()
        eng = self.engine()
        eng.step(1)
        st = eng.stats(0)
        self.stats_pressure_ms = (time.perf_counter() - t0) * 1000.0
        self.pressure.apply_stats(st, self.stats_pressure_ms)
        self.time += self.dt

    def forward_host(self, x, v, first: int = 0):
        """forward() for a caller that keeps the moving particles' state in
        host memory: x and v (page-locked float32 (count, 3) tensors holding
        particles first .. first + count) are uploaded into the step and the
        step's new x and v written back into them, the copies overlapped with
        the step's kernels (ivp_step_io).  Statistics as forward()."""
        if self.use_cfl:
            self._cfl()
        if not self.pressure_enabled:
            raise NotImplementedError("pressureEnabled = false is not supported by the fused step")
        t0 = time.perf_counter()
        eng = self.engine()
        eng.step_io(x, v, x, v, first=first, count=int(x.shape[0]))
        st = eng.stats(0)
        self.stats_pressure_ms = (time.perf_counter() - t0) * 1000.0
        self.pressure.apply_stats(st, self.stats_pressure_ms)
        self.time += self.dt

    def forward_many(self, n: int):
        """n steps queued back to back; statistics and errors of the last step."""
        if self.use_cfl:
            for _ in range(n):
                self.forward()
            return
        t0 = time.perf_counter()
        eng = self.engine()
        eng.step(int(n))
        st = eng.stats(0)
        self.stats_pressure_ms = (time.perf_counter() - t0) * 1000.0 / max(n, 1)
        self.pressure.apply_stats(st, self.stats_pressure_ms)
        self.time += n * self.dt

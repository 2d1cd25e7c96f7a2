"""PRJ: the projected-Jacobi pressure solver with the reference's interface
(`scripts/sim/forces/pressure/prj.py:120-340`), run on the same engine,
neighbour rows and reductions as IP.

`solve(dt)` runs the whole solve on the device -- dt_v_0 = dt v, then passes
of head (dt_v = dt_v_0 - dt^2 J^T lambda / m) and tail (r = dt J v + c, the
clamped lambda update, the average density error) until the error is below
`tol_opt` after at least one update or `max_iteration_opt` is reached -- and
reads the statistics once.  The divergence-free pass (`enable_df`) and the
warm start are not built (both are off by default in the reference).
"""
from __future__ import annotations

import time

from . import _lib
from .pressure_base import PressureBase


class PRJ(PressureBase):
    pressure_method = 0  # pressureMethod of the configuration (framework.py:168-174)

    def __init__(self, particle_system, neighbour_search, config):
        super().__init__(particle_system, neighbour_search, config)
        # prj.py:124-136
        self.outer_iter = 0
        self.warm_start = False
        self.omega = 0.5
        self.enable_df = False
        self.df_num_threshold = 25
        self.df_tol_opt = 1e-2
        self.stats_df_outer_iters = 0
        self.stats_df_total_cost_ms = 0.0

    @property
    def D_inv(self):
        return self.k

    def apply_stats(self, st, cost_ms: float):
        """Per-solve statistics into the stats_* fields; raises as
        check_converged does (pressure_base.py:487-495)."""
        self.reset_stats()
        self.stats_density_errors = list(st.stats_density_errors)
        self.stats_outer_iters = st.stats_outer_iters
        self.outer_iter = st.stats_outer_iters
        self.stats_final_density_error = st.stats_final_density_error
        self.stats_overflow_particles = st.overflow_particles
        self.stats_total_cost_ms = cost_ms
        n = max(len(self.stats_density_errors), 1)
        self.stats_iter_costs = [cost_ms / n] * len(self.stats_density_errors)
        if st.status == _lib.NOT_CONVERGED:
            err = self.stats_density_errors[-1] if self.stats_density_errors else self.stats_final_density_error
            raise RuntimeError(f"[PRJ] does not converge! density err={err:.2e} (tol={self.tol_opt:.2e}) "
                               f"after {self.stats_outer_iters} iters")
        if st.status == _lib.TIMEOUT:
            raise RuntimeError("[PRJ] solve stopped by the device iteration guard")
        if st.status != _lib.OK:
            raise RuntimeError(f"[PRJ] solve failed with status {st.status}")

    def _check_supported(self):
        if self.warm_start:
            raise NotImplementedError("PRJ warm start is not built (off by default, prj.py:126)")
        if self.enable_df:
            raise NotImplementedError("PRJ divergence-free pass is not built (off by default, prj.py:130)")

    def solve(self, dt):
        self._check_supported()
        t0 = time.perf_counter()
        eng = self.engine(dt)
        eng.prj_solve()
        st = eng.stats(0)
        self.apply_stats(st, (time.perf_counter() - t0) * 1000.0)

    def solve_df(self, dt):
        raise NotImplementedError("PRJ divergence-free pass is not built (off by default, prj.py:130)")

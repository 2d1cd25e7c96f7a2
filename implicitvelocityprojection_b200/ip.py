"""IP: the implicit velocity projection pressure solver with the reference's
interface (`scripts/sim/forces/pressure/ip.py:222-404`).

`solve(dt)` runs the whole solve on the device (outer loop, CG with FP64
inner products, v = d/dt, final error, divergence) as one CUDA graph with
conditional nodes, then reads the per-solve statistics once.  It raises the
reference's `RuntimeError`s on CG breakdown and on non-convergence.
"""
from __future__ import annotations

import time

from . import _lib
from .pressure_base import PressureBase


class IP(PressureBase):
    def __init__(self, particle_system, neighbour_search, config):
        super().__init__(particle_system, neighbour_search, config)
        self.tol_pcg = float(config.get_cfg("tol_pcg", 1e-6))  # ip.py:228
        self.max_iteration_pcg = 1000                           # ip.py:229

    @property
    def D_inv(self):
        return self.k

    def apply_stats(self, st, cost_ms: float):
        """Copies the engine's per-solve statistics into the stats_* fields and
        raises as the reference does (ip.py:308-309, pressure_base.py:487-495)."""
        self.reset_stats()
        self.stats_density_errors = list(st.stats_density_errors)
        self.stats_pcg_iters = list(st.stats_pcg_iters)
        self.stats_outer_iters = st.stats_outer_iters
        self.stats_final_density_error = st.stats_final_density_error
        self.stats_overflow_particles = st.overflow_particles
        self.stats_total_cost_ms = cost_ms
        n = max(len(self.stats_density_errors), 1)
        self.stats_iter_costs = [cost_ms / n] * len(self.stats_density_errors)
        if st.status == _lib.NOT_SPD:
            # ip.py:308-309: the iteration count of the failing PCG call and p^T A p
            raise RuntimeError(f"[IP] non-positive definite matrix at PCG iter {st.last_cg_iter} "
                               f"(pAp={st.last_pap:.2e})")
        if st.status == _lib.NOT_CONVERGED:
            err = self.stats_density_errors[-1] if self.stats_density_errors else self.stats_final_density_error
            raise RuntimeError(f"[IP] does not converge! density err={err:.2e} (tol={self.tol_opt:.2e}) "
                               f"after {self.stats_outer_iters} iters")
        if st.status == _lib.NBR_OVERFLOW:
            raise RuntimeError("[IP] neighbour lists truncated at neighborCacheSize dropped more pairs than the "
                               "engine's transpose-correction storage holds; raise neighborCacheSize")
        if st.status == _lib.TIMEOUT:
            raise RuntimeError("[IP] solve stopped by the device iteration guard")
        if st.status != _lib.OK:
            raise RuntimeError(f"[IP] solve failed with status {st.status}")

    def solve(self, dt):
        t0 = time.perf_counter()
        eng = self.engine(dt)
        eng.solve()
        st = eng.stats(0)
        self.apply_stats(st, (time.perf_counter() - t0) * 1000.0)

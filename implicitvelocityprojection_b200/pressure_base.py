"""PressureBase with the reference's plugin interface
(`scripts/sim/forces/pressure/pressure_base.py:280-506`).

Constructor `cls(particle_system, neighbour_search, config)`, the same solver
attributes (`tol_opt`, `max_iteration_opt`, `use_fixed_iters`, `omega`) read
from the same configuration keys, the same `stats_*` fields, and the same
`RuntimeError` texts.  The kernels run in the CUDA engine of the
`SimulationData`.
"""
from __future__ import annotations


class PressureBase:
    is_position_based = False

    def __init__(self, particle_system, neighbour_search, config):
        self.ps = particle_system
        self.ns = neighbour_search
        if getattr(neighbour_search, "ps", None) is None and hasattr(neighbour_search, "attach"):
            neighbour_search.attach(particle_system)
        self.cfg = config
        # pressure_base.py:314-317
        self.max_iteration_opt = int(config.get_cfg("maxOuterIters", 1000))
        self.use_fixed_iters = bool(config.get_cfg("fixedOuterIters", False))
        self.tol_opt = float(config.get_cfg("densityErrorTol", 1e-3))
        self.omega = float(config.get_cfg("omega", 10.0))
        # pressure_base.py:331-339
        self.stats_density_errors = []
        self.stats_iter_costs = []
        self.stats_pcg_iters = []
        self.stats_pos_residuals = []
        self.stats_outer_iters = 0
        self.stats_final_density_error = 0.0
        self.stats_final_pos_residual = 0.0
        self.stats_total_cost_ms = 0.0
        self.stats_overflow_particles = 0

    # the diagonal k = 1/(Aii + eps) lives with the particle state
    @property
    def k(self):
        return self.ps.k

    def engine(self, dt=None):
        return self.ps.engine(self, dt)

    def compute_density(self):
        """pressure_base.py:341-352 from the current lists and positions."""
        self.engine().compute_density()

    def compute_Aii(self):
        """pressure_base.py:354-365 from the current lists."""
        self.engine().compute_aii()

    def convergence_metric(self, err, pos_res):
        if getattr(self, "convergence_mode", 1) == 0:
            return pos_res, self.pos_tol, "pos residual"
        return err, self.tol_opt, "density err"

    def check_converged(self, err, n_updates, pos_res=0.0):
        """pressure_base.py:487-495."""
        metric, tol, name = self.convergence_metric(err, pos_res)
        if (not self.use_fixed_iters) and metric >= tol and n_updates >= self.max_iteration_opt:
            raise RuntimeError(f"[{type(self).__name__}] does not converge! {name}={metric:.2e} "
                               f"(tol={tol:.2e}) after {n_updates} iters")

    def reset_stats(self):
        self.stats_density_errors = []
        self.stats_iter_costs = []
        self.stats_pcg_iters = []
        self.stats_pos_residuals = []

    def solve(self, dt):
        pass

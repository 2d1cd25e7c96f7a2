"""NeighbourSearch with the reference's interface
(`scripts/sim/neighbour_search.py:81-179`).

The reference builds a Warp HashGrid (cell = support radius) and then a
fixed-size cache of neighbour ids and spiky gradients.  Here `build` and
`build_cache` run the engine's cell hash + counting sort + compact list build
(fused with density and Aii, which `Framework` reads right after).  The cache
arguments of `build_cache` are accepted for signature compatibility; the
lists live in the engine (export them with `SimulationData.neighbour_cache`).
"""
from __future__ import annotations

import math


class NeighbourSearch:
    def __init__(self, domain_size, support_radius: float, particle_data=None):
        self.support_radius = float(support_radius)
        self.grid_dims = tuple(max(1, int(math.ceil(float(domain_size[a]) / self.support_radius)))
                               for a in range(3))
        self.ps = particle_data
        self._built_for = None

    def attach(self, particle_data):
        self.ps = particle_data

    def build(self, positions=None, num_particles: int = None):
        """neighbour_search.py:116-129.  The grid build is part of build_cache
        (one fused pass); this records which particle set to index."""
        self._built_for = int(num_particles) if num_particles is not None else None

    def build_cache(self, positions=None, num_particles: int = None, cache_size: int = None, neighbor_count=None,
                    neighbor_ids=None, neighbor_gradW=None, solver=None):
        """neighbour_search.py:131-155: lists, plus density and k of every
        dynamic particle into ps.density / ps.k."""
        if self.ps is None:
            raise RuntimeError("NeighbourSearch needs the SimulationData: pass it to the constructor or attach()")
        self.ps.engine(solver).build()

    def recompute_gradW(self, *a, **k):
        """neighbour_search.py:157-179: the engine stores kernel-gradient
        weights that are rebuilt with the lists; nothing to do separately."""
        return None

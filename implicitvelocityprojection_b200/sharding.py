"""Multi-GPU placement of independent scenes.

A scene never spans GPUs (its solve needs every particle's neighbours each
phase); a batch or a request stream is split across ranks by whole scenes, one
process per GPU, with no data-path collective.  Ranks only agree on the
placement (a pure function of the scene list, computed identically
everywhere) and combine their measured totals at the end.
"""
from __future__ import annotations

import heapq
from typing import List, Sequence


def scene_cost(sc) -> float:
    """Expected work of one step of a scene: proportional to its fluid
    particles (every pass streams their neighbour rows), plus the per-particle
    passes over its boundary particles."""
    return float(sc.n_dynamic) + 0.1 * float(sc.n - sc.n_dynamic)


def assign_scenes(scenes: Sequence, world: int) -> List[List[int]]:
    """Longest-processing-time placement: scenes by decreasing cost, each to
    the rank with the least work so far (ties to the lower rank).  Returns the
    scene indices of every rank, each list in scene order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(scenes)), key=lambda i: (-scene_cost(scenes[i]), i))
    heap = [(0.0, r) for r in range(world)]
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + scene_cost(scenes[i]), r))
    return [sorted(ix) for ix in out]


def shard(scenes: Sequence, rank: int, world: int) -> list:
    """The scenes rank `rank` of `world` runs."""
    return [scenes[i] for i in assign_scenes(scenes, world)[rank]]


def combine_rate(particle_steps: float, seconds: float, group=None) -> float:
    """Whole-job particle-steps/s over ranks: the sum of the work divided by
    the slowest rank's time (torch.distributed, any backend)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return particle_steps / seconds
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else "cpu"
    w = torch.tensor([particle_steps], dtype=torch.float64, device=dev)
    t = torch.tensor([seconds], dtype=torch.float64, device=dev)
    dist.all_reduce(w, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(w.item()) / float(t.item())

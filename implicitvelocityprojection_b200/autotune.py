"""Autotuner of the engine's launch shape on the actual scenes.

The engine's neighbour sums run G lanes per particle in CTAs of G x T
threads (T particles per tile), either as persistent cooperative solves or as
one launch per phase, over full {J_ij, j} or compact {j, w_ij} neighbour rows
(identical bits), after a neighbour build by one thread per particle or one
warp per cell (identical lists).  Which choice is fastest depends on how many
tiles the scenes make per SM and on their neighbour counts, so the tuner times
every launch shape on copies of the scenes the caller will run (a few warm-up
steps, then a few CUDA-event-timed steps each), keeps the fastest, then times
both build kernels with that shape, each build launch timed on its own
inside five host-driven steps.  Choices are
cached per scene-set signature (scene count, fluid-particle total and largest
scene, each bucketed to powers of two, and the enabled forces), in memory and
optionally in a JSON file.

The reference fixes its launch shape (Warp's default block of 256 threads per
launch, and block_dim=128 for its tiled dot product,
scripts/sim/forces/pressure/pressure_base.py:425-436); this replaces that
choice.  Lane counts change the summation order of the neighbour sums, so
results of different candidates agree within the FP32 tolerance, not bit for
bit; the persistent and per-phase paths of one shape give identical bits.
"""
from __future__ import annotations

import dataclasses
import json
import math
import os
import time
from typing import Dict, List, Optional, Sequence, Tuple

# (lanes per particle, particles per CTA): 256- and 128-thread CTAs
SHAPES: Tuple[Tuple[int, int], ...] = ((2, 128), (4, 64), (8, 32), (2, 64), (4, 32), (8, 16))
# neighbour-row formats that give identical bits: full {J_ij, j} (16 B) and
# compact {j, w_ij} (8 B, J rebuilt from the positions).  Full rows win while
# the rows stay in L2; compact rows halve the row stream once they do not.
ROW_FORMATS: Tuple[int, ...] = (1, 2)
# neighbour builds with identical lists: one thread per particle, one warp per cell
BUILD_KERNELS: Tuple[int, ...] = (1, 2)
BUILD_REPS = 5

_CACHE: Dict[str, dict] = {}


@dataclasses.dataclass
class Trial:
    lanes_per_particle: int
    particles_per_block: int
    persistent: bool
    row_format: int
    ms_per_step: float

    def label(self) -> str:
        return (f"{self.lanes_per_particle}x{self.particles_per_block}/"
                f"{'persistent' if self.persistent else 'per-phase'}/{'full' if self.row_format == 1 else 'compact'}")


def signature(scenes: Sequence) -> str:
    """Cache key: scene count, total and largest fluid count (powers of two),
    pressure solvers and enabled forces."""
    nd = [int(sc.n_dynamic) for sc in scenes]
    b = lambda v: int(round(math.log2(max(v, 1))))  # noqa: E731
    forces = sorted({(int(getattr(sc, "pressure_method", 1)), int(sc.viscosity_method == 1 and sc.viscosity_coeff > 0),
                      int(getattr(sc, "surface_tension_method", 0) == 1 and getattr(sc, "surface_tension_coeff", 0) > 0))
                     for sc in scenes})
    return f"n{len(scenes)}-t{b(sum(nd))}-m{b(max(nd) if nd else 1)}-f{forces}"


def candidates(per_phase: bool = True, row_formats: Sequence[int] = ROW_FORMATS) -> List[Tuple[int, int, bool, int]]:
    out = []
    for rf in row_formats:
        out += [(g, t, True, rf) for g, t in SHAPES]
        if per_phase:
            out += [(g, t, False, rf) for g, t in SHAPES]
    return out


def _time_candidate(scenes, lanes, ppb, persistent, row_format, device, warmup, steps, base_options) -> float:
    import torch
    from .engine import Engine
    opts = dataclasses.replace(base_options, lanes_per_particle=lanes, particles_per_block=ppb,
                               persistent=persistent, row_format=row_format)
    copies = [dataclasses.replace(sc, x=sc.x.copy(), v=sc.v.copy()) for sc in scenes]
    eng = Engine(copies, device=device, options=opts)
    try:
        eng.build()
        eng.step(warmup)
        stream = torch.cuda.current_stream()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        eng.step(steps)
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b) / steps
    finally:
        eng.close()


def _time_build(scenes, lanes, ppb, persistent, row_format, build_kernel, device, warmup, reps,
                base_options) -> float:
    """Milliseconds per neighbour-build kernel launch of copies of `scenes`
    with the given build kernel, measured inside steps (ivp_profile_step:
    host-driven steps with CUDA events around every kernel), so the build
    finds the cache state a step leaves it: the slot-ordered positions the
    preceding reorder pass just wrote.  The two build kernels differ by a few
    percent of a step, less than the noise of a few timed steps."""
    from .engine import Engine
    opts = dataclasses.replace(base_options, lanes_per_particle=lanes, particles_per_block=ppb,
                               persistent=persistent, row_format=row_format, build_kernel=build_kernel)
    copies = [dataclasses.replace(sc, x=sc.x.copy(), v=sc.v.copy()) for sc in scenes]
    eng = Engine(copies, device=device, options=opts)
    try:
        eng.build()
        eng.step(max(warmup, 1))
        ms, launches = eng.profile_step(reps)["nbr_build"]
        return ms / launches
    finally:
        eng.close()


def tune(scenes: Sequence, device: str = "cuda", base_options=None, warmup: int = 2, steps: int = 3,
         per_phase: bool = True, cache_file: Optional[str] = None, force: bool = False) -> dict:
    """Times every candidate shape on copies of `scenes`, then both build
    kernels with the fastest shape, and returns {"choice":
    {lanes_per_particle, particles_per_block, persistent, row_format,
    build_kernel}, "table": [{shape, ms_per_step}], "build_ms", "signature",
    "cached"}."""
    from .engine import EngineOptions
    base = base_options or EngineOptions()
    key = signature(scenes)
    if not force:
        if key in _CACHE:
            return {**_CACHE[key], "cached": True}
        if cache_file and os.path.exists(cache_file):
            try:
                with open(cache_file) as f:
                    disk = json.load(f)
                if key in disk:
                    _CACHE[key] = disk[key]
                    return {**disk[key], "cached": True}
            except (OSError, ValueError):
                pass
    trials: List[Trial] = []
    t0 = time.perf_counter()
    # a caller that fixed the row format (e.g. the bf16 variant) keeps it
    rfs = ROW_FORMATS if base.row_format in (0, 1, 2) else (base.row_format,)
    for g, t, pers, rf in candidates(per_phase, rfs):
        ms = _time_candidate(scenes, g, t, pers, rf, device, warmup, steps, base)
        trials.append(Trial(g, t, pers, rf, ms))
    best = min(trials, key=lambda tr: tr.ms_per_step)
    build_ms = None
    if base.build_kernel == 0:
        # both build kernels with the fastest shape, each build launch timed
        # inside steps (a caller that fixed the build kernel keeps it)
        build_ms = {bk: _time_build(scenes, best.lanes_per_particle, best.particles_per_block, best.persistent,
                                    best.row_format, bk, device, warmup, BUILD_REPS, base)
                    for bk in BUILD_KERNELS}
    res = {"signature": key,
           "choice": {"lanes_per_particle": best.lanes_per_particle, "particles_per_block": best.particles_per_block,
                      "persistent": best.persistent, "row_format": best.row_format,
                      "build_kernel": min(build_ms, key=build_ms.get) if build_ms else base.build_kernel},
           "table": [{"shape": tr.label(), "ms_per_step": round(tr.ms_per_step, 4)} for tr in trials],
           "build_ms": None if build_ms is None else
           {{1: "thread per particle", 2: "warp per cell"}[bk]: round(ms, 4) for bk, ms in build_ms.items()},
           "tuning_s": round(time.perf_counter() - t0, 2), "steps_timed": steps}
    _CACHE[key] = res
    if cache_file:
        disk = {}
        if os.path.exists(cache_file):
            try:
                with open(cache_file) as f:
                    disk = json.load(f)
            except (OSError, ValueError):
                disk = {}
        disk[key] = res
        with open(cache_file, "w") as f:
            json.dump(disk, f, indent=1)
    return {**res, "cached": False}


def tuned_options(scenes: Sequence, device: str = "cuda", base_options=None, **kw):
    """EngineOptions with the tuned launch shape for `scenes`, and the tuning record."""
    from .engine import EngineOptions
    base = base_options or EngineOptions()
    res = tune(scenes, device=device, base_options=base, **kw)
    c = res["choice"]
    return dataclasses.replace(base, lanes_per_particle=c["lanes_per_particle"],
                               particles_per_block=c["particles_per_block"], persistent=c["persistent"],
                               row_format=c.get("row_format", base.row_format),
                               build_kernel=c.get("build_kernel", base.build_kernel)), res

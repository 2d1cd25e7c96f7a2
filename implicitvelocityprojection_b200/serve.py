"""Served form: a request loop over the IP step with continuous batching.

A request is one scene and a number of `Framework.forward()` steps.  The
server admits requests first-come first-served against a device-memory budget
(each scene's workspace plus its particle arrays), runs every admitted scene
in one batched engine (one set of launches per step, per-scene convergence
masks, scene results bit-identical to the scene run alone), and re-plans the
batch only at chunk boundaries: requests join or leave every `chunk_steps`
steps at most, so the engine rebuild is amortised over the chunk.  A scene's
step is a pure function of its (x, v) state, so carrying x and v across a
rebuild continues the scene exactly.

Time is either real (arrivals are waited for) or virtual (the clock advances
by the measured busy time and jumps over idle gaps), which gives the same
schedule for a saturated server without sleeping through idle periods.
"""
from __future__ import annotations

import collections
import dataclasses
import time
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

from .scenes import Request, Scene

# particle arrays bound per particle: x, v (12 B each), m, density0,
# is_dynamic, material, density, k (4 B each)
ARRAY_BYTES_PER_PARTICLE = 48


@dataclasses.dataclass
class Result:
    rid: int
    arrival_s: float
    admit_s: float
    finish_s: float
    steps: int
    n_dynamic: int
    status: int            # 0 ok, else the first failing solve's ivp status
    x: Optional[np.ndarray] = None
    v: Optional[np.ndarray] = None

    @property
    def latency_s(self) -> float:
        return self.finish_s - self.arrival_s

    @property
    def wait_s(self) -> float:
        return self.admit_s - self.arrival_s


@dataclasses.dataclass
class Report:
    results: List[Result]
    makespan_s: float
    busy_s: float
    rebuilds: int
    rebuild_s: float
    particle_steps: int
    max_active: int
    rejected: int

    def summary(self) -> dict:
        lat = np.array([r.latency_s for r in self.results]) if self.results else np.zeros(1)
        wait = np.array([r.wait_s for r in self.results]) if self.results else np.zeros(1)
        ok = sum(r.status == 0 for r in self.results)
        return {
            "requests": len(self.results) + self.rejected, "completed": ok,
            "failed": len(self.results) - ok, "rejected": self.rejected,
            "particle_steps": self.particle_steps,
            "throughput": self.particle_steps / max(self.makespan_s, 1e-9),
            "busy_throughput": self.particle_steps / max(self.busy_s, 1e-9),
            "makespan_s": self.makespan_s, "busy_s": self.busy_s,
            "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
            "wait_p50_s": float(np.percentile(wait, 50)), "wait_p99_s": float(np.percentile(wait, 99)),
            "rebuilds": self.rebuilds, "rebuild_s": self.rebuild_s, "max_active": self.max_active,
        }


class _Active:
    __slots__ = ("rid", "req", "scene", "remaining", "admit_s", "status", "footprint")

    def __init__(self, rid, req, scene, admit_s, footprint):
        self.rid = rid
        self.req = req
        self.scene = scene
        self.remaining = req.steps
        self.admit_s = admit_s
        self.status = 0
        self.footprint = footprint


class Server:
    """Continuous-batching request loop.

    `engine_factory(scenes)` returns an object with `build()`, `step(n)`,
    `get(name, i)` (host copies of "x"/"v"), `raw_stats(i).status` and
    `reset_counters()`; by default the CUDA `Engine`.  `footprint(scene)`
    gives a scene's device bytes; by default its engine workspace plus its
    particle arrays."""

    def __init__(self, engine_factory: Optional[Callable] = None, footprint: Optional[Callable] = None,
                 hbm_budget_bytes: float = 150e9, chunk_steps: int = 50, keep_state: bool = True,
                 device: str = "cuda", options=None):
        self.chunk_steps = int(chunk_steps)
        self.budget = float(hbm_budget_bytes)
        self.keep_state = keep_state
        self.device = device
        if engine_factory is None:
            from .engine import Engine

            def engine_factory(scenes, arrays=None, _dev=device, _opt=options):
                return Engine(list(scenes), device=_dev, options=_opt, arrays=arrays)
        self.engine_factory = engine_factory
        if footprint is None:
            from .engine import workspace_bytes

            def footprint(sc, _opt=options):
                return workspace_bytes([sc], _opt) + ARRAY_BYTES_PER_PARTICLE * sc.n
        self.footprint = footprint

    _KEYS = ("x", "v", "m", "density0", "is_dynamic", "material", "density", "k")

    def _carry(self, eng, members, active) -> dict:
        """Bound arrays of the next engine, in `active` order: slices of the
        current engine's tensors for continuing scenes, uploads for new ones."""
        import torch
        pos = {id(a): i for i, a in enumerate(members)}
        parts = {k: [] for k in self._KEYS}
        for a in active:
            i = pos.get(id(a))
            if i is not None:
                sl = eng.scene_slice(i)
                for k in self._KEYS:
                    parts[k].append(eng.arrays[k][sl])
                continue
            sc = a.scene
            m, _ = sc.masses()
            dev = eng.arrays["x"].device
            host = {"x": sc.x, "v": sc.v, "m": m, "density0": sc.density0,
                    "is_dynamic": sc.is_dynamic.astype(np.int32), "material": sc.material.astype(np.int32),
                    "density": sc.density0, "k": np.zeros(sc.n, np.float32)}
            for k in self._KEYS:
                parts[k].append(torch.from_numpy(np.ascontiguousarray(host[k])).to(dev, non_blocking=False))
        return {k: torch.cat(v).contiguous() for k, v in parts.items()}

    def run(self, requests: Sequence[Request], realtime: bool = False,
            on_result: Optional[Callable[[Result], None]] = None) -> Report:
        pending = collections.deque(sorted(enumerate(requests), key=lambda kv: kv[1].arrival_s))
        queue: collections.deque = collections.deque()
        active: List[_Active] = []
        results: List[Result] = []
        rejected = 0
        eng = None
        members: List[_Active] = []  # the scenes of `eng`, in engine order
        dirty = False
        busy = rebuild_s = 0.0
        rebuilds = 0
        psteps = 0
        max_active = 0
        wall0 = time.perf_counter()
        vclock = 0.0

        def now() -> float:
            return time.perf_counter() - wall0 if realtime else vclock

        while pending or queue or active:
            t = now()
            while pending and pending[0][1].arrival_s <= t:
                queue.append(pending.popleft())
            # first-come first-served admission against the memory budget
            used = sum(a.footprint for a in active)
            while queue:
                rid, req = queue[0]
                fp = self.footprint(req.scene)
                if fp > self.budget:  # can never fit
                    queue.popleft()
                    rejected += 1
                    continue
                if used + fp > self.budget:
                    break
                queue.popleft()
                sc = dataclasses.replace(req.scene, x=req.scene.x.copy(), v=req.scene.v.copy())
                active.append(_Active(rid, req, sc, max(t, req.arrival_s), fp))
                used += fp
                dirty = True
            if not active:
                if pending:
                    nxt = pending[0][1].arrival_s
                    if realtime:
                        time.sleep(max(0.0, nxt - now()))
                    else:
                        vclock = max(vclock, nxt)
                continue
            max_active = max(max_active, len(active))
            if dirty:
                t0 = time.perf_counter()
                arrays = None
                if eng is not None:
                    live = set(id(a) for a in active)
                    if hasattr(eng, "arrays") and hasattr(eng, "scene_slice"):
                        # continuing scenes carry their bound arrays into the
                        # next engine on the device; new scenes are uploaded
                        arrays = self._carry(eng, members, active)
                    else:
                        for i, a in enumerate(members):
                            if id(a) in live:
                                a.scene.x = eng.get("x", i)
                                a.scene.v = eng.get("v", i)
                    del eng
                eng = self.engine_factory([a.scene for a in active], arrays) if arrays is not None \
                    else self.engine_factory([a.scene for a in active])
                eng.build()
                members = list(active)
                rebuilds += 1
                dirty = False
                dt_rb = time.perf_counter() - t0
                rebuild_s += dt_rb
                busy += dt_rb
                if not realtime:
                    vclock += dt_rb
            n = min(self.chunk_steps, min(a.remaining for a in active))
            t0 = time.perf_counter()
            eng.step(n)
            st = []
            for i in range(len(active)):  # synchronises
                rs = eng.raw_stats(i)
                st.append(int(rs.last_failure or rs.status or 1) if rs.failed_solves > 0 else 0)
            dt_run = time.perf_counter() - t0
            busy += dt_run
            if not realtime:
                vclock += dt_run
            psteps += n * sum(a.scene.n_dynamic for a in active)
            done = []
            for i, a in enumerate(active):
                if st[i] != 0 and a.status == 0:
                    a.status = int(st[i])
                a.remaining -= n
                if a.remaining <= 0 or a.status != 0:
                    done.append(i)
            if done:
                t_fin = now()
                for i in done:
                    a = active[i]
                    r = Result(rid=a.rid, arrival_s=a.req.arrival_s, admit_s=a.admit_s, finish_s=t_fin,
                               steps=a.req.steps - max(a.remaining, 0), n_dynamic=a.scene.n_dynamic,
                               status=a.status)
                    if self.keep_state:
                        r.x, r.v = eng.get("x", i), eng.get("v", i)
                    results.append(r)
                    if on_result is not None:
                        on_result(r)
                gone = set(done)
                active = [a for i, a in enumerate(active) if i not in gone]
                dirty = True
                if not active:
                    del eng
                    eng = None
                    members = []
            eng_reset = getattr(eng, "reset_counters", None)
            if eng_reset is not None:
                eng_reset()
        makespan = now() if not realtime else time.perf_counter() - wall0
        results.sort(key=lambda r: r.rid)
        return Report(results=results, makespan_s=makespan, busy_s=busy, rebuilds=rebuilds,
                      rebuild_s=rebuild_s, particle_steps=psteps, max_active=max_active, rejected=rejected)

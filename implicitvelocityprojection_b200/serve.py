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

Two loops share the admission policy.  `run_realtime` is the served form:
arrivals are read off the wall clock, each chunk is launched asynchronously
(one CUDA-event pair per step, giving the per-step device latency), and
while it runs on the device the host admits new arrivals and prepares the
next batch: the next engine is created, its new scenes uploaded and its
graphs instantiated on a side stream, so the swap at the chunk boundary is
only device-side copies of the continuing scenes' state and a neighbour
build.  `run` (realtime=False) advances a virtual clock by the measured busy
time and jumps over idle gaps: the same schedule for a saturated server,
without sleeping through idle periods.
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
    steps: int             # steps whose solve succeeded (all requested steps for a completed request)
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

    step_ms: Optional[List[float]] = None  # device time of every batched step (real-clock loop)
    swap_ms: Optional[List[float]] = None  # host time of every chunk-boundary swap (real-clock loop)

    def summary(self) -> dict:
        lat = np.array([r.latency_s for r in self.results]) if self.results else np.zeros(1)
        wait = np.array([r.wait_s for r in self.results]) if self.results else np.zeros(1)
        ok = sum(r.status == 0 for r in self.results)
        extra = {}
        if self.step_ms:
            st = np.array(self.step_ms)
            extra = {"steps": int(st.size), "step_p50_ms": float(np.percentile(st, 50)),
                     "step_p99_ms": float(np.percentile(st, 99)), "step_mean_ms": float(st.mean())}
        if self.swap_ms:
            sw = np.array(self.swap_ms)
            extra.update({"swaps": int(sw.size), "swap_p50_ms": float(np.percentile(sw, 50)),
                          "swap_max_ms": float(sw.max())})
        return {**extra,
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
            st, ok = [], []
            for i in range(len(active)):  # synchronises
                rs = eng.raw_stats(i)
                failed = int(getattr(rs, "failed_solves", 0))
                st.append(int(rs.last_failure or rs.status or 1) if failed > 0 else 0)
                # steps of this chunk whose solve succeeded: a scene whose solve
                # failed is credited only with those (the counters are reset
                # after every chunk)
                ok.append(n if failed == 0 else max(0, min(n, int(getattr(rs, "solves", n)) - failed)))
            dt_run = time.perf_counter() - t0
            busy += dt_run
            if not realtime:
                vclock += dt_run
            psteps += sum(k * a.scene.n_dynamic for k, a in zip(ok, active))
            done = []
            for i, a in enumerate(active):
                if st[i] != 0 and a.status == 0:
                    a.status = int(st[i])
                a.remaining -= n if st[i] == 0 else ok[i]
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

    # ------------------------------------------------------------ real clock

    @staticmethod
    def _release(eng, main):
        """Device memory of an engine about to be dropped: the caching
        allocator may hand it out again only after the work enqueued on the
        main stream so far (the boundary copies read it) has run."""
        if main is None or eng is None:
            return
        for t in list(getattr(eng, "arrays", {}).values()) + [getattr(eng, "_ws_raw", None)]:
            if t is not None and getattr(t, "is_cuda", False):
                t.record_stream(main)

    def _side_stream(self):
        try:
            import torch
            if torch.cuda.is_available() and str(self.device).startswith("cuda"):
                return torch.cuda.Stream(device=self.device), torch.cuda.current_stream(self.device)
        except Exception:
            pass
        return None, None

    def _prepare(self, eng, members, nxt, side):
        """The engine of the next chunk over `nxt` (continuing members first
        keep their order), created while the current chunk runs.  Returns
        (engine, carry): carry lists (new slice, old slice) of the continuing
        scenes, whose x and v are copied at the boundary.  New scenes and every
        scene's constant arrays are uploaded now, on the side stream."""
        import contextlib
        pos = {id(a): i for i, a in enumerate(members)}
        carry = []
        ctx = contextlib.nullcontext()
        if side is not None:
            import torch
            ctx = torch.cuda.stream(side)
        with ctx:
            if eng is not None and hasattr(eng, "arrays"):
                import torch
                parts = {k: [] for k in self._KEYS}
                off = 0
                for a in nxt:
                    i = pos.get(id(a))
                    n = a.scene.n
                    if i is not None:
                        sl = eng.scene_slice(i)
                        for k in self._KEYS:
                            if k in ("x", "v"):  # still moving: copied at the boundary
                                parts[k].append(torch.empty_like(eng.arrays[k][sl]))
                            else:
                                parts[k].append(eng.arrays[k][sl].clone())
                        carry.append((slice(off, off + n), sl))
                    else:
                        sc = a.scene
                        m, _ = sc.masses()
                        host = {"x": sc.x, "v": sc.v, "m": m, "density0": sc.density0,
                                "is_dynamic": sc.is_dynamic.astype(np.int32),
                                "material": sc.material.astype(np.int32), "density": sc.density0,
                                "k": np.zeros(sc.n, np.float32)}
                        dev = eng.arrays["x"].device
                        for k in self._KEYS:
                            t = torch.from_numpy(np.ascontiguousarray(host[k]))
                            parts[k].append(t.pin_memory().to(dev, non_blocking=True))
                    off += n
                arrays = {k: torch.cat(v).contiguous() for k, v in parts.items()}
                new = self.engine_factory([a.scene for a in nxt], arrays)
            else:
                for a in nxt:  # host-side engines: carry through the scenes
                    i = pos.get(id(a))
                    if i is not None and eng is not None:
                        a.scene.x = eng.get("x", i)
                        a.scene.v = eng.get("v", i)
                new = self.engine_factory([a.scene for a in nxt])
            prep = getattr(new, "prepare", None)
            if prep is not None:
                prep()
        return new, carry

    def run_realtime(self, requests: Sequence[Request], on_result: Optional[Callable[[Result], None]] = None,
                     poll_s: float = 0.0005) -> Report:
        """The served form on the wall clock: requests are admitted as they
        arrive, also while a chunk runs on the device, and join the batch at
        the next chunk boundary."""
        side, main = self._side_stream()
        pending = collections.deque(sorted(enumerate(requests), key=lambda kv: kv[1].arrival_s))
        queue: collections.deque = collections.deque()
        joining: List[_Active] = []      # admitted, not yet in the engine
        members: List[_Active] = []      # the scenes of `eng`, in engine order
        results: List[Result] = []
        eng, chunk, n_chunk = None, None, 0
        plan = None                      # (engine, carry, members) prepared for the next chunk
        rejected = psteps = rebuilds = max_active = 0
        busy = rebuild_s = 0.0
        step_ms, swap_ms = [], []
        wall0 = time.perf_counter()

        def now():
            return time.perf_counter() - wall0

        def admit():
            t = now()
            while pending and pending[0][1].arrival_s <= t:
                queue.append(pending.popleft())
            used = sum(a.footprint for a in members) + sum(a.footprint for a in joining)
            while queue:
                rid, req = queue[0]
                fp = self.footprint(req.scene)
                if fp > self.budget:
                    queue.popleft()
                    nonlocal_rejected[0] += 1
                    continue
                if used + fp > self.budget:
                    break
                queue.popleft()
                sc = dataclasses.replace(req.scene, x=req.scene.x.copy(), v=req.scene.v.copy())
                joining.append(_Active(rid, req, sc, t, fp))
                used += fp

        nonlocal_rejected = [0]

        def launch():
            nonlocal chunk, n_chunk
            n_chunk = min(self.chunk_steps, min(a.remaining for a in members))
            chunk = eng.step_chunk(n_chunk)

        while pending or queue or joining or members:
            admit()
            if eng is None:
                if not joining:
                    if pending:
                        time.sleep(max(0.0, min(poll_s * 20, pending[0][1].arrival_s - now())))
                    continue
                t0 = time.perf_counter()
                members, joining = joining, []
                eng, _ = self._prepare(None, [], members, side)
                if side is not None:
                    main.wait_stream(side)
                eng.build()
                rebuilds += 1
                rebuild_s += time.perf_counter() - t0
                max_active = max(max_active, len(members))
                launch()
                continue
            # a chunk is in flight: prepare the next batch when it will change
            finishing = [a for a in members if a.remaining <= n_chunk]
            if plan is None and (finishing or joining):
                nxt = [a for a in members if a.remaining > n_chunk] + list(joining)
                if nxt:
                    new, carry = self._prepare(eng, members, nxt, side)
                    plan = (new, carry, nxt, len(joining))
                else:
                    plan = (None, [], [], 0)
            if not chunk.done():
                time.sleep(poll_s)
                continue
            # chunk boundary
            t_b = time.perf_counter()
            chunk.wait()
            sms = chunk.step_ms()
            step_ms.extend(sms)
            busy += sum(sms) / 1000.0
            stats = eng.raw_stats_all() if hasattr(eng, "raw_stats_all") else \
                [eng.raw_stats(i) for i in range(len(members))]
            t_fin = now()
            failed_any = False
            for a, rs in zip(members, stats):
                failed = int(getattr(rs, "failed_solves", 0))
                ok = n_chunk if failed == 0 else max(0, min(n_chunk, int(getattr(rs, "solves", n_chunk)) - failed))
                psteps += ok * a.scene.n_dynamic
                if failed and a.status == 0:
                    a.status = int(rs.last_failure or rs.status or 1)
                    failed_any = True
                a.remaining -= n_chunk if failed == 0 else ok
            done = [i for i, a in enumerate(members) if a.remaining <= 0 or a.status != 0]
            for i in done:
                a = members[i]
                r = Result(rid=a.rid, arrival_s=a.req.arrival_s, admit_s=a.admit_s, finish_s=t_fin,
                           steps=a.req.steps - max(a.remaining, 0), n_dynamic=a.scene.n_dynamic, status=a.status)
                if self.keep_state:
                    r.x, r.v = eng.get("x", i), eng.get("v", i)
                results.append(r)
                if on_result is not None:
                    on_result(r)
            eng_reset = getattr(eng, "reset_counters", None)
            if eng_reset is not None:
                eng_reset()
            gone = set(done)
            live = [a for i, a in enumerate(members) if i not in gone]
            if plan is not None and (failed_any or [id(a) for a in plan[2][:len(plan[2]) - plan[3]]] !=
                                     [id(a) for a in live]):
                plan = None  # a failure changed the membership: prepare again
            if plan is None and not joining and len(live) == len(members):
                launch()  # same batch, same engine
                swap_ms.append((time.perf_counter() - t_b) * 1000.0)
                continue
            if plan is None:
                nxt = live + list(joining)
                plan = (self._prepare(eng, members, nxt, side) + (nxt, len(joining))) if nxt else (None, [], [], 0)
            new, carry, nxt, n_join = plan
            plan = None
            joined = nxt[len(nxt) - n_join:] if n_join else []
            joining = [a for a in joining if all(a is not b for b in joined)]
            if new is not None and hasattr(new, "arrays") and side is not None:
                main.wait_stream(side)
                for nsl, osl in carry:
                    for k in ("x", "v"):
                        new.arrays[k][nsl].copy_(eng.arrays[k][osl])
            self._release(eng, main)
            del eng
            eng, members = new, nxt
            if eng is None:
                chunk = None
                continue
            eng.build()
            rebuilds += 1
            max_active = max(max_active, len(members))
            launch()
            dt_sw = time.perf_counter() - t_b
            rebuild_s += dt_sw
            swap_ms.append(dt_sw * 1000.0)
        makespan = now()
        results.sort(key=lambda r: r.rid)
        return Report(results=results, makespan_s=makespan, busy_s=busy, rebuilds=rebuilds, rebuild_s=rebuild_s,
                      particle_steps=psteps, max_active=max_active, rejected=nonlocal_rejected[0],
                      step_ms=step_ms, swap_ms=swap_ms)

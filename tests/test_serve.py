"""Served form: the request loop's scheduling on CPU with a stand-in engine,
and on the GPU bit-identity of a served request with the scene run alone."""
import dataclasses
import time

import numpy as np
import pytest

from implicitvelocityprojection_b200 import scenes as S
from implicitvelocityprojection_b200.serve import Server


class _Stats:
    status = 0
    failed_solves = 0
    last_failure = 0


class FakeEngine:
    """Steps every scene by adding the step count to x (so a test can check
    that state is carried exactly across rebuilds)."""
    live = 0
    peak = 0
    built = []

    def __init__(self, scenes):
        self.scenes = [dataclasses.replace(s, x=s.x.copy(), v=s.v.copy()) for s in scenes]
        FakeEngine.built.append([s.name for s in scenes])

    def build(self):
        pass

    def step(self, n):
        for s in self.scenes:
            s.x = s.x + np.float32(n)

    def raw_stats(self, i):
        return _Stats()

    def get(self, name, i):
        return getattr(self.scenes[i], name).copy()

    def reset_counters(self):
        pass


def _req(t, n, steps, name):
    sc = S.Scene(x=np.zeros((n, 3), np.float32), v=np.zeros((n, 3), np.float32),
                 is_dynamic=np.ones(n, np.int32), material=np.ones(n, np.int32),
                 density0=np.full(n, 1000.0, np.float32), particle_radius=0.01,
                 domain_size=np.array([1.0, 1.0, 1.0], np.float32), name=name)
    return S.Request(arrival_s=t, scene=sc, steps=steps)


def test_fcfs_admission_budget_and_state_carry():
    reqs = [_req(0.0, 10, 7, "a"), _req(0.0, 20, 12, "b"), _req(0.0, 15, 5, "c"), _req(0.5, 5, 9, "d")]
    budget = 35  # footprint = particle count: a + b fit, c waits
    FakeEngine.built = []
    srv = Server(engine_factory=FakeEngine, footprint=lambda sc: sc.n, hbm_budget_bytes=budget, chunk_steps=4)
    rep = srv.run(reqs)
    assert [r.rid for r in rep.results] == [0, 1, 2, 3]
    for r, q in zip(rep.results, reqs):
        assert r.status == 0 and r.steps == q.steps
        assert np.all(r.x == np.float32(q.steps)), (r.rid, r.x[0])  # exact across rebuilds
    # never more than the budget resident, and c (first in line) is admitted before d
    for names in FakeEngine.built:
        assert sum({"a": 10, "b": 20, "c": 15, "d": 5}[n] for n in names) <= budget
    first = {n: i for i, names in reversed(list(enumerate(FakeEngine.built))) for n in names}
    assert first["c"] <= first["d"]
    s = rep.summary()
    assert s["completed"] == 4 and s["rejected"] == 0 and s["particle_steps"] == 10 * 7 + 20 * 12 + 15 * 5 + 5 * 9


def test_oversized_request_rejected_and_idle_gaps_skipped():
    reqs = [_req(0.0, 50, 3, "big"), _req(100.0, 5, 3, "late")]
    srv = Server(engine_factory=FakeEngine, footprint=lambda sc: sc.n, hbm_budget_bytes=10, chunk_steps=2)
    rep = srv.run(reqs)
    assert rep.rejected == 1
    assert len(rep.results) == 1 and rep.results[0].rid == 1
    assert rep.results[0].admit_s >= 100.0  # virtual clock jumped to the arrival


class _Failed:
    status = 0
    solves = 4        # the chunk's four steps, one of which failed
    failed_solves = 1
    last_failure = 3  # IVP_ERR_NOT_CONVERGED


class FailingEngine(FakeEngine):
    """A scene named "bad" reports a failed solve after every chunk."""

    def raw_stats(self, i):
        return _Failed() if self.scenes[i].name == "bad" else _Stats()


def test_failed_request_leaves_batch_others_continue():
    """A request whose solve fails finishes at the end of that chunk with the
    solve's status and leaves the batch, credited only with the steps whose
    solve succeeded; the requests batched with it run to their end with their
    state carried exactly, as if it had never been there."""
    reqs = [_req(0.0, 10, 9, "a"), _req(0.0, 5, 20, "bad"), _req(0.0, 8, 6, "c")]
    FakeEngine.built = []
    srv = Server(engine_factory=FailingEngine, footprint=lambda sc: sc.n, hbm_budget_bytes=1000, chunk_steps=4)
    rep = srv.run(reqs)
    by = {r.rid: r for r in rep.results}
    assert by[1].status == 3 and by[1].steps == 3
    for rid in (0, 2):
        assert by[rid].status == 0 and by[rid].steps == reqs[rid].steps
        assert np.all(by[rid].x == np.float32(reqs[rid].steps))
    assert all("bad" not in names for names in FakeEngine.built[1:])  # re-planned without it
    s = rep.summary()
    assert s["completed"] == 2 and s["failed"] == 1 and s["rejected"] == 0
    assert s["particle_steps"] == 10 * 9 + 8 * 6 + 5 * 3  # the failed step is not counted


class _FakeChunk:
    """n steps that take `step_s` each on a pretend device."""

    def __init__(self, n, step_s):
        self.n, self.step_s = n, step_s
        self.t_end = time.perf_counter() + n * step_s

    def done(self):
        return time.perf_counter() >= self.t_end

    def wait(self):
        time.sleep(max(0.0, self.t_end - time.perf_counter()))

    def step_ms(self):
        return [1000.0 * self.step_s] * self.n


class ChunkedFakeEngine(FakeEngine):
    """FakeEngine whose chunks run asynchronously for n * step_s of wall time
    (the state is final at launch, as a device's would be at the boundary);
    records when each engine was created."""
    step_s = 0.01
    created = []

    def __init__(self, scenes):
        super().__init__(scenes)
        ChunkedFakeEngine.created.append((time.perf_counter(), [s.name for s in scenes]))

    def step_chunk(self, n):
        self.step(n)
        return _FakeChunk(n, self.step_s)

    def raw_stats_all(self):
        return [_Stats() for _ in self.scenes]


def test_realtime_admits_while_a_chunk_is_in_flight():
    """On the wall clock: b arrives while a's first chunk (20 steps, 0.2 s)
    runs; it is admitted at once and the next batch's engine is created
    before that chunk ends, so b joins at the first boundary.  State is
    carried exactly and per-step latencies are reported."""
    reqs = [_req(0.0, 10, 40, "a"), _req(0.05, 5, 10, "b")]
    FakeEngine.built = []
    ChunkedFakeEngine.created = []
    srv = Server(engine_factory=ChunkedFakeEngine, footprint=lambda sc: sc.n, hbm_budget_bytes=100, chunk_steps=20)
    rep = srv.run_realtime(reqs)
    by = {r.rid: r for r in rep.results}
    assert by[0].status == 0 and by[1].status == 0
    assert np.all(by[0].x == np.float32(40)) and np.all(by[1].x == np.float32(10))
    assert by[1].admit_s < 0.2  # admitted during the first chunk
    c0 = ChunkedFakeEngine.created[0][0]  # a's engine: its first chunk starts right after
    made = [(t - c0, names) for t, names in ChunkedFakeEngine.created]
    ab = [t for t, names in made if names == ["a", "b"]]
    assert ab and ab[0] < 0.2, made  # the next batch was prepared while the chunk ran
    assert by[1].finish_s < 0.45  # joined at the first boundary (0.2 s) and ran 10 steps
    s = rep.summary()
    # batched steps: 20 of a alone, 10 of the pair (b's remaining steps), 10 of a alone
    assert s["steps"] == 40 and abs(s["step_p50_ms"] - 10.0) < 1e-9
    assert s["particle_steps"] == 10 * 40 + 5 * 10


def test_workspace_footprint_grows_with_particles():
    from implicitvelocityprojection_b200.engine import workspace_bytes
    small = workspace_bytes([S.random_column(3000, 2.0, seed=1)])
    big = workspace_bytes([S.random_column(30000, 2.0, seed=1)])
    assert 0 < small < big


@pytest.mark.gpu
def test_served_request_equals_scene_alone():
    """Requests joining and leaving at chunk boundaries (engine rebuilt each
    time) end bit-identical to each scene stepped alone."""
    from implicitvelocityprojection_b200.engine import Engine
    scs = [S.random_column(2500, 1.5, seed=41), S.small_dam_break(3000, seed=42), S.random_column(4000, 3.0, seed=43)]
    steps = [9, 6, 8]
    reqs = [S.Request(arrival_s=t, scene=sc, steps=n) for t, sc, n in zip((0.0, 0.0, 1e-4), scs, steps)]
    rep = Server(chunk_steps=3).run(reqs)
    assert rep.rebuilds >= 2
    for r, sc, n in zip(rep.results, scs, steps):
        assert r.status == 0
        alone = Engine([sc])
        alone.build()
        alone.step(n)
        assert np.array_equal(r.x, alone.get("x")), r.rid
        assert np.array_equal(r.v, alone.get("v")), r.rid


@pytest.mark.gpu
def test_realtime_served_request_equals_scene_alone():
    """The wall-clock loop on the GPU: requests arriving while a chunk runs
    join at the next boundary through an engine prepared on a side stream
    (continuing scenes' state copied on the device); each result equals its
    scene stepped alone, bit for bit, and per-step latencies are reported."""
    from implicitvelocityprojection_b200.engine import Engine
    scs = [S.random_column(2500, 1.5, seed=51), S.small_dam_break(3000, seed=52), S.random_column(4000, 3.0, seed=53)]
    steps = [30, 12, 20]
    reqs = [S.Request(arrival_s=t, scene=sc, steps=n) for t, sc, n in zip((0.0, 0.005, 0.01), scs, steps)]
    rep = Server(chunk_steps=8).run_realtime(reqs)
    assert rep.rebuilds >= 2 and rep.summary()["steps"] >= 30
    for r, sc, n in zip(rep.results, scs, steps):
        assert r.status == 0 and r.steps == n
        alone = Engine([sc])
        alone.build()
        alone.step(n)
        assert np.array_equal(r.x, alone.get("x")), r.rid
        assert np.array_equal(r.v, alone.get("v")), r.rid

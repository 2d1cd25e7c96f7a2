"""Multi-rank placement of independent scenes, on CPU: two `gloo` ranks split
a batch by whole scenes (no data-path collective), step their scenes with the
oracle, and combine the totals; every scene's result equals the single-process
run, and the placement is disjoint, complete and balanced."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from implicitvelocityprojection_b200 import scenes as S
from implicitvelocityprojection_b200.sharding import assign_scenes, scene_cost, shard


def _batch():
    return S.batch_mix(n_scenes=6, lo=300, hi=1500, seed=3)


def test_assignment_disjoint_complete_balanced():
    scs = S.batch_mix(n_scenes=64, seed=0)
    for world in (1, 2, 3, 8):
        parts = assign_scenes(scs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(scs)))
        loads = [sum(scene_cost(scs[i]) for i in p) for p in parts]
        # LPT bound: no rank above the mean by more than the largest scene
        assert max(loads) - sum(loads) / world <= max(scene_cost(s) for s in scs) + 1e-6
    with pytest.raises(ValueError):
        assign_scenes(scs, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    import datetime
    import torch
    import torch.distributed as dist
    from oracle import oracle as O
    from implicitvelocityprojection_b200.sharding import combine_rate
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        scs = _batch()
        mine = assign_scenes(scs, world)[rank]
        res = {}
        work = 0.0
        for i in mine:
            st = O.State.from_scene(scs[i])
            st.rebuild()
            st.step(fast=False)
            res[i] = (st.x.copy(), st.v.copy(), st.status)
            work += scs[i].n_dynamic
        # rank r claims 1 + r seconds: the combined rate uses the slowest rank
        rate = combine_rate(work, 1.0 + rank)
        got = [None] * world
        dist.all_gather_object(got, sorted(res))
        out.put((rank, res, rate, got))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_a_batch():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    outs = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    scs = _batch()
    total = sum(sc.n_dynamic for sc in scs)
    by_rank = {r: (res, rate, got) for r, res, rate, got in outs}
    claimed = [sorted(by_rank[r][0]) for r in range(world)]
    assert sorted(claimed[0] + claimed[1]) == list(range(len(scs)))
    assert not set(claimed[0]) & set(claimed[1])
    for r in range(world):
        assert by_rank[r][2] == claimed  # every rank saw the same placement
        assert by_rank[r][1] == pytest.approx(total / 2.0)  # sum of work / max of times
    # each scene's result equals the single-process run
    from oracle import oracle as O
    for r in range(world):
        for i, (x, v, status) in by_rank[r][0].items():
            st = O.State.from_scene(scs[i])
            st.rebuild()
            st.step(fast=False)
            assert status == 0
            assert np.array_equal(x, st.x) and np.array_equal(v, st.v), i
    assert [len(shard(scs, r, world)) for r in range(world)] == [len(c) for c in claimed]

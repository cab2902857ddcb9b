"""Replica sharding and the max-over-ranks timing with two gloo ranks on the
CPU (the multi-GPU path has no data-path collective; this is its host
logic)."""

import os
import socket

import pytest
import torch.multiprocessing as mp

from proresraw_rs_b200 import replicas as R


def test_shard_deals_round_robin_and_covers_everything():
    items = list(range(17))
    parts = [R.shard(items, r, 3) for r in range(3)]
    assert parts[0] == [0, 3, 6, 9, 12, 15]
    assert sorted(sum(parts, [])) == items
    with pytest.raises(ValueError):
        R.shard(items, 3, 3)


def test_single_process_reductions_are_identity():
    assert R.reduce_max(2.5) == 2.5 and R.reduce_sum(4.0) == 4.0


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        w, r, lr = R.world()
        mine = R.shard(list(range(10)), r, w)
        # Rank-dependent "times": the slowest rank's value wins.
        slowest = R.reduce_max(1.0 + r)
        total = R.reduce_sum(len(mine))
        out[rank] = (w, r, mine, slowest, total)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_share_the_frames_and_agree_on_the_slowest():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs)
        res = dict(out)
    assert res[0][2] == [0, 2, 4, 6, 8] and res[1][2] == [1, 3, 5, 7, 9]
    assert res[0][3] == res[1][3] == 2.0
    assert res[0][4] == res[1][4] == 10.0

"""Multi-GPU logic of bench.py on CPU ranks (gloo, world size 2): each rank
owns disjoint queries, and the step time is the maximum over ranks."""
from __future__ import annotations

import os

import pytest
import torch.multiprocessing as mp


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    seeds = bench.shard_seeds(4, rank)
    step_ms = 10.0 + rank * 5.0
    mx = bench.reduce_max(step_ms, dist, "cpu")
    dist.barrier()
    out.put((rank, seeds, mx))
    dist.destroy_process_group()


def test_ranks_shard_queries_and_take_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    seeds0, seeds1 = res[0][1], res[1][1]
    assert not set(seeds0) & set(seeds1)
    assert len(set(seeds0)) == 4
    assert res[0][2] == res[1][2] == 15.0

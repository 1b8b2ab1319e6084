"""Several GPUs = independent replicas or shards of a batch (the advance has
no exchange step). Checked on CPU with world_size-2 gloo process groups: the
case partition every rank computes on its own is disjoint, complete and
balanced, and the bench's whole-job throughput uses the slowest rank's time."""
import os
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT

sys.path.insert(0, ROOT)


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch

    import bench
    import workloads as W
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cases = W.batch(64, seed=7)
        mine = W.shard(cases, rank, world)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        cost = sum(W.case_cost(cases[i]) for i in mine)
        costs = [None] * world
        dist.all_gather_object(costs, cost)
        t = bench.max_over_ranks(10.0 + 5.0 * rank, dist)  # this rank's "device time" in ms
        v = bench.aggregate(1000, 4, world, t)
        if rank == 0:
            q.put((gathered, costs, t, v))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_shards_and_timing():
    world, port = 2, 29511
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    mp.start_processes(_worker, args=(world, port, q), nprocs=world, join=True, start_method="spawn")
    gathered, costs, t, v = q.get(timeout=30)
    allidx = sorted(i for g in gathered for i in g)
    assert allidx == list(range(64))                      # complete and disjoint
    assert max(costs) / min(costs) < 1.05                 # balanced within 5%
    assert t == 15.0                                      # slowest rank
    assert v == 1000 * 4 * 2 / 0.015

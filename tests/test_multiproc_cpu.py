"""Multi-process (replicas) host logic on CPU with gloo, world size 2.

bench.py runs one process per GPU; each serves its own share of the pairs or
of the serving trace with no data-path collective. The cross-rank steps are
the barrier, the max of the per-rank device times, the sums of operation
counts and the all-gather of free HBM budgets that shards the trace. These
tests run exactly those functions on gloo ranks.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dev = torch.device("cpu")
        # timing: every rank ends with the slowest rank's time
        t = bench.max_over_ranks(10.0 * (rank + 1), dist, dev)
        s = bench.sum_over_ranks(100 + rank, dist, dev)
        # sharding: budgets gathered from every rank, same owner list everywhere
        budgets = [None] * world
        dist.all_gather_object(budgets, (rank + 1) << 30)
        owner = bench.shard_requests(300, budgets)
        mine = [i for i, o in enumerate(owner) if o == rank]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        dist.barrier()
        q.put((rank, t, s, budgets, owner, gathered))
    finally:
        dist.destroy_process_group()


def test_replicas_reduce_and_shard():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    owners = [r[4] for r in results]
    assert owners[0] == owners[1]                      # every rank agrees on the shard map
    for rank, t, s, budgets, owner, gathered in results:
        assert t == 20.0                               # max over ranks
        assert s == 201.0                              # sum over ranks
        assert budgets == [1 << 30, 2 << 30]
        allmine = sorted(i for part in gathered for i in part)
        assert allmine == list(range(300))             # a partition of the trace
        assert abs(len(gathered[1]) - 2 * len(gathered[0])) <= 2   # weighted by budget


def test_shard_requests_single_rank_and_equal_weights():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.shard_requests(5, [7]) == [0] * 5
    own = bench.shard_requests(8, [1, 1, 1, 1])
    assert own == [0, 1, 2, 3, 0, 1, 2, 3]
    assert bench.max_over_ranks(3.5, None, None) == 3.5

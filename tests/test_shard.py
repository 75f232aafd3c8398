"""Sharding the batched workload over ranks: the partition (host logic) and the
gather of results over a real process group (gloo, world size 2, on CPU)."""
import os
import socket

import numpy as np
import pytest

from cvrp_aco_ocl_b200.shard import gather_results, instance_cost, partition, shard_of


def test_partition_covers_each_instance_once_and_balances():
    rng = np.random.default_rng(3)
    sizes = rng.integers(101, 1002, size=512)
    costs = [instance_cost(int(n), 128) for n in sizes]
    for world in (1, 2, 3, 8):
        parts = partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(512))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)  # LPT bound
        assert parts == partition(costs, world)       # every rank derives the same split


def test_partition_edge_cases():
    assert partition([], 2) == [[], []]
    assert partition([5.0], 3) == [[0], [], []]
    with pytest.raises(ValueError):
        partition([1.0], 0)
    assert shard_of([10, 10, 10, 10], 1, 2, 0) == [0, 2] and shard_of([10, 10, 10, 10], 1, 2, 1) == [1, 3]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, sizes, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shard_of(sizes, 128, world, rank)
        # a stand-in solve per instance: length and tour derived from the index
        local = {i: (1000.0 + i, [0, i + 1, 0]) for i in mine}
        merged = gather_results(local)
        t = torch.tensor([float(rank + 1)], dtype=torch.float64)  # per-rank device time stand-in
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            q.put((merged, float(t.item()), mine))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_gather_over_gloo_two_ranks():
    import torch.multiprocessing as mp
    sizes = [101, 900, 450, 120, 1000, 300, 777]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    merged, tmax, mine0 = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert sorted(merged) == list(range(len(sizes)))
    assert all(merged[i] == (1000.0 + i, [0, i + 1, 0]) for i in merged)
    assert tmax == 2.0
    assert mine0 == shard_of(sizes, 128, 2, 0)

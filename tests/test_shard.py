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


def _balance_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from cvrp_aco_ocl_b200 import instances as I
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # the headline workload at two GPUs: 512 instances per rank, 100-1000 customers
        sizes = [x.n for x in I.gen_batch(512, 512 * world, 100, 1000)]
        mine = shard_of(sizes, 128, world, rank)
        load = torch.tensor([sum(instance_cost(sizes[i], 128) for i in mine), float(len(mine))], dtype=torch.float64)
        loads = [torch.zeros(2, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(loads, load)
        if rank == 0:
            q.put([tuple(x.tolist()) for x in loads])
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_batch_partition_balances_predicted_cost_over_gloo():
    """Both ranks derive the same split of the 1024-instance batch; the
    predicted iteration times of their shards agree within 5%."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_balance_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    loads = q.get(timeout=180)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    costs = [c for c, _ in loads]
    assert sum(n for _, n in loads) == 1024
    assert max(costs) / min(costs) <= 1.05


def test_cost_model_grows_with_size_and_ants():
    assert instance_cost(1001, 128) > instance_cost(501, 128) > instance_cost(101, 128) > 0
    assert instance_cost(501, 256) > instance_cost(501, 128)
    # the row pass term alone: 16 bytes per element over the bandwidth
    m = {"a_ns": 0.0, "b_ns": 0.0, "bw_bytes_per_ns": 16.0}
    assert instance_cost(100, 128, m) == 100.0 * 100.0

"""Sharding a batch of independent instances over ranks (one process per GPU).

Instances do not interact, so there is no collective on the data path: every
rank solves its shard in its own batch, and only the results (best lengths
and tours) travel, once, to rank 0 at the end.  The partition balances the
predicted device time of one iteration by longest-processing-time-first
assignment; ties go to the lower rank so every rank computes the same
partition without talking.

Cost model (nanoseconds per iteration of one instance of n nodes and A ants,
throughput mode with 2-opt, batched):

    A * n * (a + b * n)  +  16 * n^2 / bw

The first term is the construct and the 2-opt: every ant makes about n steps
and improves about n / route-length routes, a constant cost per node, plus the
full-row scan of the steps whose listed candidates are all taken, which grows
with n.  The second is the pheromone pass, 16 bytes of HBM traffic per matrix
element.  ``fit`` measures a, b and bw on the current GPU from batches of one
size each (``python -m cvrp_aco_ocl_b200.shard fit``); COST_MODEL holds the
values measured on a B200.
"""
from __future__ import annotations

import heapq
import json
import sys
from typing import Dict, List, Optional, Sequence, Tuple

# a, b: ns per ant and node, ns per ant and node^2; bw: bytes per ns of the pheromone pass
# (measured on a B200 by fit(): batches of 101..1001 nodes, 128 ants, 25-NN lists)
COST_MODEL = {"a_ns": 0.4181, "b_ns": 0.000172, "bw_bytes_per_ns": 4544.0}


def instance_cost(n: int, ants: int, model: Optional[Dict[str, float]] = None) -> float:
    """Predicted device time (ns) of one batched iteration of an instance."""
    m = model or COST_MODEL
    return float(ants) * float(n) * (m["a_ns"] + m["b_ns"] * float(n)) + 16.0 * float(n) * float(n) / m["bw_bytes_per_ns"]


def partition(costs: Sequence[float], world: int) -> List[List[int]]:
    """Instance indices per rank (each list ascending), LPT over `costs`."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    shards: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(s) for s in shards]


def shard_of(sizes: Sequence[int], ants: int, world: int, rank: int) -> List[int]:
    return partition([instance_cost(n, ants) for n in sizes], world)[rank]


def gather_results(local: Dict[int, Tuple[float, Sequence[int]]], group=None) -> Optional[Dict[int, Tuple[float, list]]]:
    """Collect {instance index: (best length, best tour)} from every rank on
    rank 0 (None elsewhere).  Uses torch.distributed object collectives, so it
    runs over gloo on CPU as well as over NCCL."""
    import torch.distributed as dist

    if not dist.is_initialized():
        return {k: (float(v[0]), list(v[1])) for k, v in local.items()}
    payload = {int(k): (float(v[0]), [int(x) for x in v[1]]) for k, v in local.items()}
    out = [None] * dist.get_world_size(group) if dist.get_rank(group) == 0 else None
    dist.gather_object(payload, out, dst=0, group=group)
    if dist.get_rank(group) != 0:
        return None
    merged: Dict[int, Tuple[float, list]] = {}
    for part in out:
        for k, v in part.items():
            if k in merged:
                raise RuntimeError(f"instance {k} solved on two ranks")
            merged[k] = v
    return merged


def fit(sizes: Sequence[int] = (101, 251, 401, 601, 801, 1001), ant_nodes: float = 8.2e6, ants: int = 128,
        nn: int = 25, iters: int = 4, device: int = 0) -> Dict[str, float]:
    """Measure the cost model on this GPU: for every size, a batch of
    instances of that size (mixed and large generators alternately), as many
    as make `ant_nodes` ants x nodes (the work of the 512-instance batch, so
    that every size fills the GPU), `iters` iterations timed phase by phase
    after 3 warm-up iterations; a and b by least squares of (construct + 2-opt)
    / (A n) against n, bw from the pheromone pass's bytes over its time."""
    import numpy as np

    from . import instances as I
    from ._lib import MODE_THROUGHPUT
    from .aco import Batch, Problem, default_params

    rows = []
    for n in sizes:
        count = max(16, int(round(ant_nodes / (ants * n))))
        insts = [I.gen_mixed(7000 + 31 * n + k, n - 1) if k % 2 == 0 else I.gen_large(7000 + 31 * n + k, n - 1)
                 for k in range(count)]
        p = default_params(n)
        p.mode, p.n_ants, p.nn_ants, p.nn_ls, p.device = MODE_THROUGHPUT, ants, min(nn, n - 2), min(nn, n - 2), device
        p.seed_time, p.rnd_seed = 1796300000, 4242
        with Batch([Problem.from_instance(x) for x in insts], p) as B:
            B.init()
            B.iterate(3)
            ms = B.time_phases(iters) / iters
        per_inst_ns = (float(ms[0]) + float(ms[1]) + float(ms[2])) * 1e6 / count
        rows.append((n, per_inst_ns / (ants * n), float(ms[3]) * 1e6, 16.0 * n * n * count))
    ns = np.array([r[0] for r in rows], float)
    y = np.array([r[1] for r in rows], float)  # ns per ant-node
    b, a = np.polyfit(ns, y, 1)
    bw = float(sum(r[3] for r in rows) / sum(r[2] for r in rows))
    return {"a_ns": float(a), "b_ns": float(b), "bw_bytes_per_ns": bw,
            "points": [{"n": r[0], "ns_per_ant_node": r[1], "rows_ns": r[2]} for r in rows]}


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "fit":
        print(json.dumps(fit(), indent=1))
    else:
        print(__doc__)

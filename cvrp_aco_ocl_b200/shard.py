"""Sharding a batch of independent instances over ranks (one process per GPU).

Instances do not interact, so there is no collective on the data path: every
rank solves its shard in its own batch, and only the results (best lengths
and tours) travel, once, to rank 0 at the end.  The partition balances the
estimated cost per iteration, A * n^2 (construct, 2-opt and the pheromone
pass all grow with it), by longest-processing-time-first assignment; ties go
to the lower rank so every rank computes the same partition without talking.
"""
from __future__ import annotations

import heapq
from typing import Dict, List, Optional, Sequence, Tuple


def instance_cost(n: int, ants: int) -> float:
    return float(ants) * float(n) * float(n)


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

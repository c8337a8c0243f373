"""Multi-GPU placement of batched filters (one process per GPU).

Batched filters are independent, so a batch shards by filter with no
collective on the data path: filters are assigned to ranks by LPT (longest
processing time first) on a cost proportional to N_b * T, each rank runs its
shard on its own GPU, and the per-filter results are gathered once at the
end. The plain single filter does not shard (its resampling prefix is
global); several GPUs run independent replicas of it.
"""
from __future__ import annotations

import heapq
from typing import List, Sequence


def lpt_partition(costs: Sequence[float], world: int) -> List[List[int]]:
    """Greedy LPT: items in decreasing cost go to the currently lightest rank.

    Deterministic (ties broken by rank, then by item index), so every rank
    computes the same partition without communicating.
    """
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    for p in parts:
        p.sort()
    return parts


def shard(filters: Sequence[dict], rank: int, world: int):
    """(global indices, filter dicts) of this rank's shard, balanced on N."""
    parts = lpt_partition([f["n_particles"] for f in filters], world)
    idx = parts[rank]
    return idx, [filters[i] for i in idx]


def gather_results(local_idx: Sequence[int], local_vals: Sequence[float], n_total: int, group=None):
    """All-gather per-filter results of every rank into one list of length n_total."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    objs = [None] * world
    dist.all_gather_object(objs, (list(local_idx), [float(v) for v in local_vals]), group=group)
    out = [float("nan")] * n_total
    for idx, vals in objs:
        for i, v in zip(idx, vals):
            out[i] = v
    return out

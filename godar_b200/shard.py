"""Ensemble sharding across GPUs (one process per GPU).

Independent floe fields need no exchange, so a multi-GPU run partitions the
fields across ranks and runs each rank's share as one batch; the only
collectives are a barrier and a max over ranks of the device time.  The
partition is longest-processing-time greedy on floe counts (the step cost is
about linear in floes), deterministic for a given list of sizes.
"""
from __future__ import annotations

import heapq


def lpt_partition(sizes, nranks: int):
    """Returns nranks lists of indices into sizes, balanced by total size."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    heap = [(0, r) for r in range(nranks)]
    parts = [[] for _ in range(nranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + int(sizes[i]), r))
    for p in parts:
        p.sort()
    return parts


def rank_share(sizes, rank: int, nranks: int):
    return lpt_partition(sizes, nranks)[rank]


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Max of a per-rank timing over all ranks (identity without a process
    group)."""
    if dist is None or not dist.is_initialized():
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())

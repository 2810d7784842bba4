"""Partition of independent graphs across ranks (one process per GPU).

Batched serving and multi-graph workloads shard by graph: every rank solves
its own graphs with no per-sweep exchange, and only results are gathered.
Graphs are dealt largest first to the rank with the least work so far
(longest-processing-time order), which keeps the slowest rank within one
graph of the mean. The partition is a pure function of the weights, so every
rank computes the same one without communicating.
"""

from __future__ import annotations

import heapq
from typing import List, Sequence


def partition(weights: Sequence[float], world: int) -> List[List[int]]:
    """Indices of the graphs of each rank; each list in increasing order."""
    if world < 1:
        raise ValueError("world size must be positive")
    order = sorted(range(len(weights)), key=lambda i: (-float(weights[i]), i))
    heap = [(0.0, r) for r in range(world)]
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(weights[i]), r))
    return [sorted(x) for x in out]


def gather_results(local: dict, world: int) -> dict:
    """Union of every rank's {graph index: result} (torch.distributed, any backend)."""
    if world == 1:
        return dict(local)
    import torch.distributed as dist

    parts = [None] * world
    dist.all_gather_object(parts, local)
    out = {}
    for p in parts:
        out.update(p)
    return out

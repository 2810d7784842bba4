"""Partition of independent graphs across ranks (one process per GPU).

Batched serving and multi-graph workloads shard by graph: every rank solves
its own graphs with no per-sweep exchange, and only results are gathered.
Graphs are dealt largest first to the rank with the least work so far
(longest-processing-time order), which keeps the slowest rank within one
graph of the mean. The partition is a pure function of the weights, so every
rank computes the same one without communicating.

When graphs share parameters (the same analysis rules instantiated in many
graphs, each with its own evidence and labels), learning needs one exchange
per step: every rank sums the adjoint's per-factor gradients of its graphs
into the shared rules, and one all-reduce sums them over the ranks
(shared_gradient); the updated rule probabilities go back to every factor
that instantiates them (expand_shared).
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


def shared_gradient(grad_p, rule_of_factor, n_rules: int, world: int = 1):
    """dL/d(shared rule probabilities), summed over every rank's graphs.

    grad_p: per-factor dL/dp of this rank's graphs (float64 tensor, e.g. the
    adjoint's output for a BatchEngine); rule_of_factor: the rule each
    factor instantiates, -1 for a factor with a parameter of its own (int64
    tensor on the same device). Returns a float64 tensor of n_rules entries,
    the same on every rank: one all-reduce (sum) over the process group, on
    NCCL for CUDA tensors and gloo for CPU ones."""
    import torch

    if grad_p.shape != rule_of_factor.shape:
        raise ValueError("grad_p and rule_of_factor must have one entry per factor")
    # An index outside [-1, n_rules) would make index_add_ raise a device-side
    # assert on a CUDA tensor, which poisons the CUDA context: check first.
    if rule_of_factor.numel() and (int(rule_of_factor.min()) < -1 or int(rule_of_factor.max()) >= int(n_rules)):
        raise ValueError("rule_of_factor entries must lie in [-1, n_rules)")
    g = torch.zeros(int(n_rules), dtype=torch.float64, device=grad_p.device)
    m = rule_of_factor >= 0
    g.index_add_(0, rule_of_factor[m], grad_p[m].to(torch.float64))
    if world > 1:
        import torch.distributed as dist

        dist.all_reduce(g, op=dist.ReduceOp.SUM)
    return g


def expand_shared(p_rules, rule_of_factor, p_factor):
    """Per-factor probabilities after a learning step: the shared rule's value
    where a factor instantiates one, the factor's own elsewhere."""
    if rule_of_factor.numel() and (int(rule_of_factor.min()) < -1 or int(rule_of_factor.max()) >= p_rules.shape[0]):
        raise ValueError("rule_of_factor entries must lie in [-1, number of rules)")
    out = p_factor.clone()
    m = rule_of_factor >= 0
    out[m] = p_rules[rule_of_factor[m]].to(out.dtype)
    return out

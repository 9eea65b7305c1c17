"""Instances across GPUs: one process per GPU, each relaxes its own share of the gridshells.

The DR loop has no exchange between instances (each instance is independent, as in the reference's batches:
web/js/solver_gpu.js:1-2), so there is no collective on the data path: a rank takes a weighted share of the instances,
relaxes them on its GPU, and the results are gathered on the host.  A single instance is not split ("replicas only").
"""
from __future__ import annotations

import heapq


def instance_weight(model) -> int:
    """work and device memory of one instance grow with its node, segment and crossing counts"""
    return int(model.n + model.m + 2 * model.K)


def greedy_split(weights, world):
    """largest first onto the lightest rank (LPT): every instance on exactly one rank; returns per-rank index lists"""
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    heap = [(0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + weights[i], r))
    return [sorted(x) for x in out]


def shard_for(rank, world, models):
    """the instance indices of `rank` (the same answer on every rank: deterministic, no communication needed)"""
    return greedy_split([instance_weight(m) for m in models], world)[rank]

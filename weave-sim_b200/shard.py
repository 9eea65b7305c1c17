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


def relax_sharded(models, relax, rank, world, group=None):
    """every rank relaxes its share of `models` with `relax(list of models) -> list of results` (one per model, any
    picklable value) and rank 0 gathers them; returns, on rank 0, the results in the order of `models` (None elsewhere).
    The only communication is the host-side gather after the relaxation (torch.distributed.gather_object over the
    process group: gloo on the host, or the NCCL group of the GPU ranks)."""
    import torch.distributed as dist
    mine = shard_for(rank, world, models)
    res = relax([models[i] for i in mine])
    if len(res) != len(mine):
        raise ValueError("relax_sharded: one result per model expected")
    if world == 1:
        return list(res)
    box = [None] * world if rank == 0 else None
    dist.gather_object(list(zip(mine, res)), box, dst=0, group=group)
    if rank != 0:
        return None
    out = [None] * len(models)
    for part in box:
        for i, r in part:
            if out[i] is not None:
                raise RuntimeError(f"relax_sharded: instance {i} came back from two ranks")
            out[i] = r
    if any(r is None for r in out):
        raise RuntimeError("relax_sharded: an instance came back from no rank")
    return out

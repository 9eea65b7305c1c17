"""Instances sharded across ranks (world size 2, gloo on CPU): every instance on exactly one rank, weights balanced,
the shard is the same whichever rank computes it, and a sharded relaxation (each rank relaxes its share, rank 0
gathers) gives every instance the result it has when relaxed alone."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import torch
    import weavesim_b200 as ws
    from weavesim_b200 import shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    models = ws.configs.batch_mixed(12, seed=3)
    mine = shard.shard_for(rank, world, models)
    # what every rank thinks the split is must agree; gather the shards and the weights
    t = torch.zeros(len(models), dtype=torch.int64)
    t[mine] = rank + 1
    allv = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(allv, t)
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        q.put((sum(allv).tolist(), [shard.instance_weight(m) for m in models], mine))


@pytest.mark.timeout(300)
def test_shards_cover_every_instance_once():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    owners, weights, mine0 = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # each instance owned by exactly one rank (owner ids 1 or 2, no sums of both, no zeros)
    assert all(o in (1, 2) for o in owners)
    loads = [sum(w for w, o in zip(weights, owners) if o == r) for r in (1, 2)]
    assert max(loads) - min(loads) <= max(weights)


def test_greedy_split_is_balanced():
    from weavesim_b200.shard import greedy_split
    w = [5, 9, 1, 7, 3, 3, 8, 2]
    parts = greedy_split(w, 3)
    assert sorted(i for p in parts for i in p) == list(range(8))
    loads = [sum(w[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(w)


def _relax_oracle(models, iters=60):
    """relaxes each model with the oracle on the host (the CPU stand-in for a rank's GPU) and keeps what a caller reads"""
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "oracle"))
    from oracle import Oracle
    out = []
    for m in models:
        o = Oracle(m.copy())
        o.step(iters)
        v = o.view()
        out.append({"X": v["X"].copy(), "u": v["u"].copy(), "iteration": v["iteration"], "n": m.n})
    return out


def _sharded_worker(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import weavesim_b200 as ws
    from weavesim_b200 import shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    models = ws.configs.batch_mixed(6, seed=5, max_nodes=1500)
    got = shard.relax_sharded(models, _relax_oracle, rank, world)
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        q.put(got)
    else:
        assert got is None


@pytest.mark.timeout(300)
def test_sharded_relaxation_gathers_every_result():
    import numpy as np
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import weavesim_b200 as ws
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sharded_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    alone = _relax_oracle(ws.configs.batch_mixed(6, seed=5, max_nodes=1500))
    assert len(got) == len(alone) == 6
    for g, a in zip(got, alone):
        assert g["n"] == a["n"] and g["iteration"] == a["iteration"] == 60
        assert np.array_equal(g["X"], a["X"]) and np.array_equal(g["u"], a["u"])

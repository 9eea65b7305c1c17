"""Serving loop (weave-sim_b200/serve.py): request generation on the host, and on the GPU continuous batching with
each result equal alone and in the mix."""
import numpy as np
import pytest

import weavesim_b200 as ws
from weavesim_b200 import serve


def test_variant_changes_only_what_it_should():
    md = ws.configs.dome_stiff(seed=11)
    eq = {"X": md.X + 0.01, "Q": md.Q.copy(), "u": md.cross_u + 0.1, "nprev": md.cross_nprev.copy()}
    rng = np.random.default_rng(0)
    v = serve.variant_of(md, eq, rng)
    f = v.EA / md.EA
    assert np.allclose(f, f[0]) and 0.95 <= f[0] <= 1.05
    d = v.cross_mu - md.cross_mu
    assert np.all(np.abs(d - d[0]) < 1e-12) or np.all(v.cross_mu >= 0)
    assert np.array_equal(v.X, eq["X"]) and np.array_equal(v.cross_u, eq["u"])
    s0 = md.X.reshape(-1, 3)[md.anchor_node]
    r = (v.anchor_target.reshape(-1, 3) - s0) / np.where(np.abs(md.anchor_target.reshape(-1, 3) - s0) > 0,
                                                        md.anchor_target.reshape(-1, 3) - s0, 1)
    moved = np.abs(md.anchor_target.reshape(-1, 3) - s0) > 1e-9
    assert np.all(np.abs(r[moved] - r[moved][0]) < 1e-9) and 0.98 <= r[moved][0] <= 1.02
    assert v.params["warmup_iter"] == 0 and v.params["ramp_iter"] == 0


def test_poisson_stream_shape():
    reqs = serve.poisson_stream(200.0, 50, seed=1)
    gaps = np.diff([r.arrival for r in reqs])
    assert np.all(gaps > 0) and 0.002 < gaps.mean() < 0.01
    assert all(r.kind == "fresh" and r.model.n == 1176 for r in reqs)


@pytest.mark.gpu
def test_results_equal_alone_and_in_the_mix():
    if ws.device_count() < 1:
        pytest.skip("no CUDA device")
    tpl = ws.configs.dome_stiff(seed=1)
    srv = serve.Server(tpl, slots=8, chunk=200)
    reqs = serve.poisson_stream(400.0, 12, seed=3, fresh_cap=800)
    done = srv.run(reqs, time_limit=60)
    assert len(done) == 12
    warm = list(srv.resident.values())[:2]
    vreqs = serve.poisson_stream(400.0, 6, seed=4, variant_share=1.0, variant_cap=400, warm_bank=warm)
    for r in vreqs:
        r.rid += 100
    t0 = done[-1].done
    for r in vreqs:
        r.arrival += t0
    done2 = srv.run(vreqs, time_limit=60)
    srv.dispose()
    assert sum(r.kind == "variant" for r in done2) == 6
    for r in (done[0], done[5], done2[-1]):
        s = ws.GpuSolver([r.model], precision="mixed", threads=256)
        s.step(r.iters)
        alone = s.download(0)
        s.dispose()
        assert np.array_equal(alone["X"], r.result["X"]) and np.array_equal(alone["u"], r.result["u"])


def test_topology_key_separates_what_a_slot_cannot_take():
    """requests share a pool only when ws_load_instance would accept one in the other's slot: same node, segment, joint,
    crossing, strand and clamp counts; parameter variants keep their base's key"""
    a, b = ws.configs.dome_stiff(seed=1), ws.configs.dome_stiff(seed=2)
    assert serve.topology_key(a) == serve.topology_key(b)
    small = ws.configs.dome_small(seed=1, side=3)
    assert serve.topology_key(small) != serve.topology_key(a)
    eq = {"X": a.X.copy(), "Q": a.Q.copy(), "u": a.cross_u.copy(), "nprev": a.cross_nprev.copy()}
    assert serve.topology_key(serve.variant_of(a, eq, np.random.default_rng(0))) == serve.topology_key(a)
    import cases
    one = cases.straight(1000.0, 10, anchors=[((0, 0), ws.mask(1, 1, 1, 1, 1, 1))])
    two = cases.straight(1000.0, 10, anchors=[((0, 0), ws.mask(1, 1, 1, 1, 1, 1)), ((0, 1), ws.mask(1, 1, 1, 1, 1, 1))])
    pin = cases.straight(1000.0, 10, anchors=[((0, 0), ws.mask(1, 1, 1, 1, 1, 1)), ((0, 1), ws.mask(1, 1, 1, 0, 0, 0))])
    assert serve.topology_key(one)[-1] == 1 and serve.topology_key(two)[-1] == 2 and serve.topology_key(pin)[-1] == 1


@pytest.mark.gpu
def test_mixed_topologies_served_from_their_pools():
    """requests of two topologies in one stream: each gets a pool of its own within the budget, every request is
    served, and each result is the same bits as the same model relaxed alone"""
    if ws.device_count() < 1:
        pytest.skip("no CUDA device")
    tpl = ws.configs.dome_stiff(seed=1)
    srv = serve.Server(tpl, slots=4, chunk=200)
    reqs = serve.poisson_stream(400.0, 6, seed=3, fresh_cap=600)
    small = [ws.configs.dome_small(seed=20 + i, side=3) for i in range(4)]
    for i, md in enumerate(small):
        md.params = dict(md.params, max_iter=600)
        reqs.append(serve.Request(100 + i, reqs[i].arrival + 1e-4, md, "fresh", 600))
    done = srv.run(reqs, time_limit=60)
    assert len(srv.pools) == 2 and srv.slots == 8
    assert len(done) == 10
    srv.dispose()
    for r in done:
        s = ws.GpuSolver([r.model], precision="mixed", threads=256)
        s.step(r.iters)
        alone = s.download(0)
        s.dispose()
        assert np.array_equal(alone["X"], r.result["X"]) and np.array_equal(alone["u"], r.result["u"]), r.rid

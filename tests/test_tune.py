"""The autotuner: its candidate shapes, size buckets and cache on the host (no GPU), and on a B200 the tuned context
against the oracle and the cache taking over for the next batch of the same bucket."""
import os
import subprocess
import sys

import numpy as np
import pytest

import weavesim_b200 as ws
from weavesim_b200 import solver

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_batched_candidates_cover_block_sizes_and_state():
    models = [ws.configs.dome_small(seed=s) for s in (1, 2)]
    c1 = solver.tune_candidates(models, "mixed", "cta")
    assert {(c["threads"], c["cta_state"]) for c in c1} == {(t, s) for t in (128, 256, 512) for s in (0, 1)}
    assert all(c["wide_cluster"] == 1 for c in c1)
    # stage 2 needs an instance at or above a threshold: the 3 m dome (2,328 nodes + segments) reaches none of them
    assert solver.tune_candidates(models, "mixed", "cta", after=c1[0]) == []


def test_wide_candidates_only_for_large_instances():
    big = ws.configs.dome_small(side=12)             # ~21k nodes + segments
    assert 16384 <= big.n + big.m < 32768
    best1 = {"threads": 512, "cta_state": 1, "wide_cluster": 1, "wide_min": 0, "plain_launch": 0}
    c2 = solver.tune_candidates([big], "f64", "cta", after=best1)
    assert {(c["wide_cluster"], c["wide_min"]) for c in c2} == {(cl, w) for cl in (2, 4, 8) for w in (16384, 8192)}
    assert all(c["threads"] == 512 and c["cta_state"] == 1 for c in c2)


def test_plain_candidates_are_the_launch_modes():
    c = solver.tune_candidates([ws.configs.dome_small()], "mixed", "plain")
    assert sorted(x["plain_launch"] for x in c) == [0, 1, 2]


def test_size_buckets():
    a = solver.tune_key([ws.configs.dome_small(seed=1)], "mixed", "cta", device="B200")
    b = solver.tune_key([ws.configs.dome_small(seed=7)], "mixed", "cta", device="B200")
    c = solver.tune_key([ws.configs.dome_small(seed=1)] * 40, "mixed", "cta", device="B200")
    d = solver.tune_key([ws.configs.dome_small(seed=1)], "f64", "cta", device="B200")
    e = solver.tune_key([ws.configs.dome_small(seed=1)], "mixed", "cta", device="H100")
    assert a == b                                    # same sizes, another seed: the same bucket
    assert len({a, c, d, e}) == 4 and " " not in a


def test_cache_put_get_clear():
    solver.tune_cache_clear()
    key = "testdev|f0|p1|s1|e0|b0|x22|t22"
    assert solver.tune_cache_get(key) is None
    shape = {"threads": 512, "cta_state": 1, "wide_cluster": 4, "wide_min": 16384, "plain_launch": 0, "trials": 7,
             "trial_ms": 1.5, "default_ms": 2.0}
    solver.tune_cache_put(key, shape)
    got = solver.tune_cache_get(key)
    assert {k: got[k] for k in shape} == shape
    solver.tune_cache_clear()
    assert solver.tune_cache_get(key) is None
    with pytest.raises(RuntimeError):
        solver.tune_cache_put("two words", shape)


def test_cache_file_persists_across_processes(tmp_path):
    path = tmp_path / "tune.txt"
    env = dict(os.environ, WEAVESIM_TUNE_CACHE=str(path))
    put = ("import sys; sys.path.insert(0, %r); from weavesim_b200 import solver; "
           "solver.tune_cache_put('k|1', dict(threads=256, cta_state=0, wide_cluster=2, wide_min=32768, plain_launch=0, "
           "trials=3, trial_ms=9.0, default_ms=10.0))" % ROOT)
    subprocess.run([sys.executable, "-c", put], env=env, check=True)
    assert "k|1 256 0 2 32768 0 3 9 10" in path.read_text()
    get = ("import sys; sys.path.insert(0, %r); from weavesim_b200 import solver; "
           "print(solver.tune_cache_get('k|1')['wide_cluster'])" % ROOT)
    out = subprocess.run([sys.executable, "-c", get], env=env, check=True, capture_output=True, text=True).stdout
    assert out.strip() == "2"


# ------------------------------------------------------------------------------------------------ on the GPU
@pytest.mark.gpu
def test_tuned_batch_matches_oracle_and_is_cached(oracle_mod):
    """a tuned uneven batch (one instance above the smallest wide threshold): the tuner times its candidates, the context
    starts from the models' state afterwards, FP64 gives the oracle's results, and a second batch of the same bucket
    takes the shape from the cache"""
    if ws.device_count() < 1:
        pytest.skip("no CUDA device")
    solver.tune_cache_clear()
    models = [ws.configs.dome_small(side=10, seed=3), ws.configs.dome_small(seed=4), ws.configs.dome_stiff(seed=5, side=3)]
    assert models[0].n + models[0].m >= 8192
    s = ws.GpuSolver([m.copy() for m in models], precision="f64", tune=True)
    sh = s.shape
    assert sh["source"] == "tuned" and sh["trials"] >= 3 and sh["trial_ms"] <= sh["default_ms"] * 1.0001
    assert s.read_control()[0]["iter"] == 0
    ctl = s.step(400)
    for b, m in enumerate(models):
        v = oracle_mod.Oracle(m.copy())
        v.step(400)
        ref = v.view()
        g = s.download(b, fields=("X", "u", "stuck"))
        assert ctl[b]["iter"] == 400 and ctl[b]["rollbacks"] == ref["rollbacks"], b
        assert np.linalg.norm((g["X"] - ref["X"]).reshape(-1, 3), axis=1).max() / m.span < 1e-9, b
        assert np.array_equal(g["stuck"], ref["stuck"]), b
    s.dispose()
    again = ws.GpuSolver([ws.configs.dome_small(side=10, seed=8), ws.configs.dome_small(seed=9),
                          ws.configs.dome_stiff(seed=10, side=3)], precision="f64", tune=True)
    sh2 = again.shape
    again.dispose()
    assert sh2["source"] == "cache"
    assert {k: sh2[k] for k in ("threads", "cta_state", "wide_cluster", "wide_min")} == \
           {k: sh[k] for k in ("threads", "cta_state", "wide_cluster", "wide_min")}


@pytest.mark.gpu
def test_tuned_plain_form_matches_oracle(oracle_mod):
    if ws.device_count() < 1:
        pytest.skip("no CUDA device")
    solver.tune_cache_clear()
    md = ws.configs.dome_small()
    s = ws.GpuSolver([md.copy()], precision="f64", form="plain", tune=True)
    assert s.shape["source"] == "tuned" and s.shape["plain_launch"] in (0, 1, 2)
    ctl = s.step(400)[0]
    g = s.download(0, fields=("X",))
    s.dispose()
    v = oracle_mod.Oracle(md.copy())
    v.step(400)
    ref = v.view()
    assert ctl["iter"] == 400 and ctl["rollbacks"] == ref["rollbacks"]
    assert np.linalg.norm((g["X"] - ref["X"]).reshape(-1, 3), axis=1).max() / md.span < 1e-9

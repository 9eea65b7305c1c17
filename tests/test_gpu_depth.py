"""CUDA path against the f64 oracle at the depth the benchmarks run (needs a B200: run with -m gpu).

The benchmarked configurations, each checked past the 300-iteration warm-up that holds every node
(web/js/solver_cpu.js:775-776) and into the contact ramp (1500 iterations) and the support motion:

* the 20 m shell (the headline workload, timed from iteration 600 on): FP64 in the plain and grid forms with the
  oracle's iteration and roll-back counts and within 1e-9 of the span, slide coordinates within 1e-6 segments, the
  same stick/slip states, at 330, 1000, 2000 and 3000 iterations; at 5000 and 8000, where the trajectory's chaos has
  set in (the oracle started 1e-9 of the span away departs from itself by ~3e-5 of the span), the oracle's roll-back
  count and a distance from the oracle within the oracle's own spread; the mixed policy (FP32 element math,
  two-float state, FP64 reductions) within the 1e-4 span gate at every horizon where that spread is below it;
* the stiff dome (25 x 3 mm laths, E 12 GPa, per-crossing mu ~ U(0.1, 0.5)): FP64 exact to 1500 iterations in the
  batched and plain forms; a population of them in FP64, mixed and naive FP32 against the oracle at 500 to 3000
  iterations, the mixed policy within the gate, naive FP32 reported;
* a sample of the uneven 512-gridshell batch (the largest instance and seven others across the size range) in one
  batched launch with global state, FP64 against one oracle per instance for 1000 iterations.

Every comparison also writes its raw numbers through cases.record (WEAVESIM_PARITY_RECORD).  The reference's own
GPU-vs-CPU bands are in web/README.md:77-85 and web/tests/gpu_parity.html:21-37.
"""
import threading

import numpy as np
import pytest

import cases
import weavesim_b200 as ws

pytestmark = pytest.mark.gpu

HORIZONS = (330, 1000, 2000, 3000, 5000, 8000)
EXACT = 3000                # FP64 is held to the oracle's bits (to rounding) up to here, to its chaos floor beyond
GATE = 1e-4                 # max node distance / span, the acceptance gate of the mixed policy
# FP64 against the oracle at depth: positions within 1e-9 of the span; slide coordinates (in segments) within 1e-6.  The
# slides are where the trajectory's chaos shows first: on the shell the oracle started 1e-9 of the span away differs
# from itself by 5e-6 segments at 330 iterations and 6e-3 at 2000, while FP64 on the device (another summation order)
# differs from the oracle by 2e-13 and 3e-8 (4e-7 at 3000).
SLIDE_F64 = 1e-6


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if ws.device_count() < 1:
        pytest.skip("no CUDA device")


def _snap(o):
    v = o.view()
    return {k: v[k] for k in ("X", "u", "stuck", "iteration", "rollbacks")}


def _oracle_horizons(oracle_mod, model, horizons, dst):
    o = oracle_mod.Oracle(model)
    done = 0
    for h in horizons:
        o.step(h - done)
        done = h
        dst[h] = _snap(o)


def _parallel(jobs):
    """oracle runs side by side on host threads (the oracle's library releases the GIL)"""
    th = [threading.Thread(target=f, args=a) for f, a in jobs]
    for t in th:
        t.start()
    for t in th:
        t.join()


def _perturbed(md, scale, seed=11):
    p = md.copy()
    p.X = p.X + scale * md.span * np.random.default_rng(seed).standard_normal(p.X.shape)
    return p


def _diff(g, v, md):
    return {"pos_span": cases.max_node_err_span(g["X"], v["X"], md.span),
            "slide": float(np.abs(g["u"] - v["u"]).max()) if md.K else 0.0,
            "stuck_mismatch": int(np.sum(np.asarray(g["stuck"]) != np.asarray(v["stuck"])))}


# ------------------------------------------------------------------------------------------------ the 20 m shell
@pytest.fixture(scope="module")
def shell(oracle_mod):
    md = ws.configs.shell_large()
    ref, floor = {}, {}
    _parallel([(_oracle_horizons, (oracle_mod, md.copy(), HORIZONS, ref)),
               (_oracle_horizons, (oracle_mod, _perturbed(md, 1e-9), HORIZONS, floor))])
    return md, ref, {h: _diff(floor[h], ref[h], md) for h in HORIZONS}


def _gpu_horizons(md, prec, form, horizons):
    s = ws.GpuSolver([md.copy()], precision=prec, form=form)
    out, done = {}, 0
    for h in horizons:
        ctl = s.step(h - done)[0]
        done = h
        out[h] = dict(s.download(0, fields=("X", "u", "stuck")), iteration=ctl["iter"], rollbacks=ctl["rollbacks"])
    s.dispose()
    return out


@pytest.mark.parametrize("form", ["plain", "grid"])
def test_shell_f64_matches_oracle_at_depth(shell, form):
    md, ref, floor = shell
    got = _gpu_horizons(md, "f64", form, HORIZONS)
    rows = {h: dict(_diff(got[h], ref[h], md), rollbacks=got[h]["rollbacks"], oracle_rollbacks=ref[h]["rollbacks"],
                    chaos_floor=floor[h]) for h in HORIZONS}
    cases.record(f"shell_f64_{form}", {"horizons": rows})
    for h in HORIZONS:
        g, v, r, f = got[h], ref[h], rows[h], floor[h]
        assert g["iteration"] == v["iteration"] == h
        assert g["rollbacks"] == v["rollbacks"], h
        if h <= EXACT:
            assert r["pos_span"] < 1e-9, (h, r)
            assert r["slide"] < SLIDE_F64, (h, r)
            assert r["stuck_mismatch"] == 0, (h, r)
        else:
            # past the onset of chaos: no farther from the oracle than the oracle is from itself
            assert r["pos_span"] <= max(1e-9, f["pos_span"]), (h, r)
            assert r["slide"] <= max(SLIDE_F64, f["slide"]), (h, r)
            assert r["stuck_mismatch"] <= 2 * f["stuck_mismatch"] + max(1, md.K // 1000), (h, r)


@pytest.mark.parametrize("form", ["plain", "grid"])
def test_shell_mixed_within_gate_at_depth(shell, form):
    md, ref, floor = shell
    got = _gpu_horizons(md, "mixed", form, HORIZONS)
    rows = {h: dict(_diff(got[h], ref[h], md), chaos_floor=floor[h]) for h in HORIZONS}
    cases.record(f"shell_mixed_{form}", {"horizons": rows})
    for h in HORIZONS:
        assert got[h]["iteration"] == h
        if floor[h]["pos_span"] < GATE:
            assert rows[h]["pos_span"] <= GATE, (h, rows[h])
            # slides and stick/slip states agree up to the oracle's own spread at this horizon (the stick/slip set of
            # a chaotic trajectory is only defined to that spread)
            assert rows[h]["slide"] <= max(1e-2, 2 * floor[h]["slide"]), (h, rows[h])
            assert rows[h]["stuck_mismatch"] <= 2 * floor[h]["stuck_mismatch"] + max(1, md.K // 1000), (h, rows[h])


# ------------------------------------------------------------------------------------------------ the stiff dome
@pytest.mark.parametrize("form", ["cta", "plain"])
def test_stiff_dome_f64_matches_oracle(oracle_mod, form):
    md = ws.configs.dome_stiff()
    ref = {}
    _oracle_horizons(oracle_mod, md.copy(), (500, 1000, 1500), ref)
    got = _gpu_horizons(md, "f64", form, (500, 1000, 1500))
    rows = {h: dict(_diff(got[h], ref[h], md), rollbacks=got[h]["rollbacks"]) for h in ref}
    cases.record(f"stiff_dome_f64_{form}", {"horizons": rows})
    for h in ref:
        assert got[h]["iteration"] == ref[h]["iteration"] == h
        assert got[h]["rollbacks"] == ref[h]["rollbacks"], h
        assert rows[h]["pos_span"] < 1e-9 and rows[h]["slide"] < SLIDE_F64 and rows[h]["stuck_mismatch"] == 0, (h, rows[h])


def test_precision_policies_against_oracle(oracle_mod):
    """a population of stiff domes (the precision-stress configuration), each relaxed by the oracle, by the oracle started
    1e-9 of the span away (the chaos floor), and on the device in FP64, mixed and naive FP32 (batched form); at each
    horizon every device policy is compared with the oracle.  FP64 must hold 1e-9 of the span; the mixed policy the
    1e-4 gate on every instance whose chaos floor is below it; naive FP32 is reported, not held."""
    horizons = (500, 1000, 2000, 3000)
    models = [ws.configs.dome_stiff(seed=100 + b) for b in range(24)]
    ref = [dict() for _ in models]
    flo = [dict() for _ in models]
    jobs = [(_oracle_horizons, (oracle_mod, m.copy(), horizons, ref[b])) for b, m in enumerate(models)]
    jobs += [(_oracle_horizons, (oracle_mod, _perturbed(m, 1e-9, seed=b), horizons, flo[b])) for b, m in enumerate(models)]
    _parallel(jobs)
    runs = {p: ws.GpuSolver([m.copy() for m in models], precision=p, threads=512) for p in ("f64", "mixed", "f32")}
    table, done = [], 0
    for h in horizons:
        row = {"iteration": h}
        diffs = {}
        for p, s in runs.items():
            s.step(h - done)
            diffs[p] = [_diff(s.download(b, fields=("X", "u", "stuck")), ref[b][h], m) for b, m in enumerate(models)]
        diffs["chaos_floor"] = [_diff(flo[b][h], ref[b][h], m) for b, m in enumerate(models)]
        done = h
        for p, d in diffs.items():
            pos = np.array([x["pos_span"] for x in d])
            row[p] = {"pos_span_median": float(np.median(pos)), "pos_span_max": float(pos.max()),
                      "within_gate": int(np.sum(pos <= GATE)), "slide_max": float(max(x["slide"] for x in d)),
                      "stuck_mismatch_total": int(sum(x["stuck_mismatch"] for x in d))}
        table.append(row)
        for b in range(len(models)):
            assert diffs["f64"][b]["pos_span"] < 1e-9 and diffs["f64"][b]["stuck_mismatch"] == 0, (h, b, diffs["f64"][b])
            if diffs["chaos_floor"][b]["pos_span"] < GATE:
                assert diffs["mixed"][b]["pos_span"] <= GATE, (h, b, diffs["mixed"][b])
    for s in runs.values():
        s.dispose()
    cases.record("precision_policies_stiff_domes", {"instances": len(models), "crossings": models[0].K,
                                                     "horizons": table})


# ------------------------------------------------------------------------------------------------ the uneven batch
def _batch_sample():
    """the largest instance of the 512-gridshell batch and seven others spread over its size range"""
    models = ws.configs.batch_mixed(512, seed=4)
    order = sorted(range(len(models)), key=lambda b: -models[b].n)
    picks = [order[int(q * (len(order) - 1))] for q in (0.0, 0.02, 0.1, 0.25, 0.5, 0.75, 0.9, 1.0)]
    return [models[b] for b in picks]


@pytest.fixture(scope="module")
def batch_sample(oracle_mod):
    sample = _batch_sample()
    ref = [dict() for _ in sample]
    _parallel([(_oracle_horizons, (oracle_mod, m.copy(), (1000,), ref[b])) for b, m in enumerate(sample)])
    return sample, ref


@pytest.mark.parametrize("prec,wide_cluster", [("f64", 1), ("f64", 2), ("f64", 8), ("mixed", 1), ("mixed", 2)])
def test_uneven_batch_sample_against_oracle(batch_sample, prec, wide_cluster):
    """one batched launch; wide_cluster 1 keeps every instance in one block, 2 and 8 give the instances from 32768
    nodes + segments up (the largest two of the sample) a cluster of that many blocks each"""
    sample, ref = batch_sample
    assert sample[0].n > 20000 and sample[-1].n < 1000
    s = ws.GpuSolver([m.copy() for m in sample], precision=prec, threads=256, cta_state="global",
                     wide_cluster=wide_cluster)
    n_wide = sum(m.n + m.m >= 32768 for m in sample)
    assert s.wide == ((n_wide, wide_cluster) if wide_cluster > 1 else (0, 0))
    ctl = s.step(1000)
    rows = []
    for b, m in enumerate(sample):
        d = _diff(s.download(b, fields=("X", "u", "stuck")), ref[b][1000], m)
        rows.append(dict(d, nodes=m.n, crossings=m.K, rollbacks=ctl[b]["rollbacks"],
                         oracle_rollbacks=ref[b][1000]["rollbacks"], device_ms=ctl[b]["t_end_ms"] - ctl[b]["t_start_ms"],
                         start_ms=ctl[b]["t_start_ms"]))
    s.dispose()
    cases.record(f"uneven_batch_sample_{prec}_cluster{wide_cluster}", {"instances": rows})
    for b, r in enumerate(rows):
        assert ctl[b]["iter"] == 1000
        if prec == "f64":
            assert r["rollbacks"] == r["oracle_rollbacks"], (b, r)
            assert r["pos_span"] < 1e-9 and r["slide"] < SLIDE_F64 and r["stuck_mismatch"] == 0, (b, r)
        else:
            assert r["pos_span"] <= GATE, (b, r)


def test_wide_instance_is_batch_invariant_and_deterministic():
    """a wide instance (a cluster of blocks) gives the same bits alone, in a batch with one-block instances and on a
    rerun: its reduction order depends only on its own counts, the block size and the cluster size"""
    big = ws.configs.dome_small(seed=21)
    small = [ws.configs.dome_stiff(seed=5, side=3), ws.configs.dome_small(seed=9, side=3)]
    assert all(m.n + m.m < big.n + big.m for m in small)
    for prec in ("f64", "mixed"):
        outs = []
        for batch in ([big], [big], [small[0], big, small[1]]):
            s = ws.GpuSolver([m.copy() for m in batch], precision=prec, cta_state="global", wide_cluster=4,
                             wide_min=big.n + big.m)
            assert s.wide == (1, 4)
            ctl = s.step(600)
            b = batch.index(big)
            outs.append((ctl[b], s.download(b, fields=("X", "Q", "u", "slip", "Fn"))))
            assert all(c["iter"] == 600 for c in ctl)
            assert ctl[b]["t_end_ms"] > ctl[b]["t_start_ms"] >= 0.0
            s.dispose()
        for c, g in outs[1:]:
            assert c["rollbacks"] == outs[0][0]["rollbacks"] and c["residual"] == outs[0][0]["residual"]
            for k in g:
                assert np.array_equal(g[k], outs[0][1][k]), (prec, k)


@pytest.mark.parametrize("cluster", [2, 4, 8])
@pytest.mark.parametrize("order", ["auto", "general"])
def test_wide_instance_matches_oracle(oracle_mod, cluster, order):
    """the 3 m dome relaxed by clusters of 2, 4 and 8 blocks, both side orders, FP64 against the oracle with its
    iteration and roll-back counts"""
    md = ws.configs.dome_small()
    ref = {}
    _oracle_horizons(oracle_mod, md.copy(), (400, 1000), ref)
    s = ws.GpuSolver([md.copy()], precision="f64", cta_state="global", wide_cluster=cluster, wide_min=1,
                     side_order=order)
    assert s.wide == (1, cluster)
    done = 0
    for h in (400, 1000):
        ctl = s.step(h - done)[0]
        done = h
        g = s.download(0, fields=("X", "u", "stuck"))
        d = _diff(g, ref[h], md)
        assert ctl["iter"] == h and ctl["rollbacks"] == ref[h]["rollbacks"], h
        assert d["pos_span"] < 1e-9 and d["slide"] < SLIDE_F64 and d["stuck_mismatch"] == 0, (h, d)
    s.dispose()

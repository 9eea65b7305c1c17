"""Measured workloads besides the headline single-gridshell benchmark (bench.py --workload ...).

* ``precision`` — stiff 3 m domes (25×3 mm laths, E 12 GPa, per-crossing μ ~ U(0.1, 0.5)), one instance per seed,
  relaxed for the reference's default iteration cap (5000, params.js:20-23) in FP64, in the mixed policy (FP32 element
  math, two-float state, FP64 reductions) and in naive FP32.  Reported against FP64: max node position error / span,
  slide-coordinate error, stick/slip mismatches; and the chaos floor: FP64 against FP64 started 1 nm away.
* ``batch`` — 512 independent gridshells drawn from a seed (laths per family U{6..40}, span U(2, 12) m, thickness
  U(3, 6) mm, width U(30, 60) mm, E U(8, 14) GPa, μ U(0.1, 0.5), inward displacement U(3, 10) % of the span (the
  span's reduction: each support moves radially by half of it), ~5 cm segments), relaxed together to the iteration cap.
* ``ratio`` — the batched form (592 domes) against the plain single-instance form on the 3 m dome.
* ``serve`` — the serving loop under Poisson arrivals at the given rates: fresh stiff domes (new seed each) and, with
  probability 0.3, variants (±5 % E, ±0.1 μ, ±2 % support displacement) of a resident equilibrium, warm-started; a
  sample of the served results against FP64 (the same requests relaxed again in FP64) beside FP64's own chaos floor.
* ``scene`` — the reference's example scene dome_basic (read from its scene.json by the scene reader): one solve to
  convergence (or the scene's 8000-iteration cap) in FP64 and mixed, plain and batched forms; the mixed result against
  FP64 beside the chaos floor (FP64 against FP64 started with every node moved by ~1e-9·span and ~1e-7·span, the
  size of an FP32 rounding); 64 copies relaxed together.

Every solve here stops at convergence (relative residual ≤ tol) or at its iteration cap, as CpuSolver.run does.
"""
from __future__ import annotations

import time

import numpy as np

from . import configs, serve
from ._lib import default_params
from .solver import GpuSolver

CAP = 5000          # the reference's default max_iter (web/js/params.js:20-23)


def _stiff(seed, cap=CAP):
    return configs.dome_stiff(seed=seed, params=default_params(disp_ramp_iter=3000, max_iter=cap, strength=1e5,
                                                               stick_strength=1e5))


def _relax(models, precision, iters, threads=512):
    """relax a batch in the batched form; returns (per-instance states, control, GPU ms, launches)"""
    s = GpuSolver([m.copy() for m in models], precision=precision, threads=threads)
    ctl = s.step(iters)
    ms, nl = s.last_step_stats()
    st = [s.download(b, fields=("X", "u", "state", "stuck")) for b in range(len(models))]
    s.dispose()
    return st, ctl, ms, nl


def _compare(a, b, models):
    pos = [float(np.max(np.linalg.norm((x["X"] - y["X"]).reshape(-1, 3), axis=1)) / m.span) for x, y, m in zip(a, b, models)]
    du = [float(np.max(np.abs(x["u"] - y["u"]))) if m.K else 0.0 for x, y, m in zip(a, b, models)]
    state = [int(np.sum(x["state"] != y["state"])) for x, y in zip(a, b)]
    stuck = [int(np.sum(x["stuck"] != y["stuck"])) for x, y in zip(a, b)]
    return {"pos_err_span_median": float(np.median(pos)), "pos_err_span_max": float(np.max(pos)),
            "within_1e-4_span": int(np.sum(np.array(pos) <= 1e-4)), "slide_err_max_segments": float(np.max(du)),
            "slip_state_mismatch_total": int(np.sum(state)), "stick_mismatch_total": int(np.sum(stuck))}


def run_scene(path, copies=64):
    """a real scene: time to relax it on the device, FP64 and mixed, one instance (plain and batched forms) and a batch
    of copies; the mixed positions against FP64 (max node error / span)"""
    from .scenefile import load_scene
    md = load_scene(path)
    cap = int(md.params["max_iter"])
    out = {"scene": path.rsplit("/", 1)[-1], "nodes": md.n, "segments": md.m, "crossings": md.K, "iteration_cap": cap}
    X = {}
    for prec in ("f64", "mixed"):
        for form in ("plain", "cta"):
            s = GpuSolver([md.copy()], precision=prec, form=form)
            s.step(50)                  # first-launch costs and the plain form's graph capture out of the timing
            s.load_instance(0, md.copy())                  # back to the scene's start, iteration 0
            ctl = s.step(cap)[0]
            ms = s.last_step_stats()[0]
            X[(prec, form)] = s.download(0, fields=("X",))["X"]
            s.dispose()
            out[f"{prec}_{form}"] = {"gpu_ms": ms, "iterations": ctl["iter"], "status": ctl["status"],
                                     "residual": ctl["residual"], "iters_per_s": ctl["iter"] / (ms * 1e-3)}
    for eps in (1e-9, 1e-7):
        p = md.copy()
        p.X = p.X + eps * md.span * np.random.default_rng(1).standard_normal(p.X.shape)
        s = GpuSolver([p], precision="f64", form="plain")
        s.step(cap)
        X[eps] = s.download(0, fields=("X",))["X"]
        s.dispose()

    def err(a, b):
        return float(np.linalg.norm((X[a] - X[b]).reshape(-1, 3), axis=1).max() / md.span)
    out["mixed_vs_f64_pos_err_span"] = err(("mixed", "plain"), ("f64", "plain"))
    out["chaos_floor_f64_1e-9span_pos_err_span"] = err(1e-9, ("f64", "plain"))
    out["chaos_floor_f64_1e-7span_pos_err_span"] = err(1e-7, ("f64", "plain"))
    out["f64_cta_vs_plain_pos_err_span"] = err(("f64", "cta"), ("f64", "plain"))
    s = GpuSolver([md.copy() for _ in range(copies)], precision="mixed")
    ctl = s.step(cap)
    ms = s.last_step_stats()[0]
    s.dispose()
    out["batch"] = {"copies": copies, "gpu_ms": ms, "solves_per_s": copies / (ms * 1e-3),
                    "inst_iters_per_s": sum(c["iter"] for c in ctl) / (ms * 1e-3)}
    return out


def run_precision(instances=64, iters=CAP, seed0=1, horizons=(500, 1000, 2000, 3000, 5000)):
    """FP64, FP64 started 1 nm away (the chaos floor), mixed and naive FP32 stepped side by side; at every horizon the
    three are compared with FP64"""
    models = [_stiff(seed0 + b) for b in range(instances)]
    _relax(models[:2], "mixed", 20)                       # module load and first-launch costs out of the timings
    rng = np.random.default_rng(7)
    pert = []
    for m in models:
        p = m.copy()
        p.X = p.X + 1e-9 * rng.standard_normal(p.X.shape)
        pert.append(p)
    runs = {"f64": GpuSolver([m.copy() for m in models], precision="f64", threads=512),
            "chaos_floor_f64_1nm": GpuSolver(pert, precision="f64", threads=512),
            "mixed": GpuSolver([m.copy() for m in models], precision="mixed", threads=512),
            "f32": GpuSolver([m.copy() for m in models], precision="f32", threads=512)}
    gpu_ms = {k: 0.0 for k in runs}
    ctl = {}
    out = {"instances": instances, "iterations": iters, "nodes": models[0].n, "crossings": models[0].K, "horizons": []}
    done = 0
    for h in [h for h in horizons if h <= iters]:
        st = {}
        for k, s in runs.items():
            ctl[k] = s.step(h - done)
            gpu_ms[k] += s.last_step_stats()[0]
            st[k] = [s.download(b, fields=("X", "u", "state", "stuck")) for b in range(instances)]
        done = h
        row = {"iteration": h}
        for k in ("chaos_floor_f64_1nm", "mixed", "f32"):
            row[k] = _compare(st[k], st["f64"], models)
        out["horizons"].append(row)
    for k, s in runs.items():
        out[k] = {"gpu_ms": gpu_ms[k], "inst_iters_per_s": sum(c["iter"] for c in ctl[k]) / (gpu_ms[k] * 1e-3),
                  "converged": sum(c["status"] == 1 for c in ctl[k]), "nonfinite": sum(c["status"] == 3 for c in ctl[k])}
        s.dispose()
    return out


def run_ratio(batch=592, iters=400):
    """the batched form against the plain single-instance GPU form on the 3 m dome (mixed precision)"""
    models = [configs.dome_small(seed=1 + b) for b in range(batch)]
    s = GpuSolver([models[0].copy()], precision="mixed", form="plain")
    s.step(iters, read=False)               # untimed: the first launches and the capture of the iteration graph
    s.step(iters, read=False)
    ms_plain = s.last_step_stats()[0]
    s.dispose()
    s = GpuSolver(models, precision="mixed", threads=512)
    s.step(iters, read=False)
    s.step(iters, read=False)
    ms_batch = s.last_step_stats()[0]
    s.dispose()
    plain = iters / (ms_plain * 1e-3)
    batched = batch * iters / (ms_batch * 1e-3)
    return {"workload": "dome_small (1176 nodes, 156 crossings), mixed precision", "iterations": iters,
            "plain_single_iters_per_s": plain, "batched_instances": batch, "batched_inst_iters_per_s": batched,
            "batched_over_plain": batched / plain}


def _plain_iter_ms(models, precision, iters=200):
    """device ms per iteration of the plain single-instance form on each model (after an untimed step of the same
    length, which captures the iteration graph the timed step launches)"""
    out = []
    for m in models:
        s = GpuSolver([m.copy()], precision=precision, form="plain")
        s.step(iters, read=False)
        s.step(iters, read=False)
        out.append(s.last_step_stats()[0] / iters)
        s.dispose()
    return out


def run_batch(count=512, iters=CAP, precision="mixed", threads=0, seed=4, wide_cluster=0, wide_min=0, plain_sample=16,
              tune=False):
    """the uneven batch in one batched step to the iteration cap; per-instance device times (from the block or cluster
    taking the instance up to its leaving it); and the plain single-instance form on a size-stratified sample of the
    same instances, whose per-iteration times, interpolated over the sizes of all instances, give the time the plain form
    would take to relax the whole batch one instance after another"""
    models = configs.batch_mixed(count, seed=seed)
    for m in models:
        m.params = dict(m.params, max_iter=iters)
    t0 = time.perf_counter()
    s = GpuSolver(models, precision=precision, threads=threads, wide_cluster=wide_cluster, wide_min=wide_min, tune=tune)
    create_s = time.perf_counter() - t0
    n_wide, cl = s.wide
    shape = s.shape
    # an untimed first step (the first launches of a process cost about 1.5 s here), then every instance back to its
    # start: the timed step relaxes the batch from iteration 0 as if it were the first
    s.step(20, read=False)
    for b, m in enumerate(models):
        s.load_instance(b, m)
    ctl = s.step(iters)
    ms, nl = s.last_step_stats()
    dev_bytes = s.device_bytes
    s.dispose()
    its = sum(c["iter"] for c in ctl)
    node_its = sum(c["iter"] * m.n for c, m in zip(ctl, models))
    n = np.array([m.n for m in models])
    dev = np.array([c["t_end_ms"] - c["t_start_ms"] for c in ctl])
    end = np.array([c["t_end_ms"] for c in ctl])
    big = int(np.argmax(n))
    out = {"instances": count, "iteration_cap": iters, "gpu_ms": ms, "solves_per_s": count / (ms * 1e-3),
           "inst_iters_per_s": its / (ms * 1e-3), "node_iters_per_s": node_its / (ms * 1e-3),
           "converged": sum(c["status"] == 1 for c in ctl), "nonfinite": sum(c["status"] == 3 for c in ctl),
           "nodes_min": int(n.min()), "nodes_median": int(np.median(n)), "nodes_max": int(n.max()),
           "nodes_total": int(n.sum()), "crossings_total": int(sum(m.K for m in models)), "device_bytes": dev_bytes,
           "create_s": create_s, "launches": nl, "wide_instances": n_wide, "wide_cluster": cl, "shape": shape,
           "instance_device_ms": {"min": float(dev.min()), "median": float(np.median(dev)), "max": float(dev.max()),
                                  "largest_instance": float(dev[big]), "largest_instance_end": float(end[big]),
                                  "last_end": float(end.max()), "p90_end": float(np.percentile(end, 90))},
           "longest_instance_nodes": int(n[int(np.argmax(dev))])}
    if plain_sample:
        order = np.argsort(n)
        pick = sorted(set(int(order[int(q * (count - 1))]) for q in np.linspace(0.0, 1.0, plain_sample)), key=lambda b: n[b])
        per = _plain_iter_ms([models[b] for b in pick], precision)
        xs, ys = np.array([n[b] for b in pick], dtype=float), np.array(per)
        plain_total_ms = float(np.sum(np.interp(n, xs, ys))) * iters
        out["plain_form"] = {"sample_nodes": [int(v) for v in xs], "sample_ms_per_iter": [float(v) for v in ys],
                             "batch_one_after_another_ms": plain_total_ms,
                             "solves_per_s": count / (plain_total_ms * 1e-3)}
        out["batched_over_plain"] = out["solves_per_s"] / out["plain_form"]["solves_per_s"]
    return out


def run_serve(rates=(50.0, 200.0, 1000.0), counts=(300, 600, 1000), slots=296, chunk=250, budget_bytes=150 * 10 ** 9,
              time_limit=120.0):
    tpl = _stiff(1)
    out = {"slots": slots, "chunk_iters": chunk, "fresh_cap": CAP, "variant_cap": 1500, "rates": []}
    srv = serve.Server(tpl, slots=slots, chunk=chunk, budget_bytes=budget_bytes)
    out["slots"] = srv.slots
    # a warm bank of resident equilibria for the variants
    seed_reqs = serve.poisson_stream(1e6, 8, seed=1, variant_share=0.0, fresh_cap=CAP)
    srv.run(seed_reqs, time_limit=time_limit)
    bank = list(srv.resident.values())
    served = []
    for rate, count in zip(rates, counts):
        srv.done, srv.ticks, srv.busy_slot_ticks = [], 0, 0
        reqs = serve.poisson_stream(rate, count, seed=int(rate), variant_share=0.3, fresh_cap=CAP, variant_cap=1500,
                                    warm_bank=bank)
        t0 = time.perf_counter()
        done = srv.run(reqs, time_limit=time_limit)
        wall = time.perf_counter() - t0
        served += done
        lat = serve.latency_summary(done)
        fresh = [r for r in done if r.kind == "fresh"]
        var = [r for r in done if r.kind == "variant"]
        out["rates"].append(dict(rate_per_s=rate, requests=count, finished=len(done), wall_s=wall,
                                 solves_per_s=len(done) / wall, fresh=len(fresh), variants=len(var),
                                 converged=sum(r.status == 1 for r in done),
                                 mean_busy_slots=srv.busy_slot_ticks / max(srv.ticks, 1),
                                 p50_s=lat["p50_s"], p99_s=lat["p99_s"], p999_s=lat["p999_s"], mean_s=lat["mean_s"],
                                 fresh_p50_s=serve.latency_summary(fresh)["p50_s"] if fresh else None,
                                 variant_p50_s=serve.latency_summary(var)["p50_s"] if var else None))
    srv.dispose()
    out["error_vs_f64"] = _served_error(served)
    return out


def _served_error(done, sample=64, seed=3):
    """the served (mixed-precision) results against FP64: a sample of the finished requests relaxed again from their
    start in FP64, one batch, each to the iteration count it was served at; beside it the chaos floor, FP64 started with
    every node moved by 1e-9 of the span.  Max node distance / span per request (median, max, and how many are within
    1e-4), slide coordinates (segments) and stick/slip states."""
    rng = np.random.default_rng(seed)
    pick = [done[i] for i in sorted(rng.choice(len(done), size=min(sample, len(done)), replace=False))]
    models, pert = [], []
    for r in pick:
        m = r.model.copy()
        m.params = dict(m.params, max_iter=int(r.iters))
        models.append(m)
        p = m.copy()
        p.X = p.X + 1e-9 * m.span * rng.standard_normal(p.X.shape)
        pert.append(p)
    cap = max(int(r.iters) for r in pick)
    ref, _, _, _ = _relax(models, "f64", cap)
    flo, _, _, _ = _relax(pert, "f64", cap)
    served = [{"X": r.result["X"], "u": r.result["u"], "state": r.result["state"], "stuck": r.result["stuck"]} for r in pick]
    out = {"requests": len(pick), "fresh": sum(r.kind == "fresh" for r in pick), "variants": sum(r.kind == "variant" for r in pick),
           "served_mixed": _compare(served, ref, models), "chaos_floor_f64": _compare(flo, ref, models)}
    for kind in ("fresh", "variant"):
        idx = [i for i, r in enumerate(pick) if r.kind == kind]
        if idx:
            out[f"served_mixed_{kind}"] = _compare([served[i] for i in idx], [ref[i] for i in idx], [models[i] for i in idx])
    return out

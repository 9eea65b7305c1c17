"""Benchmark of the DR hot path (one JSON line on rank 0).

Workload at N = 1: the single large gridshell ("shell_large": 20 m hexagonal plan, 60 laths per family at 0.33 m,
3.8 cm segments, supports lifted 0-2 m by a seeded field; 81,180 nodes, 81,000 segments, 8,190 crossings), relaxed in
FP32 element math with two-float positions/frames and FP64 reductions.  A step is one chunk of DR iterations; value is
DR iterations per second of the whole job (all ranks).  Between timed steps a 256 MiB buffer is written to flush L2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--chunk C] [--impl ours|reference]
    python bench.py --workload precision|batch|serve|ratio|scene   (one JSON line each; weave-sim_b200/workloads.py)

--impl reference runs the reference's CPU algorithm (the f64 restatement under oracle/, the reference's JS being
unrunnable without a JS engine) on the host cores: one replica of the workload per thread, a bounded sample of
iterations per step.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solves/s and DR iters/s at ≤1e-4·span error vs f64; p50/p99 solve latency"
UNIT = "DR iters/s"
SHELL_FIXTURE = os.path.join(ROOT, "oracle", "scenes", "shell_large.npz")


def bench_config(args, world):
    """the workload, the same in both arms (the arithmetic of each arm is in its `dtype`)"""
    return {"workload": "shell_large: 20 m hexagonal Kagome plan, 60 laths/family at 0.33 m, 3.8 cm segments, "
                        "supports lifted 0-2 m (81180 nodes, 81000 segments, 8190 crossings)",
            "nodes": 81180, "segments": 81000, "crossings": 8190, "chunk_iters": args.chunk,
            "step": f"one chunk of {args.chunk} DR iterations of the shell",
            "l2": "flushed between timed steps (256 MiB write)", "parallelism": f"instance replicas x{world}"}

# algorithmic bytes of one DR iteration: minimal state traffic if every state array is streamed once
# (node 112 B, segment 168 B, crossing 96 B per iteration)
def bytes_per_iter(n, m, K):
    return 112 * n + 168 * m + 96 * K


# DRAM bytes (read + write) of one iteration of this workload in the mixed plain form, summed over its four kernels from
# a cold-cache `ncu --set full` capture of one launch each (the plain-form summary under profiles/)
TRAFFIC_PER_ITER = (4.15 + 9.75 + 6.49 + 10.53) * 1e6


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms while the timed region runs"""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device=0):
        self.device, self.rows, self.proc = device, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
            except (ValueError, IndexError):
                continue
            for k, name in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(gpus):
    """one process per GPU under torchrun; returns (rank, world, local_rank)"""
    if gpus <= 1 or "RANK" not in os.environ:
        return 0, 1, 0
    import torch.distributed as dist
    import datetime
    rank, world, local = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"]), int(os.environ.get("LOCAL_RANK", 0))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def allmax(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def flush_l2(buf):
    import torch
    buf.add_(1)          # 256 MiB write: larger than the 126 MB L2


def run_ours(args, rank, world, local):
    import numpy as np
    import torch
    import weavesim_b200 as ws

    torch.cuda.set_device(local)
    md = ws.configs.shell_large()
    n, m, K = md.n, md.m, md.K
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")
    s = ws.GpuSolver([md.copy()], precision=args.precision, form=args.form, device=local)
    for _ in range(args.warmup):
        s.step(args.chunk, read=False)
        s.last_step_stats()
    barrier(world)
    torch.cuda.synchronize()
    times, launches = [], 0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush_l2(flush)
            torch.cuda.synchronize()
            s.step(args.chunk, read=False)
            ms, nl = s.last_step_stats()        # CUDA events on the solver's stream around the step
            times.append(ms)
            launches += nl
    torch.cuda.synchronize()
    barrier(world)
    total_ms = allmax(sum(times), world)
    ctl = s.read_control()[0]
    err = error_vs_f64(md, s.download(0, fields=("X", "u", "stuck")), ctl["iter"], local)
    # end to end through the C ABI with host buffers: upload state, relax one chunk, download the result (positions,
    # frames, slide coordinates, contact normals and stick/slip: what a caller reads back, and warm-starts from)
    result_fields = ("X", "Q", "u", "nprev", "stuck", "state")
    st0 = s.download(0)
    X, Q, u = st0["X"].copy(), st0["Q"].copy(), st0["u"].copy()
    e2e_t = []
    for _ in range(max(2, args.steps // 2)):
        t0 = time.perf_counter()
        s.upload_state(0, X, Q, u)
        s.step(args.chunk, read=False)
        out = s.download(0, fields=result_fields)
        e2e_t.append(time.perf_counter() - t0)
    h2d = X.nbytes + Q.nbytes + u.nbytes
    d2h = sum(v.nbytes for v in out.values())
    e2e_s = allmax(statistics.median(e2e_t), world)
    s.dispose()
    its = args.steps * args.chunk
    value = world * its / (total_ms * 1e-3)
    ms_iter = sum(times) / its
    bpi = bytes_per_iter(n, m, K)
    peak, peak_kind = peaks()
    achieved = bpi / (ms_iter * 1e-3) / 1e9
    return {
        "value": value, "ms_per_step": total_ms / args.steps, "launches": launches, "ctl": ctl,
        "e2e": {"value": world * args.chunk / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": TRAFFIC_PER_ITER if args.precision == "mixed" and args.form == "plain" else None,
                     "peak_kind": f"{peak_kind} hbm_gbs", "bytes_per_iter": bpi,
                     "note": "one DR iteration (four kernels, two pairs on forked graph branches) is the unit: algorithmic "
                             "state bytes per iteration / device time per iteration; traffic = DRAM bytes read + written "
                             "per iteration, summed over the four kernels from one cold-cache ncu capture"},
        "clocks": clk.summary(), "sizes": {"n": n, "m": m, "K": K}, "error_vs_f64": err,
    }


PRECISION_NOTE = {"mixed": "FP32 element math + two-float positions/frames + FP64 reductions", "f64": "FP64 throughout",
                  "f32": "naive FP32 throughout"}


def error_vs_f64(md, st, iters, device):
    """the timed run's result against FP64 at the same iteration: the shell relaxed from the same start for the same
    iterations in FP64 (the plain form, which the GPU tests hold to the f64 oracle), max node distance / span, slide
    coordinates and stick/slip states; beside it the chaos floor, FP64 against FP64 started with every coordinate moved
    by N(0, (1e-9 span)^2)"""
    import numpy as np
    import weavesim_b200 as ws

    def run(model):
        r = ws.GpuSolver([model], precision="f64", form="plain", device=device)
        r.step(iters, read=False)
        out = r.download(0, fields=("X", "u", "stuck"))
        r.dispose()
        return out

    def cmp(a, b):
        d = np.linalg.norm((a["X"] - b["X"]).reshape(-1, 3), axis=1)
        return {"pos_max_span": float(d.max() / md.span), "slide_max_segments": float(np.abs(a["u"] - b["u"]).max()),
                "stick_slip_mismatch": int(np.sum(a["stuck"] != b["stuck"]))}

    ref = run(md.copy())
    pert = md.copy()
    pert.X = pert.X + 1e-9 * md.span * np.random.default_rng(7).standard_normal(pert.X.shape)
    out = cmp(st, ref)
    floor = cmp(run(pert), ref)
    return dict(out, iterations=int(iters), crossings=int(md.K), within_1e_4_span=out["pos_max_span"] <= 1e-4,
                chaos_floor=floor)


def cpu_replicas(iters_per_replica, threads):
    """the reference's CPU algorithm (oracle/: f64 restatement of web/js/solver_cpu.js) on `threads` host threads, one
    replica of the workload each; returns aggregate DR iterations per second.  The shell is read from the oracle's
    scene fixture (made by the package's scene builder, oracle/scenes/make_scenes.py), so this leg loads the oracle's
    library alone, never the CUDA library."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import weavesim_b200 as ws
    from oracle import Oracle
    md = ws.Model.load(SHELL_FIXTURE)
    ors = [Oracle(md.copy()) for _ in range(threads)]
    for o in ors:
        o.step(1)
    t0 = time.perf_counter()
    th = [threading.Thread(target=o.step, args=(iters_per_replica,)) for o in ors]   # ctypes releases the GIL
    for t in th:
        t.start()
    for t in th:
        t.join()
    dt = time.perf_counter() - t0
    return threads * iters_per_replica / dt, dt


def cpu_scene(path):
    """CPU baseline leg of the scene workload: the reference's CPU algorithm (oracle/, f64) relaxing the scene on one
    thread to convergence or its cap; returns (seconds, iterations)"""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import weavesim_b200 as ws
    from oracle import Oracle
    md = ws.load_scene(path)
    o = Oracle(md.copy())
    t0 = time.perf_counter()
    v = o.run(int(md.params["max_iter"]), chunk=500)
    return time.perf_counter() - t0, int(v["iteration"])


def cpu_dome(iters, threads=0):
    """CPU baseline leg of the ratio workload: the reference's CPU algorithm (oracle/, f64) on the 3 m dome, one thread
    alone and one replica per host thread; returns (1-thread iters/s, all-thread instance iters/s, threads)"""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import weavesim_b200 as ws
    from oracle import Oracle
    threads = threads or os.cpu_count() or 1
    one = Oracle(ws.configs.dome_small(seed=1))
    one.step(1)
    t0 = time.perf_counter()
    one.step(iters)
    cpu1 = iters / (time.perf_counter() - t0)
    ors = [Oracle(ws.configs.dome_small(seed=1 + b)) for b in range(threads)]
    for o in ors:
        o.step(1)
    t0 = time.perf_counter()
    th = [threading.Thread(target=o.step, args=(iters,)) for o in ors]    # ctypes releases the GIL
    for t in th:
        t.start()
    for t in th:
        t.join()
    return cpu1, threads * iters / (time.perf_counter() - t0), threads


def run_reference(args, rank, world):
    if rank != 0:
        return None
    cores = os.cpu_count() or 1
    vals = []
    for _ in range(args.warmup):
        cpu_replicas(2, cores)
    for _ in range(args.steps):
        v, _ = cpu_replicas(args.ref_iters, cores)
        vals.append(v)
    value = statistics.median(vals)
    sample = f"{cores} replicas of shell_large (one per thread), {args.ref_iters} DR iterations each per step"
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * cores * args.ref_iters / value, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": bench_config(args, world), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_workload(args):
    import weavesim_b200 as ws
    from weavesim_b200 import workloads
    t0 = time.perf_counter()
    with ClockSampler(0) as clk:
        if args.workload == "precision":
            r = workloads.run_precision(instances=args.instances or 64)
            metric = "position / slide / stick-slip agreement with FP64 after the 5000-iteration cap, and throughput"
        elif args.workload == "batch":
            r = workloads.run_batch(count=args.instances or 512, wide_cluster=args.wide_cluster, threads=args.threads,
                                    wide_min=args.wide_min, tune=not args.no_tune, plain_sample=0 if args.no_plain else 16)
            metric = "solves/s and DR iters/s of 512 mixed gridshells to the 5000-iteration cap"
        elif args.workload == "ratio":
            r = workloads.run_ratio()
            cpu1, cpuN, threads = cpu_dome(r["iterations"])
            r.update(cpu_port_1_thread_iters_per_s=cpu1, cpu_port_threads=threads,
                     cpu_port_all_threads_inst_iters_per_s=cpuN, batched_over_cpu_all_threads=r["batched_inst_iters_per_s"] / cpuN,
                     batched_over_cpu_1_thread=r["batched_inst_iters_per_s"] / cpu1)
            metric = "batched vs plain single-instance GPU form vs the CPU port, DR iters/s on the 3 m dome"
        elif args.workload == "scene":
            path = os.path.join(ROOT, "tests", "golden", "dome_basic_scene.json")
            r = workloads.run_scene(path)
            cpu_s, cpu_it = cpu_scene(path)
            r.update(cpu_port_1_thread_solve_s=cpu_s, cpu_port_iterations=cpu_it,
                     f64_plain_over_cpu=cpu_s / (r["f64_plain"]["gpu_ms"] * 1e-3),
                     mixed_plain_over_cpu=cpu_s / (r["mixed_plain"]["gpu_ms"] * 1e-3))
            metric = "time to relax the reference's example scene dome_basic: GPU forms and precisions vs the CPU port"
        else:
            r = workloads.run_serve()
            metric = "p50/p99/p99.9 solve latency and solves/s under Poisson arrivals"
    print(json.dumps({"workload": args.workload, "metric": metric, "result": r, "clocks": clk.summary(),
                      "wall_s": time.perf_counter() - t0, "data": "synthetic (seeded)", "gpu": ws.device_count() > 0}),
          flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--chunk", type=int, default=200, help="DR iterations per step")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["f64", "mixed", "f32"])
    ap.add_argument("--form", default="plain", choices=["plain", "grid", "cta"])
    ap.add_argument("--ref-iters", type=int, default=10, help="DR iterations per replica per step of the CPU arm")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="shell_large",
                    choices=["shell_large", "precision", "batch", "serve", "ratio", "scene"],
                    help="shell_large: the headline line; the others measure the stiff-dome precision variants, the "
                         "512-gridshell mixed batch and the serving loop (single GPU)")
    ap.add_argument("--instances", type=int, default=0, help="instances of the precision / batch workloads")
    ap.add_argument("--wide-cluster", type=int, default=0, help="batch workload: blocks per wide instance (1: none)")
    ap.add_argument("--wide-min", type=int, default=0, help="batch workload: nodes + segments of a wide instance")
    ap.add_argument("--threads", type=int, default=0, help="batch workload: threads per block of the one-block kernels")
    ap.add_argument("--no-tune", action="store_true",
                    help="batch workload: the launch shape from --threads / --wide-cluster / --wide-min instead of the "
                         "autotuner's (the default: the autotuner picks it, or takes it from its cache)")
    ap.add_argument("--no-plain", action="store_true", help="batch workload: skip the plain-form comparison")
    args = ap.parse_args()
    if args.workload != "shell_large":
        run_workload(args)
        return
    rank, world, local = dist_setup(args.gpus)
    if args.impl == "reference":
        out = run_reference(args, rank, world)
        if rank == 0:
            print(json.dumps(out), flush=True)
        return
    r = run_ours(args, rank, world, local)
    if rank != 0:
        return
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        v, dt = cpu_replicas(args.ref_iters * 2, cores)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{cores} replicas of shell_large, {args.ref_iters * 2} DR iterations each ({dt:.1f} s)"}
    out = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": {"mixed": "f32+two-float+f64", "f64": "f64", "f32": "f32"}[args.precision], "data": "synthetic (seeded)",
           "config": bench_config(args, world), "form": args.form, "precision": PRECISION_NOTE[args.precision],
           "e2e": r["e2e"], "gpu_launches": r["launches"], "roofline": r["roofline"], "cpu_baseline": cpu,
           "clocks": r["clocks"], "error_vs_f64": r["error_vs_f64"], "residual_after": r["ctl"]["residual"],
           "iterations_after": r["ctl"]["iter"]}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()

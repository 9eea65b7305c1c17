"""Serving loop: continuous batching of relaxation requests on one GPU.

* Requests are served from pools of device-resident slots (one instance each), one pool per topology (the element
  counts a slot is made for: nodes, segments, joints, clamps, crossings, strands).  A pool is created when the first
  request of its topology arrives, with as many slots as the device-memory budget left over allows (bytes of one slot
  measured on the device) up to ``slots``; requests of a topology whose pool is full, or for which the budget has no
  room, wait.  Nothing is allocated while a pool runs.
* A request is admitted when a slot of its pool is free (``GpuSolver.load_instance``: goals, contact set-up and state
  of the new model replace the slot's, the other slots keep running); otherwise it waits in arrival order.
* Every tick advances the busy slots of every pool by ``chunk`` DR iterations, one batched launch a pool (one thread
  block per slot, each stopping at its own convergence or iteration cap), so requests at different stages share the
  device.
* Finished slots are downloaded (positions, frames, slide coordinates, stick/slip) and freed.
* A variant request (±E, ±μ, ±support displacement of a resident equilibrium) starts from that equilibrium with the
  contact fully on and no warm-up, the warm start of CpuSolver.rebuildGoals (web/js/solver_cpu.js:719-732).

Latency is measured on the host clock from a request's arrival to the end of its download.
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field

import numpy as np

from . import configs
from ._lib import default_params
from .solver import GpuSolver


@dataclass
class Request:
    rid: int
    arrival: float                  # seconds since the start of the run
    model: object
    kind: str                       # "fresh" | "variant"
    cap: int                        # iteration cap of the solve
    base: int = -1                  # rid of the resident equilibrium a variant starts from
    admitted: float = 0.0
    done: float = 0.0
    iters: int = 0
    status: int = 0
    result: dict = field(default_factory=dict)


def variant_of(model, eq, rng, disp_ramp=500):
    """A parameter variant of a resident equilibrium: E × (1 ± 5 %), μ ± 0.1, support displacement × (1 ± 2 %); the
    state starts at the equilibrium `eq` (X, Q, u, nprev of a finished solve)."""
    v = model.copy()
    f = 1.0 + rng.uniform(-0.05, 0.05)
    for k in ("EA", "EIx", "EIy", "GJ", "GA"):
        setattr(v, k, getattr(v, k) * f)
    v.cross_mu = np.clip(v.cross_mu + rng.uniform(-0.1, 0.1), 0.0, None)
    if v.anchor_target is not None:
        start = model.X.reshape(-1, 3)[model.anchor_node]           # the flat positions of the supports
        tgt = v.anchor_target.reshape(-1, 3)
        v.anchor_target = (start + (tgt - start) * (1.0 + rng.uniform(-0.02, 0.02))).ravel()
    v.X = eq["X"].copy()
    v.Q = eq["Q"].copy()
    v.cross_u = eq["u"].copy()
    v.cross_nprev = eq["nprev"].copy()
    v.params = dict(v.params, warmup_iter=0, ramp_iter=0, disp_ramp_iter=disp_ramp)
    return v


def topology_key(md):
    """the element counts a serving slot is made for (ws_load_instance refuses a model whose counts differ): nodes,
    segments, joints, crossings, strands and clamp joints (one per segment at an anchor that holds a rotation)"""
    rot = np.asarray(md.anchor_node)[(np.asarray(md.anchor_mask).astype(np.int64) & 0x38) != 0]
    seg = np.concatenate([np.asarray(md.seg_i0), np.asarray(md.seg_i1)])
    clamps = int(np.isin(seg, rot).sum())
    return (int(md.n), int(md.m), int(md.p), int(md.K), int(md.n_strands), clamps)


class _Pool:
    """the slots of one topology: a batched solver over `count` copies of a template, its free and busy slots"""

    def __init__(self, template, count, precision, threads, device):
        self.solver = GpuSolver([template.copy() for _ in range(count)], precision=precision, threads=threads,
                                device=device)
        self.slots = count
        self.free = collections.deque(range(count))
        self.busy = {}                  # slot -> Request


class Server:
    def __init__(self, template, slots=64, budget_bytes=150 * 10 ** 9, precision="mixed", threads=256, chunk=250, device=0):
        self.precision, self.threads, self.device = precision, threads, device
        self.max_slots, self.budget_bytes = slots, budget_bytes
        self.chunk = chunk
        self.pools = {}                 # topology -> _Pool
        self.per_slot = {}              # topology -> device bytes of one slot
        self.used_bytes = 0
        self.queue = collections.deque()
        self.done = []
        self.resident = {}              # rid -> (model, equilibrium state) kept for warm starts
        self.ticks = 0
        self.busy_slot_ticks = 0
        self._pool(template)
        if not self.pools:
            raise RuntimeError("serve: the device-memory budget holds no slot of the template")

    @property
    def slots(self):
        return sum(p.slots for p in self.pools.values())

    def _pool(self, model):
        """the pool of the model's topology, created within the budget when there is none; None when it cannot be"""
        key = topology_key(model)
        pool = self.pools.get(key)
        if pool is not None:
            return pool
        if key not in self.per_slot:
            probe = GpuSolver([model.copy()], precision=self.precision, threads=self.threads, device=self.device)
            self.per_slot[key] = max(int(probe.device_bytes), 1)
            probe.dispose()
        count = int(min(self.max_slots, (self.budget_bytes - self.used_bytes) // self.per_slot[key]))
        if count < 1:
            return None
        pool = _Pool(model, count, self.precision, self.threads, self.device)
        self.used_bytes += pool.solver.device_bytes
        self.pools[key] = pool
        return pool

    def submit(self, req: Request):
        self.queue.append(req)

    def _admit(self, now):
        waiting = collections.deque()
        while self.queue and self.queue[0].arrival <= now:
            req = self.queue.popleft()
            pool = self._pool(req.model)
            if pool is None or not pool.free:
                waiting.append(req)             # its topology has no free slot (or no room in the budget) yet
                continue
            b = pool.free.popleft()
            pool.solver.load_instance(b, req.model)
            req.admitted = now
            pool.busy[b] = req
        waiting.extend(self.queue)
        self.queue = waiting

    def tick(self, now):
        """admit, advance every busy slot by one chunk, retire the finished ones; returns the number retired"""
        self._admit(now)
        busy = [p for p in self.pools.values() if p.busy]
        if not busy:
            return 0
        self.ticks += 1
        retired = 0
        for pool in busy:
            slots = sorted(pool.busy)
            ctl = pool.solver.step(self.chunk, instances=slots)
            self.busy_slot_ticks += len(slots)
            for b in slots:
                c = ctl[b]
                req = pool.busy[b]
                if c["status"] != 0 or c["iter"] >= req.cap:
                    st = pool.solver.download(b)
                    req.result = {"X": st["X"], "Q": st["Q"], "u": st["u"], "nprev": st["nprev"], "state": st["state"],
                                  "stuck": st["stuck"], "residual": c["residual"]}
                    req.iters, req.status = c["iter"], c["status"]
                    del pool.busy[b]
                    pool.free.append(b)
                    retired += 1
                    if req.kind == "fresh":
                        self.resident[req.rid] = (req.model, req.result)
                    req.done = time.perf_counter() - self.t0
                    self.done.append(req)
        return retired

    def run(self, requests, time_limit=120.0):
        """serve a list of requests (sorted by arrival) in real time; returns the finished ones"""
        self.t0 = time.perf_counter()
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        while True:
            now = time.perf_counter() - self.t0
            while pending and pending[0].arrival <= now:
                self.submit(pending.popleft())
            if not any(p.busy for p in self.pools.values()) and not self.queue:
                if not pending:
                    break
                time.sleep(max(0.0, min(pending[0].arrival - now, 0.01)))
                continue
            if not any(p.busy for p in self.pools.values()) and not pending and all(
                    self._pool(r.model) is None for r in self.queue):
                raise RuntimeError("serve: queued requests whose topology the device-memory budget cannot hold")
            self.tick(now)
            if now > time_limit:
                break
        return self.done

    def dispose(self):
        for p in self.pools.values():
            p.solver.dispose()
        self.pools = {}


def poisson_stream(rate, count, seed=5, variant_share=0.3, fresh_cap=6000, variant_cap=1500, warm_bank=None):
    """requests at Poisson arrivals: fresh gridshells drawn like the stiff 3 m dome (25×3 mm, E 12 GPa, μ ~ U(0.1, 0.5)
    per crossing, new seed each) and, with probability `variant_share`, variants of an equilibrium from `warm_bank`
    (a list of (model, state) pairs)."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        if warm_bank and rng.uniform() < variant_share:
            base_model, eq = warm_bank[int(rng.integers(len(warm_bank)))]
            out.append(Request(i, t, variant_of(base_model, eq, rng), "variant", variant_cap))
        else:
            md = configs.dome_stiff(seed=int(rng.integers(1, 2 ** 31)),
                                    params=default_params(disp_ramp_iter=3000, max_iter=fresh_cap, strength=1e5,
                                                          stick_strength=1e5))
            out.append(Request(i, t, md, "fresh", fresh_cap))
    return out


def latency_summary(done):
    lat = np.array([r.done - r.arrival for r in done]) if done else np.zeros(1)
    return {"count": len(done), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "p999_s": float(np.percentile(lat, 99.9)), "mean_s": float(lat.mean())}

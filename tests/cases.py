"""Test scenes: the constructions of the reference's web/tests/cases.mjs:10-66 (mm, N) and the gridshell workloads.

* straight(L, nseg)            cases.mjs:10-13
* cantilever(nseg, dir)        rod_bench.mjs:27-36 (60×30 mm, E 1e4 N/mm², G 625, tip load 10 N, clamped at frame (0,0))
* crossing(load, pull, ...)    cases.mjs:14-28 (two 1000 mm laths, 10 segments, h = 30, B free in x)
* case_by_name(name)           cases.mjs:29-50 (cantilever, cantilever_edge, torsion, cross_press/stick/slip/locked,
                               cross_w23) and browser_cases.js:41-45 (cross_al)
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

import weavesim_b200 as ws

E_MM, G_MM, KAPPA = 1e4, 625.0, 5.0 / 6.0


def mm_params(**over):
    """the reference's defaults in its own units (params.js:8-23: strength 1e4 N/mm, epsilon 15 mm)"""
    kw = dict(strength=1e4, stick_strength=1e4, epsilon=15.0)
    kw.update(over)
    return ws.default_params(**kw)


def straight(L=1000.0, nseg=10, normals=None, anchors=(), loads=(), **kw):
    pts = np.array([[L * i / nseg, 0.0, 0.0] for i in range(nseg + 1)])
    return ws.polylines([pts], normals=None if normals is None else [normals], anchors=anchors, loads=loads,
                        E=E_MM, G=G_MM, **kw)


def cantilever(nseg=10, direction=2, P=10.0, tol=1e-10, max_iter=600000, w=60.0, h=30.0, L=1000.0):
    md = straight(L, nseg, anchors=[((0, 0), ws.mask(1, 1, 1, 1, 1, 1))], width=w, height=h,
                  params=mm_params(tol=tol, max_iter=max_iter, contacts=0))
    tip = int(np.argmax(md.X[0::3]))
    md.load_const[3 * tip + direction] -= P
    md.tip = tip
    return md


def timoshenko(direction=2, P=10.0, L=1000.0, w=60.0, h=30.0):
    I = w * h ** 3 / 12 if direction == 2 else h * w ** 3 / 12
    return P * L ** 3 / (3 * E_MM * I) + P * L / (KAPPA * G_MM * w * h)


def crossing(load=-50.0, pull=0.0, mu=0.35, freeB=True, nseg=10, L=1000.0, h=30.0, locked=False, local=False, roll=(0.0, 0.0),
             pin=False, **prm):
    P = np.array([[-L / 2 + L * i / nseg, 0.0, 0.0] for i in range(nseg + 1)])
    PB = np.array([[0.0, -L / 2 + L * i / nseg, h] for i in range(nseg + 1)])
    mid = nseg // 2
    fixA = ws.mask(1, 1, 1, 0, 0, 1)
    fixB = ws.mask(0, 1, 1, 0, 0, 1) if freeB else fixA
    prm.setdefault("max_iter", 20000)
    # section normals: z, rolled by roll[s] radians about the lath's own axis (A runs along x, B along y)
    nA = np.tile([0.0, -math.sin(roll[0]), math.cos(roll[0])], (nseg + 1, 1))
    nB = np.tile([math.sin(roll[1]), 0.0, math.cos(roll[1])], (nseg + 1, 1))
    md = ws.polylines([P, PB], normals=[nA, nB], knot_rows=[[0, mid, nseg], [0, mid, nseg]], knots=[((0, 1), (1, 1))],
                      anchors=[((0, 0), fixA), ((0, 2), fixA), ((1, 0), fixB), ((1, 2), fixB)] + ([((0, 1), fixA)] if pin else []),
                      loads=[((1, 1), (pull, 0.0, load), local)], mu=mu, E=E_MM, G=G_MM, params=mm_params(**prm))
    if locked:
        md.cross_locked[:] = 1
    md.roll = roll
    return md


def torsion(nseg=10, L=1000.0):
    normals = [[0.0, -math.sin(math.pi / 2 * i / nseg), math.cos(math.pi / 2 * i / nseg)] for i in range(nseg + 1)]
    md = straight(L, nseg, normals=normals, anchors=[((0, 0), ws.mask(1, 1, 1, 1, 1, 1)), ((0, 1), ws.mask(1, 1, 1, 0, 0, 1))],
                  params=mm_params(contacts=0, max_iter=20000))
    return md


def case_by_name(name):
    if name in ("cantilever", "cantilever_edge"):
        return cantilever(10, 2 if name == "cantilever" else 1, tol=1e-4, max_iter=20000)
    if name == "torsion":
        return torsion()
    pulls = {"cross_press": 0.0, "cross_stick": 5.0, "cross_slip": 12.0, "cross_locked": 12.0}
    if name in pulls:
        return crossing(-50.0, pulls[name], locked=name == "cross_locked")
    if name == "cross_w23":      # W2 rotational friction + W3 seat law, seats from the start (cases.mjs:48)
        return crossing(-50.0, 5.0, rot_friction=1, seat_law=1, dent_after_iter=0, slip_rate=0.3)
    if name == "cross_al":       # augmented-Lagrangian gap (browser_cases.js:45)
        return crossing(-50.0, 0.0, augmented=1, al_every=600, strength=2000.0)
    raise KeyError(name)


def max_rel_disp_error(Xa, Xb, X0):
    """largest |ΔX| against the largest displacement (selftest.html:53-56), floored at 1e-9 × model size"""
    d = np.abs(Xa - X0).max()
    s = np.abs(X0).max()
    return np.abs(Xa - Xb).max() / max(d, 1e-9 * s, 1e-300)


def max_node_err_span(Xa, Xb, span):
    """max over nodes of |X_a − X_b|₂ / span"""
    return float(np.linalg.norm((Xa - Xb).reshape(-1, 3), axis=1).max() / span)


def utm_beam(mode, sched, nseg=10, settle=10 ** 6, avg=10, tol=1e-8, max_iter=2_000_000):
    """three-point bending under the load protocol: a 1000 mm lath pinned at one end and on a roller at the other
    (twist held at both), the probe at mid-span along −z; force (mode 1) or travel (mode 2) per increment"""
    md = straight(1000.0, nseg, anchors=[((0, 0), ws.mask(1, 1, 1, 0, 0, 1)), ((0, 1), ws.mask(0, 1, 1, 0, 0, 1))],
                  params=mm_params(contacts=0, max_iter=max_iter, tol=tol))
    md.protocol = dict(mode=mode, probe=nseg // 2, sched=list(sched), settle=settle, avg=avg, axis=(0.0, 0.0, -1.0))
    return md


def beam_midspan_stiffness(L=1000.0, w=60.0, h=30.0):
    """Timoshenko: P / δ of a simply supported beam under a mid-span load (bending about the 60 mm face)"""
    I = w * h ** 3 / 12
    return 1.0 / (L ** 3 / (48 * E_MM * I) + L / (4 * KAPPA * G_MM * w * h))


def ground_beam(pull=0.0, q=10.0, mu=0.5, nseg=10, L=1000.0, **prm):
    """a 1000 mm lath lying on the ground (scene.floor at its underside, z = −15) under 10 N down at every node, held
    only in y and against twist at one end (the ground carries it); `pull` along x at the free end"""
    prm.setdefault("max_iter", 20000)
    md = straight(L, nseg, anchors=[((0, 0), ws.mask(0, 1, 0, 0, 0, 1))],
                  params=mm_params(contacts=0, floor=1, floor_z=-15.0, floor_mu=mu, **prm))
    md.load_const[2::3] -= q
    md.load_const[3 * nseg] += pull
    md.node_w = np.full(md.n, 60.0)
    md.node_h = np.full(md.n, 30.0)
    return md


def permute_nodes(md, seed=0):
    """The same model with its nodes renumbered by a seeded permutation (node i becomes perm[i]): every node-indexed
    array reordered and every node index remapped.  Strands then no longer number their nodes consecutively, so the
    solver gathers a crossing side's nodes instead of computing them.  Returns (model, perm)."""
    perm = np.random.default_rng(seed).permutation(md.n).astype(np.int32)
    p = md.copy()

    def reorder(a, width):
        if a is None or a.size == 0:
            return a
        b = np.empty_like(a).reshape(md.n, width)
        b[perm] = a.reshape(md.n, width)
        return b.reshape(-1)
    for k in ("X", "X0", "load_const"):
        setattr(p, k, reorder(getattr(md, k), 3))
    for k in ("node_w", "node_h"):
        setattr(p, k, reorder(getattr(md, k), 1))
    for k in ("seg_i0", "seg_i1", "local_load_node", "anchor_node"):
        a = getattr(md, k)
        if a is not None and a.size:
            setattr(p, k, perm[a].astype(np.int32))
    if md.protocol:
        p.protocol = dict(md.protocol, probe=int(perm[md.protocol["probe"]]))
    p.node_offset = None
    return p, perm


def unpermute(X, perm):
    """node positions of a permuted model back in the original numbering"""
    return X.reshape(-1, 3)[perm].reshape(-1)


def record(name, data):
    """append one named result (a JSON line) to the file WEAVESIM_PARITY_RECORD names, when it is set: the raw numbers
    behind the tolerances of the parity tests"""
    path = os.environ.get("WEAVESIM_PARITY_RECORD")
    if not path:
        return
    with open(path, "a") as f:
        f.write(json.dumps({"test": name, **data}) + "\n")


def ground_only(tilt=0.0, drop=5.0, q=10.0, nseg=10, L=1000.0, mu=0.5, **prm):
    """a 1000 mm lath that only the ground holds (no anchor): its underside starts `drop` mm above the ground at the
    first node, and `drop + tilt` mm above it at the last; 10 N down at every node (solver_cpu.js:520-533: the
    rigid-body freedoms carry it down, level it and bring it to rest)"""
    prm.setdefault("max_iter", 60000)
    md = straight(L, nseg, params=mm_params(contacts=0, floor=1, floor_z=-15.0 - drop, floor_mu=mu, **prm))
    md.X[2::3] += tilt * md.X[0::3] / L
    md.X0 = md.X.copy()
    md.load_const[2::3] -= q
    md.node_w = np.full(md.n, 60.0)
    md.node_h = np.full(md.n, 30.0)
    return md

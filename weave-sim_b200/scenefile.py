"""scene.json reader: a model from a scene file of the reference and its mesh.

Follows the reference's reading path: Scene.fromJSON (web/js/scene.js:142-190) for the parameters and their defaults
(web/js/params.js:6-25), Mesh.fromBytes (web/js/mesh.js:23-31, 62-125) for the STL / OBJ file, the vertex weld and the
scale, UnitSystem (web/js/units.js) for the self-weight, sectionStiffness / beamFactors / beamActivations
(params.js:43-57) for the laths; the topology, the anchors' selectors and the loads are built by the library
(ws_scene_mesh).  Supported: lath groups by strand (a hybrid weave: each group's material, section and beam for its
strands' segments, joints, crossing sides, nodes, self-weight and knot offsets), selectors frame / all_start / all_end /
all_ends / strand / knots / boundary, loads gravity / udl per length or per area / point (world or local), the ground,
every contact and solver parameter the solver has.  Anything else (lath groups by piece of a discretisation, the region
selector) raises NotImplementedError rather than being ignored.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import re
import struct

import numpy as np

from . import _lib
from ._lib import Model, check, default_params, lib

LENGTH_TO_M = {"mm": 1e-3, "cm": 1e-2, "m": 1.0}
FORCE_TO_N = {"N": 1.0, "kN": 1e3}
G_SI = 9.80665
MATERIAL = {"E": 10000.0, "G": 625.0, "density": 700.0, "E90": 800.0, "fc90": 8.0, "H": 30.0}
SECTION = {"width": 60.0, "height": 30.0, "Ix": None, "Iy": None, "J": None}
CONTACT = {"mu": 0.35, "strength": 1e4, "stick_strength": 1e4, "torsion_factor": 1.0, "epsilon": 15.0, "ramp_iter": 1500,
           "slip_rate": 1.0, "locked": False, "rot_friction": False, "rot_factor": 1.0, "seat_law": "off", "seat_gap": True,
           "dent_rate": 0.01, "dent_after_iter": -1, "edge_threshold": 0.5, "augmented": False, "al_every": 600}
BEAM = {"mode": "simple", "activation": 1.0, "stiffness": 1.0, "activation_flat": 1.0, "activation_edge": 1.0,
        "activation_twist": 1.0, "stiffness_flat": 1.0, "stiffness_edge": 1.0, "stiffness_twist": 1.0,
        "stiffness_axial": 1.0, "stiffness_shear": 1.0}
SOLVER = {"max_iter": 5000, "tol": 1e-4, "damping": 1.0, "kinetic_damping": True, "mass_scale": 1.5, "warmup_iter": 300,
          "prestress": "flat"}
WEAVE = {"subdivisions": 4, "overhang": 0.0, "offset_mode": "half_height", "flip_knots": [], "seed_strand_phase": 0}
FLOOR_MU = 0.4
SELECTORS = {"frame": 0, "all_start": 1, "all_end": 2, "all_ends": 3, "strand": 4, "boundary": 5}


class WsMeshCfg(C.Structure):
    _fields_ = [("n_vertices", C.c_int32), ("n_faces", C.c_int32), ("vertices", _lib._dp), ("faces", _lib._ip),
                ("subdivisions", C.c_int32), ("half_height", C.c_int32), ("seed_strand_phase", C.c_int32),
                ("n_flips", C.c_int32), ("flips", _lib._ip), ("overhang", C.c_double), ("width", C.c_double),
                ("height", C.c_double), ("EA", C.c_double), ("EIx", C.c_double), ("EIy", C.c_double), ("GJ", C.c_double),
                ("GA", C.c_double), ("activation", C.c_double * 3), ("line_weight", C.c_double),
                ("gravity_dir", C.c_double * 3), ("udl_on", C.c_int32), ("pad0", C.c_int32), ("udl", C.c_double * 3),
                ("mu", C.c_double), ("fc90", C.c_double), ("E90", C.c_double), ("H", C.c_double),
                ("n_anchors", C.c_int32), ("pad1", C.c_int32), ("anchor_kind", _lib._ip), ("anchor_id", _lib._ip),
                ("anchor_mask", _lib._bp), ("n_loads", C.c_int32), ("pad2", C.c_int32), ("load_frames", _lib._ip),
                ("load_F", _lib._dp), ("load_local", _lib._bp), ("params", _lib.WsParams),
                ("n_groups", C.c_int32), ("n_assign", C.c_int32), ("groups", C.c_void_p),
                ("assign_strand", _lib._ip), ("assign_group", _lib._ip)]


class WsLathGroup(C.Structure):
    _fields_ = [("width", C.c_double), ("height", C.c_double), ("EA", C.c_double), ("EIx", C.c_double),
                ("EIy", C.c_double), ("GJ", C.c_double), ("GA", C.c_double), ("activation", C.c_double * 3),
                ("line_weight", C.c_double), ("fc90", C.c_double), ("E90", C.c_double), ("H", C.c_double)]


def _defaults(defaults, d):
    """fromDict (params.js:27-31): the defaults, overridden by the known keys of d"""
    out = dict(defaults)
    for k in defaults:
        if d and k in d and d[k] is not None:
            out[k] = d[k]
    return out


# ---------------------------------------------------------------------------------------------------- mesh files
def parse_stl(buf: bytes):
    """triangles of a binary or ASCII STL (parseSTL, mesh.js:62-86): unwelded vertices, faces 3t, 3t+1, 3t+2"""
    if len(buf) >= 84:
        n = struct.unpack_from("<I", buf, 80)[0]
        if 84 + 50 * n == len(buf):
            rec = np.frombuffer(buf, dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", 9), ("a", "<u2")]), count=n, offset=84)
            V = rec["v"].astype(np.float64).ravel()
            return V, np.arange(3 * n, dtype=np.int32)
    vals = [float(x) for m in re.finditer(r"vertex\s+([-+0-9.eE]+)\s+([-+0-9.eE]+)\s+([-+0-9.eE]+)", buf.decode("latin-1"))
            for x in m.groups()]
    nt = len(vals) // 9
    if not nt:
        raise ValueError("no triangles found (binary or ASCII STL expected)")
    return np.array(vals[:9 * nt], dtype=np.float64), np.arange(3 * nt, dtype=np.int32)


def parse_obj(text: str):
    """vertices and fan-triangulated faces of an OBJ file (parseOBJ, mesh.js:88-103)"""
    V, F = [], []
    for raw in text.splitlines():
        line = raw.strip()
        if line.startswith("v "):
            p = line.split()
            V.extend(float(x) for x in p[1:4])
        elif line.startswith("f "):
            nv = len(V) // 3
            idx = [(nv + int(t.split("/")[0])) if int(t.split("/")[0]) < 0 else int(t.split("/")[0]) - 1 for t in line.split()[1:]]
            for k in range(1, len(idx) - 1):
                F.extend((idx[0], idx[k], idx[k + 1]))
    if not F:
        raise ValueError("no faces in the OBJ file")
    return np.array(V, dtype=np.float64), np.array(F, dtype=np.int32)


def weld(V, F, tol=1e-9):
    """merge duplicated vertices (weld, mesh.js:106-125): coordinates quantised at tol × the model size (rounded half to
    even), unique rows in lexicographic order, the first occurrence kept; faces that collapse are dropped"""
    P = np.asarray(V, dtype=np.float64).reshape(-1, 3)
    if not len(P):
        return V, F
    q = max(float(np.ptp(P, axis=0).max()), 1.0) * tol
    key = np.round(P / q)                          # numpy rounds half to even
    order = np.lexsort((np.arange(len(P)), key[:, 2], key[:, 1], key[:, 0]))
    ks = key[order]
    new = np.ones(len(P), dtype=bool)
    new[1:] = np.any(ks[1:] != ks[:-1], axis=1)
    uid = np.cumsum(new) - 1
    inv = np.empty(len(P), dtype=np.int64)
    inv[order] = uid
    first = order[new]
    Fw = inv[np.asarray(F, dtype=np.int64).reshape(-1, 3)]
    keep = (Fw[:, 0] != Fw[:, 1]) & (Fw[:, 1] != Fw[:, 2]) & (Fw[:, 0] != Fw[:, 2])
    return P[first].ravel().copy(), Fw[keep].astype(np.int32).ravel()


def read_mesh(path, scale=1.0):
    """Mesh.fromBytes (mesh.js:23-31): parse, scale, weld; an .npz holds a mesh already welded (arrays V, F)"""
    if path.lower().endswith(".npz"):
        z = np.load(path)
        return np.asarray(z["V"], dtype=np.float64) * float(scale), np.asarray(z["F"], dtype=np.int32)
    with open(path, "rb") as f:
        buf = f.read()
    V, F = parse_obj(buf.decode("utf-8", "replace")) if path.lower().endswith(".obj") else parse_stl(buf)
    return weld(V * float(scale), F)


# ---------------------------------------------------------------------------------------------------- scene
def _rect_torsion(a, b):
    if a < b:
        a, b = b, a
    r = b / a
    return a * b ** 3 * (1.0 / 3.0 - 0.21 * r * (1.0 - r ** 4 / 12.0))


def _lath_group(mat, sec, beam, prestress, line_factor):
    """one lath group's section, stiffness, prestress shares, self-weight per length and material across the grain:
    sectionStiffness x beamFactors and beamActivations (params.js:43-57), UnitSystem.selfWeightLineLoad (units.js:21-25);
    line_factor converts density x area to the self-weight per length in scene units (0: gravity off)"""
    w, h = float(sec["width"]), float(sec["height"])
    A = w * h
    Ix = sec["Ix"] if sec["Ix"] is not None else w * h ** 3 / 12.0
    Iy = sec["Iy"] if sec["Iy"] is not None else h * w ** 3 / 12.0
    J = sec["J"] if sec["J"] is not None else _rect_torsion(w, h)
    if beam["mode"] == "advanced":
        fEA, fIx, fIy, fGJ, fGA = (float(beam[k]) for k in ("stiffness_axial", "stiffness_flat", "stiffness_edge",
                                                             "stiffness_twist", "stiffness_shear"))
        act = [beam["activation_flat"], beam["activation_edge"], beam["activation_twist"]]
    else:
        k = float(beam["stiffness"])
        fEA, fIx, fIy, fGJ, fGA = 1.0, k, k, k, 1.0
        act = [beam["activation"]] * 3
    if prestress == "asbuilt":                      # rod_cosserat.js:59: no prestress share at all
        act = [0.0, 0.0, 0.0]
    act = [min(max(float(a), 0.0), 1.0) for a in act]
    E, G = float(mat["E"]), float(mat["G"])
    g = WsLathGroup()
    g.width, g.height = w, h
    g.EA, g.EIx, g.EIy, g.GJ, g.GA = E * A * fEA, E * Ix * fIx, E * Iy * fIy, G * J * fGJ, 5.0 / 6.0 * G * A * fGA
    for k in range(3):
        g.activation[k] = act[k]
    g.line_weight = float(mat["density"]) * A * line_factor
    g.fc90, g.E90, g.H = float(mat["fc90"]), float(mat["E90"]), float(mat["H"])
    return g


def load_scene(path, mesh_path=None) -> Model:
    """A model of the scene file `path` (its mesh path taken relative to the file, or `mesh_path`)."""
    with open(path) as f:
        d = json.load(f)
    if (d.get("version", 1) or 1) > 1:
        raise ValueError(f"scene version {d['version']} newer than supported 1")
    units = d.get("units") or {}
    L = LENGTH_TO_M[units.get("length", "mm")]
    Fu = FORCE_TO_N[units.get("force", "N")]
    mesh = d.get("mesh") or {}
    mp = mesh_path or os.path.join(os.path.dirname(os.path.abspath(path)), mesh.get("path", ""))
    V, F = read_mesh(mp, float(mesh.get("scale", 1.0) or 1.0))
    weave = _defaults(WEAVE, d.get("weave"))
    mat = _defaults(MATERIAL, d.get("material"))
    md_ = d.get("material") or {}
    stress = (1.0 / (1e-3 * 1e-3)) / (Fu / (L * L))      # N/mm² → scene stress (older scenes: defaults in N/mm²)
    for k in ("E90", "fc90", "H"):
        if k not in md_:
            mat[k] = MATERIAL[k] * stress
    sec = _defaults(SECTION, d.get("section"))
    beam = _defaults(BEAM, d.get("beam"))
    contact = _defaults(CONTACT, d.get("contact"))
    solver = _defaults(SOLVER, d.get("solver"))
    loads = d.get("loads") or {}
    grav = loads.get("gravity") or {}
    line_factor = L * L * G_SI / Fu * L if grav.get("enabled", True) else 0.0     # UnitSystem.selfWeightLineLoad
    # lath groups (Scene.fromJSON, scene.js:170-176; group(g), strandGroup(s), scene.js:51-62): group 1 is the scene's
    # own material, section and beam; groups 2.. come from hybrid.groups, their materials without the older-scene
    # conversion; a strand's group from hybrid.assign
    hyb = d.get("hybrid") or {}
    groups, assign = [], []
    if hyb.get("enabled"):
        if any(v for v in (hyb.get("pieces") or {}).values()):
            raise NotImplementedError("lath groups by piece of a discretisation (hybrid.pieces)")
        raw = hyb.get("groups") or []
        groups = [_lath_group(_defaults(MATERIAL, g.get("material")), _defaults(SECTION, g.get("section")),
                              _defaults(BEAM, g.get("beam")), solver["prestress"], line_factor) for g in raw]
        for k, v in (hyb.get("assign") or {}).items():
            gi = int(v)
            if 2 <= gi <= 1 + len(groups):
                assign.append((int(k), gi))
    base = _lath_group(mat, sec, beam, solver["prestress"], line_factor)
    w, h = base.width, base.height
    cfg = WsMeshCfg()
    keep = []

    def arr(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a.ctypes.data_as(C.POINTER({np.float64: C.c_double, np.int32: C.c_int32, np.uint8: C.c_uint8}[dt]))

    cfg.n_vertices, cfg.n_faces = len(V) // 3, len(F) // 3
    cfg.vertices, cfg.faces = arr(V, np.float64), arr(F, np.int32)
    cfg.subdivisions = int(weave["subdivisions"])
    cfg.half_height = 1 if weave["offset_mode"] == "half_height" else 0
    cfg.seed_strand_phase = int(weave["seed_strand_phase"])
    flips = np.array([[int(a), int(b)] for a, b in weave["flip_knots"]], dtype=np.int32).reshape(-1, 2)
    cfg.n_flips, cfg.flips = len(flips), arr(flips.ravel(), np.int32)
    cfg.overhang = float(weave["overhang"])
    cfg.width, cfg.height = w, h
    cfg.EA, cfg.EIx, cfg.EIy, cfg.GJ, cfg.GA = base.EA, base.EIx, base.EIy, base.GJ, base.GA
    for k in range(3):
        cfg.activation[k] = base.activation[k]
    cfg.line_weight = base.line_weight
    if grav.get("enabled", True):
        gd = grav.get("direction") or [0.0, 0.0, -1.0]
        for k in range(3):
            cfg.gravity_dir[k] = float(gd[k])
    udl = loads.get("udl") or {}
    if udl.get("enabled"):
        per = udl.get("per", "length")
        if per not in ("length", "area"):
            raise ValueError(f"udl per {per}")
        cfg.udl_on = 1 if per == "length" else 2
        for k in range(3):
            cfg.udl[k] = float(udl["q"][k])
    cfg.mu = float(contact["mu"])
    cfg.fc90, cfg.E90, cfg.H = base.fc90, base.E90, base.H
    if groups:
        garr = (WsLathGroup * len(groups))(*groups)
        keep.append(garr)
        cfg.n_groups = len(groups)
        cfg.groups = C.cast(garr, C.c_void_p)
        cfg.n_assign = len(assign)
        cfg.assign_strand = arr(np.array([a for a, _ in assign], dtype=np.int32), np.int32)
        cfg.assign_group = arr(np.array([g for _, g in assign], dtype=np.int32), np.int32)
    kinds, ids, masks = [], [], []
    for a in d.get("anchors") or []:
        sel = a.get("select") or {}
        t = sel.get("type", "frame")
        fix = a.get("fix") or [1, 1, 1, 0, 0, 0]
        m = sum(1 << i for i, f in enumerate(fix) if f)
        if t == "knots":
            for s, kk in sel.get("ids") or []:
                kinds.append(0); ids.append((int(s), int(kk))); masks.append(m)
        elif t in SELECTORS:
            kinds.append(SELECTORS[t])
            ids.append(tuple(int(x) for x in sel["id"]) if t == "frame" else (int(sel.get("strand", 0)), 0))
            masks.append(m)
        else:
            raise NotImplementedError(f"anchor selector {t}")
    cfg.n_anchors = len(kinds)
    cfg.anchor_kind = arr(np.array(kinds, dtype=np.int32), np.int32)
    cfg.anchor_id = arr(np.array(ids, dtype=np.int32).reshape(-1, 2).ravel(), np.int32)
    cfg.anchor_mask = arr(np.array(masks, dtype=np.uint8), np.uint8)
    pts = loads.get("point") or []
    cfg.n_loads = len(pts)
    cfg.load_frames = arr(np.array([[int(p["frame"][0]), int(p["frame"][1])] for p in pts], dtype=np.int32).reshape(-1, 2).ravel(), np.int32)
    cfg.load_F = arr(np.array([[float(x) for x in p["F"]] for p in pts], dtype=np.float64).reshape(-1, 3).ravel(), np.float64)
    cfg.load_local = arr(np.array([1 if p.get("space", "world") == "local" else 0 for p in pts], dtype=np.uint8), np.uint8)
    prm = default_params(
        mass_scale=float(solver["mass_scale"]), damping=float(solver["damping"]), tol=float(solver["tol"]),
        kinetic_damping=int(bool(solver["kinetic_damping"])), warmup_iter=int(solver["warmup_iter"]),
        max_iter=int(solver["max_iter"]), strength=float(contact["strength"]),
        stick_strength=float(contact["stick_strength"]), torsion_factor=float(contact["torsion_factor"]),
        epsilon=float(contact["epsilon"]), ramp_iter=int(contact["ramp_iter"]), slip_rate=float(contact["slip_rate"]),
        edge_threshold=float(contact["edge_threshold"]), augmented=int(bool(contact["augmented"])),
        al_every=int(contact["al_every"]), rot_friction=int(bool(contact["rot_friction"])),
        rot_factor=float(contact["rot_factor"]), seat_law=0 if contact["seat_law"] == "off" else 1,
        seat_gap=int(bool(contact["seat_gap"])), dent_rate=float(contact["dent_rate"]),
        dent_after_iter=int(contact["dent_after_iter"]))
    fl = d.get("floor") or {}
    fz = fl.get("z")
    if fl.get("enabled") and fz is not None:
        fmu = fl.get("mu")
        prm.update(floor=1, floor_z=float(fz), floor_mu=float(fmu) if fmu is not None and float(fmu) >= 0 else FLOOR_MU)
    cfg.params = _lib.params_struct(prm)
    sc = C.c_void_p()
    L_ = lib()
    L_.ws_scene_mesh.argtypes = [C.POINTER(WsMeshCfg), C.POINTER(C.c_void_p)]
    check(L_.ws_scene_mesh(C.byref(cfg), C.byref(sc)), "ws_scene_mesh")
    model = _lib._from_scene(sc)
    if contact["locked"]:
        model.cross_locked[:] = 1
    return model

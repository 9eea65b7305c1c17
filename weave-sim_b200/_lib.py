"""ctypes binding of libweavesim_b200.so (the C ABI declared in include/weavesim.h).

The library is built in-tree (``weave-sim_b200/csrc/Makefile``).  There is no fallback: if the shared library is
missing, importing the solver raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("WEAVESIM_B200_LIB") or os.path.join(HERE, "libweavesim_b200.so")

WS_OK = 0
WS_PREC_F64, WS_PREC_MIXED, WS_PREC_F32 = 0, 1, 2
WS_FORM_CTA, WS_FORM_GRID, WS_FORM_PLAIN = 0, 1, 2
WS_RUNNING, WS_CONVERGED, WS_MAX_ITER, WS_NONFINITE = 0, 1, 2, 3
PRECISIONS = {"f64": WS_PREC_F64, "mixed": WS_PREC_MIXED, "f32": WS_PREC_F32}
FORMS = {"cta": WS_FORM_CTA, "grid": WS_FORM_GRID, "plain": WS_FORM_PLAIN}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_bp = C.POINTER(C.c_uint8)


class WsParams(C.Structure):
    _fields_ = [("mass_scale", C.c_double), ("damping", C.c_double), ("tol", C.c_double),
                ("kinetic_damping", C.c_int32), ("warmup_iter", C.c_int32), ("max_iter", C.c_int32),
                ("contacts", C.c_int32), ("strength", C.c_double), ("stick_strength", C.c_double),
                ("torsion_factor", C.c_double), ("epsilon", C.c_double), ("ramp_iter", C.c_int32),
                ("disp_ramp_iter", C.c_int32), ("slip_rate", C.c_double), ("edge_threshold", C.c_double),
                ("augmented", C.c_int32), ("al_every", C.c_int32), ("rot_friction", C.c_int32), ("seat_law", C.c_int32),
                ("seat_gap", C.c_int32), ("dent_after_iter", C.c_int32), ("rot_factor", C.c_double), ("dent_rate", C.c_double),
                ("floor", C.c_int32), ("pad1", C.c_int32), ("floor_z", C.c_double), ("floor_mu", C.c_double)]


PARAM_KEYS = [f[0] for f in WsParams._fields_ if not f[0].startswith("pad")]


PROTOCOL_MAX_INC = 64


class WsProtocol(C.Structure):
    _fields_ = [("mode", C.c_int32), ("probe", C.c_int32), ("n_inc", C.c_int32), ("settle", C.c_int32),
                ("avg", C.c_int32), ("pad0", C.c_int32), ("axis", C.c_double * 3),
                ("sched", C.c_double * PROTOCOL_MAX_INC)]


class WsModel(C.Structure):
    _fields_ = [("n", C.c_int32), ("m", C.c_int32), ("p", C.c_int32), ("n_strands", C.c_int32), ("K", C.c_int32),
                ("pad0", C.c_int32),
                ("X", _dp), ("X0", _dp), ("Q", _dp), ("l0", _dp), ("seg_i0", _ip), ("seg_i1", _ip), ("seg_offset", _ip),
                ("joint_seg0", _ip), ("joint_seg1", _ip), ("joint_len", _dp), ("omega0", _dp),
                ("EA", _dp), ("EIx", _dp), ("EIy", _dp), ("GJ", _dp), ("GA", _dp), ("load_const", _dp),
                ("n_local_loads", C.c_int32), ("n_anchors", C.c_int32),
                ("local_load_node", _ip), ("local_load_F", _dp), ("anchor_node", _ip), ("anchor_mask", _bp),
                ("anchor_target", _dp),
                ("cross_strand", _ip), ("cross_wk", _dp), ("cross_hk", _dp), ("cross_u", _dp), ("cross_nprev", _dp),
                ("cross_enabled", _bp), ("cross_locked", _bp), ("cross_mu", _dp),
                ("cross_fc90", _dp), ("cross_E90", _dp), ("cross_H", _dp), ("params", WsParams),
                ("protocol", C.POINTER(WsProtocol)), ("node_w", _dp), ("node_h", _dp)]


class WsKagomeCfg(C.Structure):
    _fields_ = [("side", C.c_int32), ("subdivisions", C.c_int32), ("edge", C.c_double), ("width", C.c_double),
                ("height", C.c_double), ("E", C.c_double), ("G", C.c_double), ("density", C.c_double),
                ("mu", C.c_double), ("mu_lo", C.c_double), ("mu_hi", C.c_double), ("inward", C.c_double),
                ("lift", C.c_double), ("z_noise", C.c_double), ("gravity", C.c_int32), ("seed", C.c_uint32),
                ("params", WsParams)]


class WsPolylineCfg(C.Structure):
    _fields_ = [("n_strands", C.c_int32), ("node_count", _ip), ("points", _dp), ("normals", _dp),
                ("knot_count", _ip), ("knot_rows", _ip), ("n_knots", C.c_int32), ("knots", _ip),
                ("thickness", C.c_double), ("n_anchors", C.c_int32), ("anchor_frames", _ip), ("anchor_masks", _bp),
                ("n_loads", C.c_int32), ("load_frames", _ip), ("load_F", _dp), ("load_local", _bp),
                ("width", C.c_double), ("height", C.c_double), ("E", C.c_double), ("G", C.c_double),
                ("density", C.c_double), ("mu", C.c_double), ("gravity", C.c_int32), ("params", WsParams)]


class WsControl(C.Structure):
    _fields_ = [("iter", C.c_int32), ("status", C.c_int32), ("rollbacks", C.c_int32), ("pending_zero", C.c_int32),
                ("ke", C.c_double), ("ke_prev", C.c_double), ("residual", C.c_double), ("res_force", C.c_double),
                ("res_torque", C.c_double), ("fref", C.c_double), ("e_stretch", C.c_double), ("e_shear", C.c_double),
                ("e_bend", C.c_double), ("e_twist", C.c_double), ("e_contact", C.c_double),
                ("utm_inc", C.c_int32), ("utm_phase", C.c_int32), ("e_floor", C.c_double),
                ("t_start_ms", C.c_double), ("t_end_ms", C.c_double)]

    def as_dict(self):
        return {f[0]: getattr(self, f[0]) for f in self._fields_}


class WsOpts(C.Structure):
    _fields_ = [("precision", C.c_int32), ("form", C.c_int32), ("threads", C.c_int32), ("device", C.c_int32),
                ("budget_bytes", C.c_uint64), ("cta_state", C.c_int32), ("side_order", C.c_int32),
                ("wide_cluster", C.c_int32), ("wide_min", C.c_int32), ("tune", C.c_int32)]


class WsShape(C.Structure):
    _fields_ = [(k, C.c_int32) for k in ("threads", "cta_state", "wide_cluster", "wide_min", "plain_launch", "source",
                                         "trials", "pad0")] + [("trial_ms", C.c_double), ("default_ms", C.c_double)]

    SOURCES = {0: "options", 1: "tuned", 2: "cache"}

    def as_dict(self):
        d = {f[0]: getattr(self, f[0]) for f in self._fields_ if f[0] != "pad0"}
        d["source"] = self.SOURCES.get(d["source"], d["source"])
        return d


class WsStateOut(C.Structure):
    _fields_ = [(k, _dp) for k in ("X", "Q", "V", "W", "u", "nprev", "slip")] + \
               [("stuck", _bp), ("state", _bp)] + \
               [(k, _dp) for k in ("Fn", "Ft", "gap", "N", "Vsh", "M", "reactions")] + \
               [("ctype", _bp)] + [(k, _dp) for k in ("theta", "phi", "area", "pressure", "util")] + \
               [(k, _dp) for k in ("lambda", "dent", "M_rot", "rot_slip", "utm", "floor_F")] + [("floor_state", _bp)] + \
               [(k, _dp) for k in ("seg_M", "node_M", "disp")]


_lib = None


def lib():
    """The loaded library (raises when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C weave-sim_b200/csrc` "
                               "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        L.ws_last_error.argtypes = [C.c_char_p, C.c_size_t]
        L.ws_params_default.argtypes = [C.POINTER(WsParams)]
        L.ws_scene_kagome.argtypes = [C.POINTER(WsKagomeCfg), C.POINTER(C.c_void_p)]
        L.ws_scene_polylines.argtypes = [C.POINTER(WsPolylineCfg), C.POINTER(C.c_void_p)]
        L.ws_scene_model.argtypes = [C.c_void_p]
        L.ws_scene_model.restype = C.POINTER(WsModel)
        L.ws_scene_node_offset.argtypes = [C.c_void_p]
        L.ws_scene_node_offset.restype = _ip
        L.ws_scene_span.argtypes = [C.c_void_p]
        L.ws_scene_span.restype = C.c_double
        L.ws_scene_free.argtypes = [C.c_void_p]
        L.ws_model_goals.argtypes = [C.POINTER(WsModel), _dp, _dp, _dp, _dp, _dp]
        if hasattr(L, "ws_device_count"):
            L.ws_device_count.restype = C.c_int
        if hasattr(L, "ws_create"):
            L.ws_create.argtypes = [C.POINTER(C.POINTER(WsModel)), C.c_int32, C.POINTER(WsOpts), C.POINTER(C.c_void_p)]
            L.ws_step.argtypes = [C.c_void_p, C.c_int32, _bp, C.POINTER(WsControl)]
            L.ws_read_control.argtypes = [C.c_void_p, C.POINTER(WsControl)]
            L.ws_download.argtypes = [C.c_void_p, C.c_int32, C.POINTER(WsStateOut)]
            L.ws_upload_state.argtypes = [C.c_void_p, C.c_int32, _dp, _dp, _dp]
            L.ws_set_params.argtypes = [C.c_void_p, C.c_int32, C.POINTER(WsModel)]
            L.ws_internalize.argtypes = [C.c_void_p, C.c_int32]
            L.ws_load_instance.argtypes = [C.c_void_p, C.c_int32, C.POINTER(WsModel)]
            L.ws_relax_noalloc.argtypes = [C.POINTER(WsModel), C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                                           C.POINTER(WsStateOut), C.POINTER(WsControl)]
            L.ws_stream.argtypes = [C.c_void_p]
            L.ws_stream.restype = C.c_void_p
            L.ws_cta_resident.argtypes = [C.c_void_p]
            L.ws_cta_resident.restype = C.c_int
            L.ws_wide_instances.argtypes = [C.c_void_p, C.POINTER(C.c_int32)]
            L.ws_wide_instances.restype = C.c_int
            L.ws_get_shape.argtypes = [C.c_void_p, C.POINTER(WsShape)]
            L.ws_tune_key.argtypes = [C.POINTER(C.POINTER(WsModel)), C.c_int32, C.POINTER(WsOpts), C.c_char_p,
                                      C.c_char_p, C.c_size_t]
            L.ws_tune_candidates.argtypes = [C.POINTER(C.POINTER(WsModel)), C.c_int32, C.POINTER(WsOpts),
                                             C.POINTER(WsShape), C.POINTER(WsShape), C.c_int32]
            L.ws_tune_cache_get.argtypes = [C.c_char_p, C.POINTER(WsShape)]
            L.ws_tune_cache_put.argtypes = [C.c_char_p, C.POINTER(WsShape)]
            L.ws_side_order.argtypes = [C.c_void_p]
            L.ws_side_order.restype = C.c_int
            L.ws_device_bytes.argtypes = [C.c_void_p]
            L.ws_device_bytes.restype = C.c_uint64
            L.ws_last_step_stats.argtypes = [C.c_void_p, _dp, C.POINTER(C.c_int64)]
            L.ws_destroy.argtypes = [C.c_void_p]
        _lib = L
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(2048)
    lib().ws_last_error(buf, 2048)
    return buf.value.decode(errors="replace")


def check(rc: int, what: str):
    if rc != WS_OK:
        raise RuntimeError(f"{what} failed ({rc}): {last_error()}")


def default_params(**over) -> dict:
    p = WsParams()
    lib().ws_params_default(C.byref(p))
    d = {k: getattr(p, k) for k in PARAM_KEYS}
    for k, v in over.items():
        if k not in d:
            raise KeyError(f"unknown parameter {k}")
        d[k] = v
    return d


def params_struct(d: dict) -> WsParams:
    p = WsParams()
    for k in PARAM_KEYS:
        setattr(p, k, d[k])
    return p


def _ptr(a, ct):
    return None if a is None else a.ctypes.data_as(C.POINTER(ct))


class Model:
    """Host copy of a ws_model: numpy arrays that tests, benchmarks and the serving loop can edit before a solver is
    built from them (loads, anchors, stiffness, parameters)."""

    FLOAT = ("X", "X0", "Q", "l0", "joint_len", "omega0", "EA", "EIx", "EIy", "GJ", "GA", "load_const",
             "local_load_F", "cross_wk", "cross_hk", "cross_u", "cross_nprev", "cross_mu", "anchor_target",
             "cross_fc90", "cross_E90", "cross_H", "node_w", "node_h")
    INT = ("seg_i0", "seg_i1", "seg_offset", "joint_seg0", "joint_seg1", "local_load_node", "anchor_node",
           "cross_strand")
    BYTE = ("anchor_mask", "cross_enabled", "cross_locked")
    OPTIONAL = ("omega0", "anchor_target", "cross_fc90", "cross_E90", "cross_H", "node_w", "node_h")   # NULL: None

    def __init__(self):
        self.n = self.m = self.p = self.n_strands = self.K = 0
        self.params = default_params()
        self.protocol = None       # dict(mode, probe, sched, settle, avg, axis): a load protocol (ws_protocol)
        self.node_offset = None
        self.span = 0.0

    @classmethod
    def from_struct(cls, md: WsModel, node_offset=None, span=0.0) -> "Model":
        self = cls()
        self.n, self.m, self.p, self.n_strands, self.K = md.n, md.m, md.p, md.n_strands, md.K
        nl, na = md.n_local_loads, md.n_anchors
        sizes = {"X": 3 * self.n, "X0": 3 * self.n, "Q": 4 * self.m, "l0": self.m, "joint_len": self.p,
                 "omega0": 3 * self.p, "EA": self.m, "EIx": self.m, "EIy": self.m, "GJ": self.m, "GA": self.m,
                 "load_const": 3 * self.n, "local_load_F": 3 * nl, "cross_wk": 2 * self.K, "cross_hk": 2 * self.K,
                 "cross_u": 2 * self.K, "cross_nprev": 3 * self.K, "cross_mu": self.K,
                 "seg_i0": self.m, "seg_i1": self.m, "seg_offset": self.n_strands + 1, "joint_seg0": self.p,
                 "joint_seg1": self.p, "local_load_node": nl, "anchor_node": na, "cross_strand": 2 * self.K,
                 "anchor_mask": na, "cross_enabled": self.K, "cross_locked": self.K,
                 "anchor_target": 3 * na, "cross_fc90": 2 * self.K, "cross_E90": 2 * self.K, "cross_H": 2 * self.K,
                 "node_w": self.n, "node_h": self.n}
        for k, dt in [(k, np.float64) for k in cls.FLOAT] + [(k, np.int32) for k in cls.INT] + \
                     [(k, np.uint8) for k in cls.BYTE]:
            ptr, n = getattr(md, k), sizes[k]
            if not ptr and k in cls.OPTIONAL:
                arr = None
            elif not ptr or n == 0:
                arr = np.zeros(n, dtype=dt)
            else:
                arr = np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt, copy=True)
            setattr(self, k, arr)
        self.params = {k: getattr(md.params, k) for k in PARAM_KEYS}
        if node_offset is not None:
            self.node_offset = np.asarray(node_offset, dtype=np.int32).copy()
        self.span = float(span)
        return self

    def copy(self) -> "Model":
        other = Model.__new__(Model)
        for k, v in self.__dict__.items():
            setattr(other, k, v.copy() if isinstance(v, (np.ndarray, dict)) else v)
        return other

    COUNTS = ("n", "m", "p", "n_strands", "K")

    def save(self, path):
        """the model as a compressed .npz: every array, the counts, the span and the parameters (no load protocol)"""
        if self.protocol:
            raise ValueError("Model.save: a model with a load protocol is not saved")
        arrays = {k: v for k, v in self.__dict__.items() if isinstance(v, np.ndarray)}
        meta = {f"count_{k}": np.int64(getattr(self, k)) for k in self.COUNTS}
        np.savez_compressed(path, **arrays, **meta, span=np.float64(self.span),
                            param_keys=np.array(list(self.params)), param_values=np.array(list(self.params.values()),
                                                                                           dtype=np.float64))

    @classmethod
    def load(cls, path) -> "Model":
        """a model saved by ``save``; reading it does not load the solver library"""
        self = cls.__new__(cls)
        with np.load(path) as z:
            for k in self.COUNTS:
                setattr(self, k, int(z[f"count_{k}"]))
            self.span = float(z["span"])
            ints = {f[0] for f in WsParams._fields_ if f[1] is C.c_int32}
            self.params = {str(k): (int(v) if str(k) in ints else float(v))
                           for k, v in zip(z["param_keys"], z["param_values"])}
            self.protocol = None
            self.node_offset = z["node_offset"].copy() if "node_offset" in z else None
            for k in self.FLOAT + self.INT + self.BYTE:
                setattr(self, k, z[k].copy() if k in z else None)
        for k in self.INT + self.BYTE:
            if getattr(self, k) is None:
                raise ValueError(f"Model.load: {path} has no {k}")
        for k in self.FLOAT:
            if getattr(self, k) is None and k not in self.OPTIONAL:
                raise ValueError(f"Model.load: {path} has no {k}")
        return self

    def struct(self) -> WsModel:
        """A WsModel pointing into this object's arrays (keep the Model alive while the struct is used)."""
        md = WsModel()
        md.n, md.m, md.p, md.n_strands, md.K = self.n, self.m, self.p, self.n_strands, self.K
        for k in self.FLOAT:
            if getattr(self, k) is None:
                setattr(md, k, None)
                continue
            a = np.ascontiguousarray(getattr(self, k), dtype=np.float64)
            setattr(self, k, a)
            setattr(md, k, _ptr(a, C.c_double))
        for k in self.INT:
            a = np.ascontiguousarray(getattr(self, k), dtype=np.int32)
            setattr(self, k, a)
            setattr(md, k, _ptr(a, C.c_int32))
        for k in self.BYTE:
            a = np.ascontiguousarray(getattr(self, k), dtype=np.uint8)
            setattr(self, k, a)
            setattr(md, k, _ptr(a, C.c_uint8))
        md.n_local_loads = len(self.local_load_node)
        md.n_anchors = len(self.anchor_node)
        md.params = params_struct(self.params)
        if self.protocol:
            pr = WsProtocol()
            sched = list(self.protocol["sched"])
            if not 1 <= len(sched) <= PROTOCOL_MAX_INC:
                raise ValueError(f"a load protocol has 1..{PROTOCOL_MAX_INC} increments")
            pr.mode, pr.probe, pr.n_inc = int(self.protocol["mode"]), int(self.protocol["probe"]), len(sched)
            pr.settle, pr.avg = int(self.protocol["settle"]), int(self.protocol["avg"])
            for k in range(3):
                pr.axis[k] = float(self.protocol["axis"][k])
            for k, v in enumerate(sched):
                pr.sched[k] = float(v)
            self._protocol_struct = pr          # kept alive with the model
            md.protocol = C.pointer(pr)
        return md

    def goals(self) -> dict:
        """the goals the device will use (masses, static frame stiffness, initialised contacts), built on the host"""
        st = self.struct()
        out = {"mass": np.zeros(self.n), "k_rot_static": np.zeros(3 * self.m), "u": np.zeros(2 * self.K),
               "nprev": np.zeros(3 * self.K)}
        lref = C.c_double()
        check(lib().ws_model_goals(C.byref(st), *[_ptr(out[k], C.c_double) for k in ("mass", "k_rot_static", "u", "nprev")],
                                   C.byref(lref)), "ws_model_goals")
        out["l_ref"] = lref.value
        return out

    # handy views
    def anchored_nodes(self, translation=True):
        mask = self.anchor_mask & (7 if translation else 0x3F)
        return self.anchor_node[mask != 0]


def _from_scene(sc) -> Model:
    L = lib()
    md = L.ws_scene_model(sc).contents
    off = np.ctypeslib.as_array(L.ws_scene_node_offset(sc), shape=(md.n_strands + 1,)).copy()
    model = Model.from_struct(md, off, L.ws_scene_span(sc))
    L.ws_scene_free(sc)
    return model


def kagome(side, subdivisions, edge, width, height, E, G, density, mu=0.3, mu_range=None, inward=0.0, lift=0.0,
           z_noise=0.0, gravity=True, seed=1, params=None) -> Model:
    cfg = WsKagomeCfg()
    cfg.side, cfg.subdivisions, cfg.edge = side, subdivisions, edge
    cfg.width, cfg.height, cfg.E, cfg.G, cfg.density = width, height, E, G, density
    cfg.mu = mu
    cfg.mu_lo, cfg.mu_hi = (mu_range if mu_range else (0.0, 0.0))
    cfg.inward, cfg.lift, cfg.z_noise, cfg.gravity, cfg.seed = inward, lift, z_noise, int(gravity), seed
    cfg.params = params_struct(params or default_params())
    sc = C.c_void_p()
    check(lib().ws_scene_kagome(C.byref(cfg), C.byref(sc)), "ws_scene_kagome")
    return _from_scene(sc)


def polylines(strands, normals=None, knot_rows=None, knots=(), anchors=(), loads=(), width=60.0, height=30.0,
              E=1e4, G=625.0, density=700.0, mu=0.35, gravity=False, thickness=30.0, params=None) -> Model:
    """Stand-alone laths (topologyFromPolylines): strands = list of (N_s, 3) point arrays; anchors = [((s, k), mask)];
    loads = [((s, k), (Fx, Fy, Fz), local)]; knots = [((sa, ka), (sb, kb))]."""
    cfg = WsPolylineCfg()
    counts = np.array([len(s) for s in strands], dtype=np.int32)
    pts = np.ascontiguousarray(np.concatenate([np.asarray(s, dtype=np.float64).reshape(-1, 3) for s in strands]).ravel())
    keep = [counts, pts]
    cfg.n_strands = len(strands)
    cfg.node_count = _ptr(counts, C.c_int32)
    cfg.points = _ptr(pts, C.c_double)
    if normals is not None:
        nrm = np.ascontiguousarray(np.concatenate([np.asarray(n, dtype=np.float64).reshape(-1, 3) for n in normals]).ravel())
        keep.append(nrm)
        cfg.normals = _ptr(nrm, C.c_double)
    if knot_rows is not None:
        kc = np.array([len(r) for r in knot_rows], dtype=np.int32)
        kr = np.array([x for r in knot_rows for x in r], dtype=np.int32)
        keep += [kc, kr]
        cfg.knot_count, cfg.knot_rows = _ptr(kc, C.c_int32), _ptr(kr, C.c_int32)
    kn = np.array([[a[0], a[1], b[0], b[1]] for a, b in knots], dtype=np.int32).ravel()
    keep.append(kn)
    cfg.n_knots, cfg.knots = len(knots), _ptr(kn, C.c_int32) if len(knots) else None
    af = np.array([f for f, _ in anchors], dtype=np.int32).ravel()
    am = np.array([m for _, m in anchors], dtype=np.uint8)
    lf = np.array([f for f, _, _ in loads], dtype=np.int32).ravel()
    lF = np.array([F for _, F, _ in loads], dtype=np.float64).ravel()
    ll = np.array([1 if loc else 0 for _, _, loc in loads], dtype=np.uint8)
    keep += [af, am, lf, lF, ll]
    cfg.n_anchors = len(anchors)
    cfg.anchor_frames, cfg.anchor_masks = _ptr(af, C.c_int32), _ptr(am, C.c_uint8)
    cfg.n_loads = len(loads)
    cfg.load_frames, cfg.load_F, cfg.load_local = _ptr(lf, C.c_int32), _ptr(lF, C.c_double), _ptr(ll, C.c_uint8)
    cfg.thickness = thickness
    cfg.width, cfg.height, cfg.E, cfg.G, cfg.density, cfg.mu = width, height, E, G, density, mu
    cfg.gravity = int(gravity)
    cfg.params = params_struct(params or default_params())
    sc = C.c_void_p()
    check(lib().ws_scene_polylines(C.byref(cfg), C.byref(sc)), "ws_scene_polylines")
    del keep
    return _from_scene(sc)


def mask(*dofs) -> int:
    """anchor mask from DOF flags [X, Y, Z, rX, rY, rZ] (1 = fixed)"""
    return sum(1 << i for i, f in enumerate(dofs) if f)

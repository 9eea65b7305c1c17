"""GpuSolver: the reference's batched solver interface (web/js/solver_gpu.js:62-523) over the C ABI of
include/weavesim.h.

    solver = GpuSolver([model, ...], precision="mixed", form="cta")
    ctl = solver.step(1000)             # GpuSolver.step: runs up to n iterations, each instance stops at convergence
    state = solver.download(0)          # GpuSolver.download: positions, frames, slide coordinates, stick/slip, forces
    solver.update_params(0, variant)    # GpuSolver.updateParams + CpuSolver.rebuildGoals: warm start
    solver.internalize(0)               # CpuSolver.internalize / GpuSolver.internalize

Unlike the reference, the instances of one solver need not share a topology (uneven gridshells in one launch).
Every call goes to the CUDA library; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import PROTOCOL_MAX_INC, WsControl, WsOpts, WsStateOut, check, lib

STATUS = {0: "running", 1: "converged", 2: "max_iter", 3: "non_finite"}


def device_count() -> int:
    return int(lib().ws_device_count())


STATE_FIELDS = ("X", "Q", "V", "W", "u", "nprev", "slip", "Fn", "Ft", "gap", "N", "Vsh", "M", "reactions", "stuck", "state",
                "ctype", "theta", "phi", "area", "pressure", "util", "lambda", "dent", "M_rot", "rot_slip", "utm", "floor_F",
                "floor_state", "seg_M", "node_M", "disp")


_PTR = {np.dtype(np.uint8): C.POINTER(C.c_uint8), np.dtype(np.float64): C.POINTER(C.c_double)}


def _state_buffers(md, fields=None):
    """host arrays for one instance's state and the ws_state_out pointing at them; fields left out stay NULL.  The
    arrays are left uninitialised: ws_download writes every element of every array it is given."""
    n, m, p, K = md.n, md.m, md.p, md.K
    size = {"X": 3 * n, "Q": 4 * m, "V": 3 * n, "W": 3 * m, "u": 2 * K, "nprev": 3 * K, "slip": K, "Fn": K, "Ft": K,
            "gap": K, "N": m, "Vsh": 2 * m, "M": 3 * p, "reactions": 3 * n, "stuck": K, "state": K,
            "ctype": K, "theta": K, "phi": 2 * K, "area": K, "pressure": K, "util": K,
            "lambda": K, "dent": K, "M_rot": K, "rot_slip": K, "utm": 4 * PROTOCOL_MAX_INC, "floor_F": 3 * n,
            "floor_state": n, "seg_M": 3 * m, "node_M": 4 * n, "disp": 3 * n}
    names = STATE_FIELDS if fields is None else tuple(fields)
    bad = [k for k in names if k not in size]
    if bad:
        raise ValueError(f"unknown state fields {bad}; known: {STATE_FIELDS}")
    out = {k: np.empty(size[k], dtype=np.uint8 if k in ("stuck", "state", "ctype", "floor_state") else np.float64)
           for k in names}
    so = WsStateOut()
    for k, a in out.items():
        setattr(so, k, C.cast(a.ctypes.data, _PTR[a.dtype]) if a.size else None)
    return out, so


def relax_noalloc(model, n_iter, precision="mixed", threads=256, stream=None):
    """One small instance relaxed inside the library's static device scratch (ws_relax_noalloc): for callers that cannot
    allocate device memory.  Returns (state, control)."""
    st = model.struct()
    out, so = _state_buffers(model)
    ctl = WsControl()
    prec = _lib.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    check(lib().ws_relax_noalloc(C.byref(st), prec, int(n_iter), int(threads), stream, C.byref(so), C.byref(ctl)),
          "ws_relax_noalloc")
    return out, ctl.as_dict()


def _opts(precision="mixed", form="cta", side_order="auto"):
    o = WsOpts()
    o.precision = _lib.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    o.form = _lib.FORMS[form] if isinstance(form, str) else int(form)
    o.side_order = {"auto": 0, "general": 1}[side_order]
    return o


def _model_array(models):
    structs = [m.struct() for m in models]
    return structs, (C.POINTER(_lib.WsModel) * len(structs))(*[C.pointer(s) for s in structs])


def tune_key(models, precision="mixed", form="cta", device=None) -> str:
    """the autotuner's size bucket of a batch (ws_tune_key; needs no GPU when `device` names one)"""
    keep, arr = _model_array(models)
    o = _opts(precision, form)
    buf = C.create_string_buffer(512)
    check(lib().ws_tune_key(arr, len(models), C.byref(o), device.encode() if device else None, buf, 512), "ws_tune_key")
    return buf.value.decode()


def tune_candidates(models, precision="mixed", form="cta", after=None):
    """the shapes the autotuner times (ws_tune_candidates): stage 1, or stage 2 at the stage-1 shape `after` (a dict)"""
    keep, arr = _model_array(models)
    o = _opts(precision, form)
    aft = None
    if after is not None:
        aft = _lib.WsShape()
        for k in ("threads", "cta_state", "wide_cluster", "wide_min", "plain_launch"):
            setattr(aft, k, int(after[k]))
    out = (_lib.WsShape * 64)()
    n = lib().ws_tune_candidates(arr, len(models), C.byref(o), C.byref(aft) if aft is not None else None, out, 64)
    if n < 0:
        check(n, "ws_tune_candidates")
    return [out[i].as_dict() for i in range(min(n, 64))]


def tune_cache_get(key):
    sh = _lib.WsShape()
    return sh.as_dict() if lib().ws_tune_cache_get(key.encode(), C.byref(sh)) == 1 else None


def tune_cache_put(key, shape: dict):
    sh = _lib.WsShape()
    for k, v in shape.items():
        if k != "source":
            setattr(sh, k, v)
    check(lib().ws_tune_cache_put(key.encode(), C.byref(sh)), "ws_tune_cache_put")


def tune_cache_clear():
    lib().ws_tune_cache_clear()


class GpuSolver:
    def __init__(self, models, precision="mixed", form="cta", threads=0, device=0, budget_bytes=0, side_order="auto",
                 cta_state="auto", wide_cluster=0, wide_min=0, tune=False):
        if not isinstance(models, (list, tuple)):
            models = [models]
        self.models = list(models)
        self.B = len(self.models)
        self._structs = [m.struct() for m in self.models]
        arr = (C.POINTER(_lib.WsModel) * self.B)(*[C.pointer(s) for s in self._structs])
        opts = WsOpts()
        opts.precision = _lib.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        opts.form = _lib.FORMS[form] if isinstance(form, str) else int(form)
        opts.threads, opts.device, opts.budget_bytes = int(threads), int(device), int(budget_bytes)
        opts.side_order = {"auto": 0, "general": 1}[side_order]
        opts.cta_state = {"auto": 0, "global": 1}[cta_state]
        opts.wide_cluster, opts.wide_min, opts.tune = int(wide_cluster), int(wide_min), int(bool(tune))
        self.precision, self.form = precision, form
        h = C.c_void_p()
        check(lib().ws_create(arr, self.B, C.byref(opts), C.byref(h)), "ws_create")
        self.h = h

    # ------------------------------------------------------------------------------------------- running
    def step(self, n_iter, instances=None, read=True):
        """Up to n_iter DR iterations on the selected instances (all by default); returns the control blocks."""
        mask = None
        if instances is not None:
            m = np.zeros(self.B, dtype=np.uint8)
            m[list(instances)] = 1
            mask = m.ctypes.data_as(C.POINTER(C.c_uint8))
            self._mask = m
        ctl = (WsControl * self.B)() if read else None
        check(lib().ws_step(self.h, int(n_iter), mask, ctl), "ws_step")
        return [c.as_dict() for c in ctl] if read else None

    def read_control(self):
        ctl = (WsControl * self.B)()
        check(lib().ws_read_control(self.h, ctl), "ws_read_control")
        return [c.as_dict() for c in ctl]

    def run(self, max_iter=None, chunk=1000, instances=None):
        """step() in chunks until every selected instance has stopped (GpuSolver in app.js / calibrate.js loops)."""
        max_iter = max_iter or max(m.params["max_iter"] for m in self.models)
        done = 0
        ctl = self.read_control()
        sel = list(range(self.B)) if instances is None else list(instances)
        while done < max_iter:
            k = min(chunk, max_iter - done)
            ctl = self.step(k, instances=sel)
            done += k
            if all(ctl[b]["status"] != 0 for b in sel):
                break
        return ctl

    def last_step_stats(self):
        ms = C.c_double()
        nl = C.c_int64()
        check(lib().ws_last_step_stats(self.h, C.byref(ms), C.byref(nl)), "ws_last_step_stats")
        return ms.value, nl.value

    # ------------------------------------------------------------------------------------------- state
    def download(self, b=0, fields=None) -> dict:
        """state of instance b (ws_download); `fields` (names of _state_buffers) limits the copy to those arrays"""
        out, so = _state_buffers(self.models[b], fields)
        check(lib().ws_download(self.h, int(b), C.byref(so)), "ws_download")
        return out

    def upload_state(self, b, X, Q, u=None):
        X = np.ascontiguousarray(X, dtype=np.float64)
        Q = np.ascontiguousarray(Q, dtype=np.float64)
        up = None if u is None else np.ascontiguousarray(u, dtype=np.float64)
        dp = C.POINTER(C.c_double)
        check(lib().ws_upload_state(self.h, int(b), X.ctypes.data_as(dp), Q.ctypes.data_as(dp),
                                    None if up is None else up.ctypes.data_as(dp)), "ws_upload_state")

    def update_params(self, b, model):
        """warm start with the stiffness, loads, friction, parameters and support targets of `model`"""
        st = model.struct()
        self._keep = (model, st)
        check(lib().ws_set_params(self.h, int(b), C.byref(st)), "ws_set_params")
        self.models[b] = model

    def load_instance(self, b, model):
        """slot b takes a new model of the same element counts; its iteration count restarts at 0"""
        st = model.struct()
        self._keep_load = (model, st)
        check(lib().ws_load_instance(self.h, int(b), C.byref(st)), "ws_load_instance")
        self.models[b] = model

    def internalize(self, b):
        check(lib().ws_internalize(self.h, int(b)), "ws_internalize")

    @property
    def stream(self):
        return lib().ws_stream(self.h)

    @property
    def resident(self):
        """True when the batched form holds its instances in shared memory"""
        return bool(lib().ws_cta_resident(self.h))

    @property
    def shape(self):
        """the launch shape in use (ws_get_shape): threads, cta_state, wide_cluster, wide_min, plain_launch, and whether
        it came from the options, the tuner or the tuner's cache"""
        sh = _lib.WsShape()
        check(lib().ws_get_shape(self.h, C.byref(sh)), "ws_get_shape")
        return sh.as_dict()

    @property
    def wide(self):
        """(instances relaxed by a thread-block cluster each, blocks per cluster) in the batched form"""
        cl = C.c_int32()
        n = lib().ws_wide_instances(self.h, C.byref(cl))
        return int(n), int(cl.value)

    @property
    def side_order(self):
        """'short' when the crossing sides are ranked inside the element kernel (slides under one segment per
        iteration), 'general' otherwise"""
        return "short" if lib().ws_side_order(self.h) == 1 else "general"

    @property
    def device_bytes(self):
        return int(lib().ws_device_bytes(self.h))

    def dispose(self):
        h, self.h = getattr(self, "h", None), None
        if h:
            lib().ws_destroy(h)

    def __del__(self):
        try:
            self.dispose()
        except Exception:
            pass

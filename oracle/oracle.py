"""ORACLE — test infrastructure, not product code.

ctypes wrapper of oracle/_build/liboracle.so, the f64 CPU restatement of the reference's CpuSolver
(web/js/solver_cpu.js:661-875 with web/js/rod_cosserat.js).  Only tests, the smoke check and the CPU-baseline leg of
the benchmark use it, as the checker of the CUDA path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")

_dp = C.POINTER(C.c_double)


class OrcView(C.Structure):
    _fields_ = [(k, C.c_int32) for k in ("n", "m", "p", "K", "iteration", "converged", "rollbacks", "has_contact")] + \
               [(k, C.c_double) for k in ("residual", "ke_prev", "ke", "fref", "res_force", "res_torque", "l_ref",
                                          "e_stretch", "e_shear", "e_bend", "e_twist", "e_contact")] + \
               [(k, _dp) for k in ("X", "X0", "V", "Q", "W", "u", "nprev", "slip", "Fn", "Ft", "gap", "state", "N",
                                   "Vsh", "M", "reactions", "mass", "inertia3", "k_rot_static", "F", "T", "tm")] + \
               [("stuck", C.POINTER(C.c_uint8)), ("ctype", C.POINTER(C.c_int32))] + \
               [(k, _dp) for k in ("theta", "phi", "area", "pressure", "util", "lambda", "dent", "M_rot", "rot_slip")] + \
               [("utm", _dp), ("utm_inc", C.c_int32), ("utm_phase", C.c_int32), ("utm_done", C.c_int32),
                ("has_floor", C.c_int32), ("floor_F", _dp), ("e_floor", C.c_double), ("floor_state", C.POINTER(C.c_uint8)),
                ("res_rigid", C.c_double), ("rb_v", C.c_double * 3), ("rb_w", C.c_double * 3)]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.orc_create.argtypes = [C.c_void_p]
        L.orc_create.restype = C.c_void_p
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_step.argtypes = [C.c_void_p, C.c_int32]
        L.orc_rebuild.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_internalize.argtypes = [C.c_void_p]
        L.orc_view_get.argtypes = [C.c_void_p, C.POINTER(OrcView)]
        L.orc_rod_eval.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
        L.orc_rod_eval.restype = C.c_double
        L.orc_set_clamps.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_uint8)]
        L.orc_set_state.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.orc_segment_moments.argtypes = [C.c_void_p, _dp]
        L.orc_node_layers.argtypes = [C.c_void_p, _dp]
        _lib = L
    return _lib


def _arr(p, n):
    if not p or n == 0:
        return np.zeros(n)
    return np.ctypeslib.as_array(p, shape=(n,))


class Oracle:
    """CpuSolver restated in f64 over a weavesim_b200 Model (goals and contact initialisation are built here too)."""

    def __init__(self, model):
        self.model = model
        md = model.struct()
        self.h = lib().orc_create(C.byref(md))
        if not self.h:
            raise RuntimeError("oracle: model rejected")

    def __del__(self):
        h, self.h = getattr(self, "h", None), None
        if h and _lib is not None:
            _lib.orc_free(h)

    def step(self, n=1) -> bool:
        return bool(lib().orc_step(self.h, int(n)))

    def run(self, max_iter=None, chunk=100):
        max_iter = max_iter or self.model.params["max_iter"]
        done = 0
        while done < max_iter:
            k = min(chunk, max_iter - done)
            if self.step(k):
                break
            done += k
        return self.view()

    def rebuild(self, model):
        """rebuildGoals with the parameters of `model` (warm start)"""
        md = model.struct()
        lib().orc_rebuild(self.h, C.byref(md))

    def internalize(self):
        lib().orc_internalize(self.h)

    def _v(self):
        v = OrcView()
        lib().orc_view_get(self.h, C.byref(v))
        return v

    def view(self, copy=True) -> dict:
        v = self._v()
        n, m, p, K = v.n, v.m, v.p, v.K
        out = {k: getattr(v, k) for k in ("n", "m", "p", "K", "iteration", "converged", "rollbacks", "residual",
                                           "ke_prev", "ke", "fref", "res_force", "res_torque", "l_ref", "e_stretch",
                                           "e_shear", "e_bend", "e_twist", "e_contact")}
        sizes = {"X": 3 * n, "X0": 3 * n, "V": 3 * n, "Q": 4 * m, "W": 3 * m, "u": 2 * K, "nprev": 3 * K, "slip": K,
                 "Fn": K if v.has_contact else 0, "Ft": K if v.has_contact else 0, "gap": K if v.has_contact else 0,
                 "state": K if v.has_contact else 0, "N": m, "Vsh": 2 * m, "M": 3 * p, "reactions": 3 * n,
                 "mass": n, "inertia3": 3 * m, "k_rot_static": 3 * m, "F": 3 * n, "T": 3 * m, "tm": 3 * m}
        for k, s in sizes.items():
            a = _arr(getattr(v, k), s)
            out[k] = a.copy() if copy else a
        st = _arr(v.stuck, K) if K else np.zeros(0, dtype=np.uint8)
        out["stuck"] = np.array(st, dtype=np.uint8)
        hc = K and v.has_contact
        out["ctype"] = np.ctypeslib.as_array(v.ctype, shape=(K,)).astype(np.uint8) if hc else np.zeros(0, dtype=np.uint8)
        out["utm"] = _arr(v.utm, 4 * 64).copy()
        out["utm_inc"], out["utm_phase"], out["utm_done"] = v.utm_inc, v.utm_phase, v.utm_done
        out["e_floor"] = v.e_floor
        out["res_rigid"] = v.res_rigid
        out["rb_v"], out["rb_w"] = np.array(list(v.rb_v)), np.array(list(v.rb_w))
        out["floor_F"] = _arr(v.floor_F, 3 * n).copy() if v.has_floor else np.zeros(3 * n)
        out["floor_state"] = np.ctypeslib.as_array(v.floor_state, shape=(n,)).copy() if v.has_floor else np.zeros(n, np.uint8)
        for k, s_ in (("theta", K), ("phi", 2 * K), ("area", K), ("pressure", K), ("util", K), ("lambda", K), ("dent", K),
                      ("M_rot", K), ("rot_slip", K)):
            a = _arr(getattr(v, k), s_) if hc else np.zeros(0)
            out[k] = a.copy() if copy else a
        return out

    def rod_eval(self, X, Q):
        v = self._v()
        X = np.ascontiguousarray(X, dtype=np.float64)
        Q = np.ascontiguousarray(Q, dtype=np.float64)
        F = np.zeros(3 * v.n)
        T = np.zeros(3 * v.m)
        e = lib().orc_rod_eval(self.h, X.ctypes.data_as(_dp), Q.ctypes.data_as(_dp), F.ctypes.data_as(_dp),
                               T.ctypes.data_as(_dp))
        return e, F, T

    def set_clamps(self, clamps):
        """clamps: [(node, seg, mask3)], re-frozen at the current frames"""
        nc = len(clamps)
        node = (C.c_int32 * nc)(*[c[0] for c in clamps])
        seg = (C.c_int32 * nc)(*[c[1] for c in clamps])
        mk = (C.c_uint8 * nc)(*[c[2] for c in clamps])
        lib().orc_set_clamps(self.h, nc, node, seg, mk)

    def set_state(self, X=None, Q=None, omega0=None):
        keep = [np.ascontiguousarray(a, dtype=np.float64) if a is not None else None for a in (X, Q, omega0)]
        ptrs = [a.ctypes.data_as(_dp) if a is not None else None for a in keep]
        lib().orc_set_state(self.h, *ptrs)

    def node_layers(self):
        """Mx, My, T, N at the nodes (fields.js nodeValues): [4, n]"""
        v = self._v()
        out = np.zeros(4 * v.n)
        lib().orc_node_layers(self.h, out.ctypes.data_as(_dp))
        return out.reshape(4, v.n)

    def segment_moments(self):
        v = self._v()
        out = np.zeros(3 * v.m)
        lib().orc_segment_moments(self.h, out.ctypes.data_as(_dp))
        return out

"""The C ABI boundary (include/weavesim.h): exports, error codes, host-side goal assembly against the oracle."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import cases
import weavesim_b200 as ws
from weavesim_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "weavesim.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ws_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) >= 20
    lib = C.CDLL(_lib.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_no_device_is_an_error_not_a_fallback():
    if ws.device_count() > 0:
        pytest.skip("a CUDA device is present")
    with pytest.raises(RuntimeError, match=r"\(-5\).*no CUDA device"):
        ws.GpuSolver([ws.configs.dome_small()])


def test_malformed_models_are_rejected():
    md = ws.configs.dome_small()
    bad = md.copy()
    bad.seg_i1[3] = bad.n + 5
    with pytest.raises(RuntimeError, match="segment node out of range"):
        bad.goals()
    bad = md.copy()
    bad.l0[0] = 0.0
    with pytest.raises(RuntimeError, match="rest length"):
        bad.goals()
    bad = md.copy()
    bad.cross_strand[0] = md.n_strands
    with pytest.raises(RuntimeError, match="crossing strand"):
        bad.goals()
    buf = C.create_string_buffer(256)
    n = _lib.lib().ws_last_error(buf, 256)
    assert n > 0 and b"crossing strand" in buf.value


@pytest.mark.parametrize("make", [lambda: ws.configs.dome_small(), lambda: ws.configs.dome_stiff(),
                                  lambda: cases.crossing(-50.0, 5.0), lambda: cases.cantilever(10)])
def test_host_goals_match_oracle(oracle_mod, make):
    """masses, static frame stiffness and the initialised contacts of the product's host set-up are those of the
    oracle's restatement of CpuSolver._buildGoals + PolylineContact.initialize"""
    md = make()
    g = md.goals()
    v = oracle_mod.Oracle(md).view()
    assert np.array_equal(g["mass"], v["mass"])
    assert np.array_equal(g["k_rot_static"], v["k_rot_static"])
    assert np.array_equal(g["u"], v["u"])
    assert np.array_equal(g["nprev"], v["nprev"])
    assert g["l_ref"] == v["l_ref"]

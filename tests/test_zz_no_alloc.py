"""The allocation-free entry point ws_relax_noalloc, checked through the C ABI against ws_create + ws_step +
ws_download.

It exists for callers that cannot allocate device memory themselves: a framework whose pool or caching allocator owns
the GPU's memory, or a serving process that must not allocate once it is running.  The instance lives in a static
device array of the library instead, so the checks here are: the same result as the ordinary entry point on two calls
in a row (the second call starts from whatever the first left in the shared array), and a clear refusal for a model
larger than the array.  This file is collected last on purpose.
"""
import numpy as np
import pytest

import cases
import weavesim_b200 as ws
from weavesim_b200 import solver


def test_oversized_model_is_refused():
    md = ws.configs.shell_large()
    with pytest.raises(RuntimeError, match=r"\(-1\).*bytes of device scratch"):
        solver.relax_noalloc(md, 10)


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [("f64", 1e-9), ("mixed", 1e-5)])
def test_matches_ordinary_entry_point_on_two_calls(prec, tol):
    if ws.device_count() < 1:
        pytest.skip("no CUDA device")
    models = [ws.configs.dome_small(seed=1), ws.configs.dome_stiff(seed=2)]
    for call, md in enumerate(models):
        s = ws.GpuSolver([md.copy()], precision=prec, threads=256)
        ctl_ref = s.step(400)[0]
        ref = s.download(0)
        s.dispose()
        st, ctl = solver.relax_noalloc(md.copy(), 400, prec, threads=256)
        assert ctl["iter"] == ctl_ref["iter"] == 400, call
        assert cases.max_node_err_span(st["X"], ref["X"], md.span) < tol, call
        assert np.abs(st["u"] - ref["u"]).max() < 1e-6, call
        assert np.abs(st["Q"] - ref["Q"]).max() < 1e-6, call
        assert np.array_equal(st["stuck"], ref["stuck"]), call

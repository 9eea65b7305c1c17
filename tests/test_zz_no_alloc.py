"""The allocation-free entry point ws_relax_noalloc, checked through the C ABI against ws_create + ws_step +
ws_download.

It exists for callers that cannot allocate device memory themselves: a framework whose pool or caching allocator owns
the GPU's memory, or a serving process that must not allocate once it is running.  The instance lives in a static
device array of the library instead, so the checks here are: the same bits as the ordinary entry point running the same
kernel (the batched form with global state and the same block size) on two calls in a row (the second call starts from
whatever the first left in the shared array), no change in the device's free memory across a call, and a clear refusal
for a model larger than the array.  This file is collected last on purpose.
"""
import numpy as np
import pytest

import weavesim_b200 as ws
from weavesim_b200 import solver

FIELDS = ("X", "Q", "V", "W", "u", "nprev", "slip", "Fn", "Ft", "gap", "N", "M", "reactions", "stuck", "state")


def test_oversized_model_is_refused():
    md = ws.configs.shell_large()
    with pytest.raises(RuntimeError, match=r"\(-1\).*bytes of device scratch"):
        solver.relax_noalloc(md, 10)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f64", "mixed"])
def test_matches_ordinary_entry_point_on_two_calls(prec):
    if ws.device_count() < 1:
        pytest.skip("no CUDA device")
    import torch
    models = [ws.configs.dome_small(seed=1), ws.configs.dome_stiff(seed=2)]
    solver.relax_noalloc(models[0].copy(), 0, prec, threads=256)          # device code loaded, the array reserved
    for call, md in enumerate(models):
        s = ws.GpuSolver([md.copy()], precision=prec, threads=256, cta_state="global")
        assert not s.resident
        ctl_ref = s.step(400)[0]
        ref = s.download(0)
        s.dispose()
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        st, ctl = solver.relax_noalloc(md.copy(), 400, prec, threads=256)
        assert torch.cuda.mem_get_info()[0] == free0, call
        assert ctl["iter"] == ctl_ref["iter"] == 400, call
        assert ctl["rollbacks"] == ctl_ref["rollbacks"] and ctl["residual"] == ctl_ref["residual"], call
        for k in FIELDS:
            assert np.array_equal(st[k], ref[k]), (call, k)

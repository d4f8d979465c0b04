"""The allocation-free FDK backprojection entry point
(rtkb_fdk_backproject_static_scratch), for callers that cannot allocate
device memory during a reconstruction.  Called through the C ABI and checked
against rtkb_fdk_backproject on two calls in a row (the second with a shorter
stack, so stale scratch from the first call must not leak into it).  Collected
last, so a run that stops at the first failure has run every other test."""
import ctypes as C

import numpy as np
import pytest

from tests.gpu_util import REL_L2_TOL, rel_l2, to_np

pytestmark = pytest.mark.gpu


def _call(lib, fn, g, vd, pd, p, v0):
    import torch

    out = torch.empty_like(v0)
    rc = fn(g.handle, C.byref(vd), C.byref(pd), C.c_void_p(p.data_ptr()), C.c_void_p(v0.data_ptr()),
            C.c_void_p(out.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, lib.rtkb_last_error()
    return out


def test_static_scratch_matches_allocating_entry_point(rtkb):
    import torch

    lib = rtkb.load()
    gen = torch.Generator(device="cuda").manual_seed(7)
    cases = [(120, (96, 80, 88), (160, 128)), (40, (64, 72, 56), (128, 120))]  # second call: shorter stack
    for nproj, vsize, (nu, nv) in cases:
        g = rtkb.geometry.circular(nproj, 1000.0, 1536.0, projOffsetX=4.0, projOffsetY=-2.0)
        vd = rtkb.make_desc(vsize, (1.5, 1.5, 1.5))
        pd = rtkb.make_desc((nu, nv, nproj), (1.0, 1.0, 1.0))
        p = torch.rand((nproj, nv, nu), device="cuda", generator=gen) * 2 - 1
        v0 = torch.rand((vsize[2], vsize[1], vsize[0]), device="cuda", generator=gen)
        ref = _call(lib, lib.rtkb_fdk_backproject, g, vd, pd, p, v0)
        got = _call(lib, lib.rtkb_fdk_backproject_static_scratch, g, vd, pd, p, v0)
        assert rel_l2(to_np(got), to_np(ref)) < REL_L2_TOL
    assert rtkb.ops.device_status() == 0


def test_static_scratch_rejects_oversized_stacks(rtkb):
    import torch

    lib = rtkb.load()
    g = rtkb.geometry.circular(2049, 1000.0, 1536.0)
    vd = rtkb.make_desc((4, 4, 4), (1.0,) * 3)
    pd = rtkb.make_desc((8, 8, 2049), (1.0,) * 3)
    p = torch.zeros((2049, 8, 8), device="cuda")
    v = torch.zeros((4, 4, 4), device="cuda")
    rc = lib.rtkb_fdk_backproject_static_scratch(g.handle, C.byref(vd), C.byref(pd), C.c_void_p(p.data_ptr()),
                                                 C.c_void_p(v.data_ptr()), C.c_void_p(v.data_ptr()), None)
    assert rc == rtkb._capi.RTKB_ERR_INVALID_ARGUMENT
    assert b"2048" in lib.rtkb_last_error()

"""The allocation-free FDK backprojection entry point
(rtkb_fdk_backproject_static_scratch), for callers that cannot allocate
device memory during a reconstruction: applications whose device memory is
reserved up front by their own allocator, and on-line loops that cannot take
cudaMalloc's implicit device synchronisation.

Called through the C ABI on two calls in a row (the second with a shorter
stack, so stale scratch from the first call must not leak into it) and
checked three ways: bit-identical to rtkb_fdk_backproject (the same kernels
run), within the FP32 tolerance of the FP64 oracle, and without growing the
library's device memory pool.  A tilted detector takes the generic per-voxel
path, whose path modes also live in the static array.  Collected last, so a
run that stops at the first failure has run every other test."""
import ctypes as C

import numpy as np
import pytest

from tests.gpu_util import REL_L2_TOL, pair_geometry, pair_image, rel_l2, to_np

pytestmark = pytest.mark.gpu


def _call(lib, fn, g, vd, pd, p, v0):
    import torch

    out = torch.empty_like(v0)
    rc = fn(g.handle, C.byref(vd), C.byref(pd), C.c_void_p(p.data_ptr()), C.c_void_p(v0.data_ptr()),
            C.c_void_p(out.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, lib.rtkb_last_error()
    return out


def _params(n, oop=0.0):
    return [(1000.0, 1536.0, i * 360.0 / n, 4.0, -2.0, oop) for i in range(n)]


@pytest.mark.parametrize("oop", [0.0, 7.0], ids=["circular", "tilted"])
def test_static_scratch_matches_allocating_entry_point(rtkb, oracle, oop):
    import torch

    lib = rtkb.load()
    rng = np.random.default_rng(7)
    cases = [(120, (96, 80, 88), (160, 128)), (40, (64, 72, 56), (128, 120))]  # second call: shorter stack
    for nproj, vsize, (nu, nv) in cases:
        gl, go = pair_geometry(rtkb, oracle, _params(nproj, oop))
        vd, vo = pair_image(rtkb, oracle, vsize, (1.5, 1.5, 1.5))
        pd, po = pair_image(rtkb, oracle, (nu, nv, nproj), (1.0, 1.0, 1.0))
        p_np = rng.uniform(-1, 1, size=(nproj, nv, nu)).astype(np.float32)
        v_np = rng.uniform(0, 1, size=(vsize[2], vsize[1], vsize[0])).astype(np.float32)
        p, v0 = torch.from_numpy(p_np).cuda(), torch.from_numpy(v_np).cuda()
        ref = _call(lib, lib.rtkb_fdk_backproject, gl, vd, pd, p, v0)
        torch.cuda.synchronize()
        rtkb.ops.trim_memory_pool()
        reserved_before = rtkb.ops.memory_pool_reserved()
        got = _call(lib, lib.rtkb_fdk_backproject_static_scratch, gl, vd, pd, p, v0)
        torch.cuda.synchronize()
        assert rtkb.ops.memory_pool_reserved() == reserved_before
        assert torch.equal(got, ref)
        want = oracle.backproject(go, vo, po, p_np.astype(np.float64), v_np.astype(np.float64), fdk=True)
        assert rel_l2(to_np(got), want) < REL_L2_TOL
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

"""Failure detection without a GPU fault.

* A bounded device-side wait that runs out: rtkb_wait_self_test waits, with
  the library's bounded mbarrier wait, on a barrier that nobody arrives at.
  With the wait limit lowered to a few thousand polls it gives up, records the
  timeout in the device status word and returns; rtkb_device_status reports
  RTKB_ERR_TIMEOUT once and then 0, and the context keeps working (a TMA-staged
  backprojection afterwards is correct).
* Allocation failures made on the host: rtkb_inject_allocation_failures makes
  the next scratch allocations fail as if the device were out of memory.  One
  failure takes the pool's trim-and-retry path (the call succeeds, and the
  memory the pool held from an earlier, larger call is returned first); two
  failures make the call fail with a CUDA status before any work is enqueued.
"""
import ctypes as C

import numpy as np
import pytest

from tests.gpu_util import REL_L2_TOL, pair_geometry, pair_image, rel_l2, to_gpu, to_np

pytestmark = pytest.mark.gpu


def _small_bp(rtkb, oracle):
    params = [(1000.0, 1536.0, i * 9.0, 3.0, -2.0) for i in range(40)]
    gl, go = pair_geometry(rtkb, oracle, params)
    vd, vo = pair_image(rtkb, oracle, (64, 48, 56), (2.0,) * 3)
    pd, po = pair_image(rtkb, oracle, (128, 96, 40), (1.5, 1.5, 1.0))
    p = np.random.default_rng(2).uniform(-1, 1, size=oracle.shape_of(po)).astype(np.float32).astype(np.float64)
    return gl, go, vd, vo, pd, po, p


def test_bounded_wait_times_out_and_context_survives(rtkb, oracle):
    import torch

    lib = rtkb.load()
    assert rtkb.ops.device_status() == 0
    prev = C.c_uint(0)
    assert lib.rtkb_set_wait_limit(4096, C.byref(prev)) == 0
    try:
        assert lib.rtkb_wait_self_test(None) == 0
        assert rtkb.ops.device_status() == rtkb._capi.RTKB_ERR_TIMEOUT
        assert rtkb.ops.device_status() == 0  # read and cleared
    finally:
        assert lib.rtkb_set_wait_limit(prev.value, None) == 0
    assert prev.value == 1 << 22
    assert lib.rtkb_set_wait_limit(0, None) == rtkb._capi.RTKB_ERR_INVALID_ARGUMENT
    gl, go, vd, vo, pd, po, p = _small_bp(rtkb, oracle)
    got = to_np(rtkb.ops.fdk_backproject(gl, vd, pd, to_gpu(p), torch.zeros(oracle.shape_of(vo), device="cuda")))
    assert rtkb.ops.device_status() == 0
    assert rel_l2(got, oracle.backproject(go, vo, po, p, fdk=True)) < REL_L2_TOL


def test_allocation_failure_trims_and_retries(rtkb, oracle):
    import torch

    lib = rtkb.load()
    g = rtkb.geometry.circular(16, 1000.0, 1536.0)
    big_vd = rtkb.make_desc((128, 96, 112), (1.0,) * 3)
    pd = rtkb.make_desc((96, 64, 16), (1.5, 1.5, 1.0))
    big = torch.rand((112, 96, 128), device="cuda")
    rtkb.ops.joseph_forward_project(g, big_vd, pd, big, torch.zeros((16, 64, 96), device="cuda"))
    torch.cuda.synchronize()
    held = rtkb.ops.memory_pool_reserved()
    gl, go, vd, vo, pd2, po, p = _small_bp(rtkb, oracle)
    assert lib.rtkb_inject_allocation_failures(1) == 0
    got = to_np(rtkb.ops.fdk_backproject(gl, vd, pd2, to_gpu(p), torch.zeros(oracle.shape_of(vo), device="cuda")))
    torch.cuda.synchronize()
    # the retry trimmed what the large forward projection had left reserved
    assert rtkb.ops.memory_pool_reserved() < held
    assert rel_l2(got, oracle.backproject(go, vo, po, p, fdk=True)) < REL_L2_TOL
    assert lib.rtkb_inject_allocation_failures(2) == 0
    out = torch.full(oracle.shape_of(vo), 7.0, device="cuda")
    with pytest.raises(rtkb.RtkbError):
        rtkb.ops.fdk_backproject(gl, vd, pd2, to_gpu(p), torch.zeros_like(out), out=out)
    torch.cuda.synchronize()
    assert bool((out == 7.0).all())  # nothing was enqueued
    assert lib.rtkb_inject_allocation_failures(0) == 0
    assert rtkb.ops.device_status() == 0

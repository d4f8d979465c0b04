"""The library's scratch memory pool (rtkb_memory_pool_reserved,
rtkb_trim_memory_pool): scratch freed by one call stays reserved across the
caller's synchronise for the next call, results do not depend on it, and a
trim returns it."""
import numpy as np
import pytest
import torch

from tests.gpu_util import to_np

pytestmark = pytest.mark.gpu


def test_scratch_pool_keeps_and_trims(rtkb):
    g = rtkb.geometry.circular(16, 1000.0, 1536.0)
    vd = rtkb.make_desc((64, 48, 56), (2.0, 2.0, 2.0))
    pd = rtkb.make_desc((96, 64, 16), (1.5, 1.5, 1.0))
    x = torch.rand((56, 48, 64), device="cuda", generator=torch.Generator(device="cuda").manual_seed(1))

    def forward():
        return rtkb.ops.joseph_forward_project(g, vd, pd, x, torch.zeros((16, 64, 96), device="cuda"))

    torch.cuda.synchronize()
    rtkb.ops.trim_memory_pool()
    first = to_np(forward())
    torch.cuda.synchronize()
    kept = rtkb.ops.memory_pool_reserved()
    # the projector's scratch: two volume copies and two quad-expanded copies
    nvox = 64 * 48 * 56
    assert kept >= 2 * 4 * nvox + 32 * nvox
    again = to_np(forward())
    torch.cuda.synchronize()
    assert rtkb.ops.memory_pool_reserved() == kept  # reused, not grown
    assert np.array_equal(first, again)
    assert rtkb.ops.trim_memory_pool() == 0
    assert rtkb.ops.memory_pool_reserved() == 0

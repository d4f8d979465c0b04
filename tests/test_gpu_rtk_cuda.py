"""RTK's own CUDA FDK back projector (CUDA_reconstruct_conebeam, compiled
unchanged from the RTK sources by oracle/rtk_cuda/Makefile) on a B200,
against the FP64 oracle and the product on the same filtered projections.

This runs the reference itself: it pins the oracle's half-pixel, index,
normalisation and FDK-weighting conventions to RTK's GPU code, at the
precision of RTK's texture-filtered interpolation (its texture unit keeps 8
fractional bits of the interpolation weights).  Skipped when the library was
not built (no RTK source tree where it was built)."""
import numpy as np
import pytest

from tests import phantoms
from tests.gpu_util import REL_L2_TOL, pair_geometry, pair_image, rel_l2, to_gpu, to_np

pytestmark = pytest.mark.gpu


def test_rtk_cuda_fdk_backprojection_agrees_with_oracle(rtkb, oracle):
    import torch

    from oracle import rtk_cuda

    if not rtk_cuda.available():
        pytest.skip("RTK's CUDA back projector was not built (no RTK source tree)")
    n = 90
    params = [(600.0, 1200.0, i * 360.0 / n, 6.0, -4.0, 0, 0, 20, 15) for i in range(n)]
    gl, go = pair_geometry(rtkb, oracle, params)
    vd, vo = pair_image(rtkb, oracle, (128, 128, 128), (2.0,) * 3, origin=(-127.0,) * 3)
    pd, po = pair_image(rtkb, oracle, (128, 128, n), (4.0,) * 3, origin=(-254.0,) * 3)
    sl = phantoms.shepp_logan(116.0)
    p = oracle.project_ellipsoids(go, po, sl)
    f = oracle.ramp_filter(po, oracle.fdk_weight(go, po, p), oracle.ramp_params()).astype(np.float32)
    f64 = f.astype(np.float64)
    ref = oracle.backproject(go, vo, po, f64, fdk=True)
    mats = rtk_cuda.filter_matrices(oracle, go, vo, po)
    d_proj = to_gpu(f64)
    vin = torch.zeros((128, 128, 128), device="cuda")
    vout = torch.zeros_like(vin)
    torch.cuda.synchronize()
    rtk_cuda.fdk_backproject((128, 128, n), (128, 128, 128), mats, vin.data_ptr(), vout.data_ptr(),
                             d_proj.data_ptr())
    torch.cuda.synchronize()
    got_rtk = to_np(vout)
    got = to_np(rtkb.ops.fdk_backproject(gl, vd, pd, d_proj, torch.zeros_like(vin)))
    fov = phantoms.fov_mask(go, vo, po)
    e_rtk = rel_l2(got_rtk[fov], ref[fov])
    e_prod = rel_l2(got[fov], ref[fov])
    # the reference's texture-filtered kernel follows the oracle's conventions
    # (a half-pixel or index slip would show at the 1e-1 level)
    assert e_rtk < 5e-3, e_rtk
    assert e_prod < REL_L2_TOL, e_prod
    assert rel_l2(got_rtk[fov], got[fov]) < 5e-3

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


# RTK's own CPU<->CUDA comparisons of these filters (test/rtkfdkprojweightcompcudatest.cxx,
# test/rtkparkershortscancompcudatest.cxx, test/rtkdisplaceddetectorcompcudatest.cxx) hold them to an
# error per pixel of 1e-5 of FP32 images; the oracle (FP64) is held to the same here.
WEIGHT_TOL = 1e-5


def _weighting_case(rtkb, oracle, params, size, index=(0, 0, 0)):
    gl, go = pair_geometry(rtkb, oracle, params)
    pd, po = pair_image(rtkb, oracle, size, (0.8, 0.9, 1.0), index=index)
    p = np.random.default_rng(len(params)).uniform(0.5, 1.5, size=oracle.shape_of(po)).astype(np.float32)
    return gl, go, pd, po, p


def _need_rtk():
    from oracle import rtk_cuda

    if not rtk_cuda.available():
        pytest.skip("RTK's CUDA filters were not built (no RTK source tree)")
    return rtk_cuda


def test_rtk_cuda_fdk_weighting_agrees_with_oracle(rtkb, oracle):
    """kernel_weight_projection (src/rtkCudaFDKWeightProjectionFilter.cu) on an
    irregular cone-beam stack (offsets, tilts, source offsets) with a shifted
    region, against the oracle's FDKWeightProjectionFilter restatement and the
    product."""
    import torch

    rtk_cuda = _need_rtk()
    params = [(1000.0 + 3 * i, 1536.0 - 2 * i, i * 7.3, 12.0 - i, -6.0 + 0.5 * i, 2.0, -1.5, 4.0, -3.0)
              for i in range(24)]
    gl, go, pd, po, p = _weighting_case(rtkb, oracle, params, (96, 80, 24), index=(-7, 3, 0))
    ref = oracle.fdk_weight(go, po, p.astype(np.float64))
    d_in = torch.from_numpy(p).cuda()
    d_out = torch.empty_like(d_in)
    torch.cuda.synchronize()
    rtk_cuda.fdk_weight(oracle, go, po, d_in.data_ptr(), d_out.data_ptr())
    torch.cuda.synchronize()
    assert rel_l2(to_np(d_out), ref) < WEIGHT_TOL
    assert rel_l2(to_np(rtkb.ops.fdk_weight(gl, pd, d_in)), ref) < WEIGHT_TOL


def test_rtk_cuda_parker_agrees_with_oracle(rtkb, oracle):
    """kernel_parker_weight (src/rtkCudaParkerShortScanImageFilter.cu) on a
    200 deg short scan with source and detector offsets, against the
    oracle's ParkerShortScanImageFilter restatement and the product."""
    import torch

    rtk_cuda = _need_rtk()
    params = [(1000.0, 1536.0, i * 200.0 / 90, 8.0, 0.0, 0.0, 0.0, 3.0, 0.0) for i in range(90)]
    gl, go, pd, po, p = _weighting_case(rtkb, oracle, params, (120, 16, 90))
    ref, short = oracle.parker_weight(go, po, p.astype(np.float64))
    assert short
    d_in = torch.from_numpy(p).cuda()
    d_out = torch.empty_like(d_in)
    torch.cuda.synchronize()
    assert rtk_cuda.parker_weight(oracle, go, po, d_in.data_ptr(), d_out.data_ptr())
    torch.cuda.synchronize()
    assert rel_l2(to_np(d_out), ref) < WEIGHT_TOL
    assert rel_l2(to_np(rtkb.ops.parker_short_scan(gl, pd, d_in)[0]), ref) < WEIGHT_TOL


@pytest.mark.parametrize("offset", [60.0, -45.0])
def test_rtk_cuda_displaced_detector_agrees_with_oracle(rtkb, oracle, offset):
    """kernel_displaced_weight (src/rtkCudaDisplacedDetectorImageFilter.cu) on
    a detector displaced to either side (output padded on the truncated
    side), against the oracle's DisplacedDetectorImageFilter restatement and
    the product."""
    import torch

    rtk_cuda = _need_rtk()
    params = [(1000.0, 1536.0, i * 4.0, offset, 0.0) for i in range(90)]
    gl, go, pd, po, p = _weighting_case(rtkb, oracle, params, (160, 12, 90))
    ref, i0, s0 = oracle.displaced_detector(go, po, p.astype(np.float64), pad=True)
    d_in = torch.from_numpy(p).cuda()
    d_out = torch.zeros((90, 12, s0), device="cuda")
    torch.cuda.synchronize()
    assert rtk_cuda.displaced_weight(oracle, go, po, d_in.data_ptr(), d_out.data_ptr()) == (i0, s0)
    torch.cuda.synchronize()
    assert rel_l2(to_np(d_out), ref) < WEIGHT_TOL
    assert rel_l2(to_np(rtkb.ops.displaced_detector(gl, pd, d_in)[0]), ref) < WEIGHT_TOL


# FP32 cuFFT against the FP64 oracle: measured ~1e-7 on these stacks
RAMP_TOL = 1e-5


@pytest.mark.parametrize("size,kw", [((128, 24, 8), {}), ((128, 24, 8), {"hann": 0.8, "truncation": 0.1}),
                                     ((128, 16, 6), {"truncation": 0.6}), ((96, 1, 6), {"shepplogan": 0.9}),
                                     ((100, 12, 5), {"cosine": 0.7, "truncation": 0.25, "pad": 1}),
                                     ((64, 20, 4), {"hann": 0.8, "hann_y": 0.8}),
                                     ((100, 13, 3), {"hann_y": 0.5, "truncation": 0.2}),
                                     ((96, 16, 4), {"hann_y": 1.0, "pad_y": 1}),
                                     ((100, 12, 5), {"gpf": 13}), ((99, 8, 3), {"gpf": 13, "pad": 1, "hann": 0.9}),
                                     ((120, 16, 4), {"gpf": 13, "truncation": 0.3}),
                                     ((64, 20, 4), {"gpf": 13, "hann_y": 0.8})])
def test_rtk_cuda_ramp_filter_agrees_with_oracle(rtkb, oracle, size, kw):
    """RTK's CUDA ramp filter (CUDA_padding + CUDA_fft_convolution: a 3-D
    cuFFT of the padded stack times the 1-D kernel spectrum, or the 2-D one
    of HannCutFrequencyY through multiply_kernel2D) against the oracle and
    the product; with a greatest prime factor of 13 (RTK built with FFTW) on
    padded lengths 200, 99, 240 and height 40, which cuFFT transforms as they
    are and the product embeds in power-of-two FFTs.  With truncation 0.6 the extent floor(0.6 * 128)
    = 76 exceeds the 64 columns of zero padding: RTK mirrors 64 columns with
    the weights of extent 76, and the case measures the margin by running
    RTK's kernels with the weights of extent 64 instead."""
    import torch

    from oracle import rtk_cuda

    _need_rtk()
    nu, nv, n = size
    pd, po = pair_image(rtkb, oracle, size, (0.8, 0.8, 1.0), origin=(-0.4 * (nu - 1), -0.4 * (nv - 1), 0.0))
    rng = np.random.default_rng(nu + nv)
    u = np.linspace(-1.0, 1.0, nu)
    p = (30.0 + 20.0 * np.cos(1.3 * u)[None, None, :] + rng.uniform(0.0, 5.0, size=(n, nv, nu))).astype(np.float32)
    params = oracle.ramp_params(**kw)
    ref = oracle.ramp_filter(po, p.astype(np.float64), params)
    d_in = torch.from_numpy(p).cuda()
    d_out = torch.empty_like(d_in)
    torch.cuda.synchronize()
    padded = rtk_cuda.fft_ramp(oracle, po, params, d_in.data_ptr(), d_out.data_ptr())
    torch.cuda.synchronize()
    got_rtk = to_np(d_out)
    e_rtk = rel_l2(got_rtk, ref)
    assert e_rtk < RAMP_TOL, e_rtk
    got = to_np(rtkb.ops.ramp_filter(pd, d_in, rtkb.ops.ramp_params(**kw)))
    assert rel_l2(got, ref) < RAMP_TOL
    assert rel_l2(got, got_rtk) < RAMP_TOL
    zeroext = (padded - nu) // 2
    ext = int(np.floor(kw.get("truncation", 0.0) * nu))
    if ext > zeroext:
        clamped = oracle.ramp_params(**dict(kw, truncation=(zeroext + 0.5) / nu))
        d_slip = torch.empty_like(d_in)
        rtk_cuda.fft_ramp(oracle, po, clamped, d_in.data_ptr(), d_slip.data_ptr())
        torch.cuda.synchronize()
        e_slip = rel_l2(to_np(d_slip), ref)
        assert e_slip > 100 * RAMP_TOL, e_slip

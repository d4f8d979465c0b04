"""Regularised CG (rtkb_regularized_cg), TV denoising (rtkb_tv_denoising_bpdq)
and the total-variation measure (rtkb_total_variation) against the FP64
oracle restating include/rtkRegularizedConjugateGradientConeBeamReconstructionFilter.hxx,
include/rtkDenoisingBPDQImageFilter.hxx and include/rtkTotalVariationImageFilter.hxx;
RTK's own tests (test/rtktotalvariationtest.cxx,
test/rtkregularizedconjugategradienttest.cxx case 1) through the GPU path."""
import numpy as np
import pytest
import torch

from tests.gpu_util import pair_geometry, pair_image, rel_l2, to_gpu, to_np
from tests.test_osem_oracle import _quality
from tests.test_regularized_cg_oracle import _rtk_regularized_cg_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("gamma,niter,dims", [(0.3, 1, (1, 1, 1)), (0.3, 2, (1, 1, 1)), (0.1, 10, (1, 1, 1)),
                                              (0.2, 6, (1, 0, 1)), (0.05, 4, (0, 1, 0))])
def test_tv_denoising_matches_oracle(rtkb, oracle, gamma, niter, dims):
    vd, vo = pair_image(rtkb, oracle, (21, 18, 16), (1.0, 2.0, 1.5))
    f = np.random.default_rng(niter).uniform(0.0, 1.0, oracle.shape_of(vo)).astype(np.float32).astype(np.float64)
    ref = oracle.tv_denoising_bpdq(vo, f, gamma, niter, dims=dims)
    got = to_np(rtkb.ops.tv_denoising_bpdq(vd, to_gpu(f), gamma, niter, dimensions=dims))
    assert rel_l2(got, ref) < 1e-6, rel_l2(got, ref)
    # in place gives the same values
    x = to_gpu(f)
    rtkb.ops.tv_denoising_bpdq(vd, x, gamma, niter, dimensions=dims, out=x)
    assert np.array_equal(to_np(x), got)


def test_total_variation_matches_oracle(rtkb, oracle):
    vd, vo = pair_image(rtkb, oracle, (33, 20, 17), (0.5, 1.0, 2.0))
    f = np.random.default_rng(5).normal(size=oracle.shape_of(vo)).astype(np.float32).astype(np.float64)
    ref = oracle.total_variation(vo, f)
    got = rtkb.ops.total_variation(vd, to_gpu(f))
    assert abs(got - ref) <= 1e-6 * abs(ref), (got, ref)


def test_rtk_total_variation_test_on_gpu(rtkb, oracle):
    """test/rtktotalvariationtest.cxx: 64^3 uniform(0, 1) at 4 mm, 100 BPDQ iterations at gamma 0.3 at least
    halve the total variation; and the oracle's volume."""
    vd, vo = pair_image(rtkb, oracle, (64, 64, 64), (4.0,) * 3, origin=(0.0,) * 3)
    f = np.random.default_rng(0).uniform(0.0, 1.0, oracle.shape_of(vo)).astype(np.float32).astype(np.float64)
    x = to_gpu(f)
    out = rtkb.ops.tv_denoising_bpdq(vd, x, 0.3, 100)
    before, after = rtkb.ops.total_variation(vd, x), rtkb.ops.total_variation(vd, out)
    assert after < before / 2, (before, after)
    ref = oracle.tv_denoising_bpdq(vo, f, 0.3, 100)
    assert rel_l2(to_np(out), ref) < 1e-5, rel_l2(to_np(out), ref)


def _problem(rtkb, oracle, n=20, seed=0):
    params = [(600.0, 900.0, i * 360.0 / n) for i in range(n)]
    gl, go = pair_geometry(rtkb, oracle, params)
    vd, vo = pair_image(rtkb, oracle, (24, 20, 22), (6.0,) * 3)
    pd, po = pair_image(rtkb, oracle, (48, 40, n), (4.0, 4.0, 1.0))
    rng = np.random.default_rng(seed)
    truth = rng.uniform(0.0, 1.0, size=oracle.shape_of(vo))
    p = oracle.joseph_forward(go, vo, truth, po).astype(np.float32).astype(np.float64)
    return gl, go, vd, vo, pd, po, p


@pytest.mark.parametrize("kw", [
    dict(main_loop_iterations=2, cg_iterations=3, gamma_tv=0.05, tv_iterations=3),
    dict(main_loop_iterations=3, cg_iterations=2, tikhonov=20.0, gamma=5.0, gamma_tv=0.02, tv_iterations=4,
         tv_dimensions=(True, True, False), soft_threshold_on_image=True, soft_threshold=0.01),
    dict(main_loop_iterations=2, cg_iterations=3, positivity=False, tv=False),
])
def test_regularized_cg_matches_oracle(rtkb, oracle, kw):
    gl, go, vd, vo, pd, po, p = _problem(rtkb, oracle)
    x0 = np.zeros(oracle.shape_of(vo))
    okw = dict(kw)
    okw["main_iterations"] = okw.pop("main_loop_iterations")
    if "tv_dimensions" in okw:
        okw["tv_dims"] = okw.pop("tv_dimensions")
    if "soft_threshold_on_image" in okw:
        okw["soft_threshold_value"] = okw.pop("soft_threshold")
        okw["soft_threshold"] = okw.pop("soft_threshold_on_image")
    ref = oracle.regularized_cg(go, vo, po, p, x0, **okw)
    x = to_gpu(x0)
    rtkb.ops.regularized_cg(gl, vd, pd, to_gpu(p), x, **kw)
    assert rtkb.ops.device_status() == 0
    # FP32 CG runs (restarted each main iteration) through the thresholds against FP64
    assert rel_l2(to_np(x), ref) < 2e-4, rel_l2(to_np(x), ref)


def test_regularized_cg_weights_without_displaced_detector(rtkb, oracle):
    gl, go, vd, vo, pd, po, p = _problem(rtkb, oracle, seed=3)
    w = np.random.default_rng(4).uniform(0.5, 1.5, oracle.shape_of(po)).astype(np.float32).astype(np.float64)
    x0 = np.zeros(oracle.shape_of(vo))
    ref = oracle.regularized_cg(go, vo, po, p, x0, main_iterations=2, cg_iterations=3, weights=w, gamma_tv=0.05,
                                tv_iterations=2)
    x = to_gpu(x0)
    rtkb.ops.regularized_cg(gl, vd, pd, to_gpu(p), x, weights=to_gpu(w), main_loop_iterations=2, cg_iterations=3,
                            gamma_tv=0.05, tv_iterations=2, displaced_detector=False)
    assert rel_l2(to_np(x), ref) < 2e-4, rel_l2(to_np(x), ref)
    with pytest.raises(rtkb.RtkbError, match="invalid regularised CG parameters"):
        rtkb.ops.regularized_cg(gl, vd, pd, to_gpu(p), x, tv_iterations=0)


def test_rtk_regularized_cg_case_1_on_gpu(rtkb, oracle):
    """test/rtkregularizedconjugategradienttest.cxx case 1 (positivity + TV) through rtkb_regularized_cg."""
    g, vol, proj, p, ref = _rtk_regularized_cg_case()
    n = proj.size[2]
    gl, _ = pair_geometry(rtkb, oracle, [(600.0, 1200.0, i * 360.0 / n) for i in range(n)])
    vd = rtkb.make_desc((64, 64, 64), (4.0,) * 3, origin=(-127.0,) * 3)
    pd = rtkb.make_desc((64, 64, n), (8.0,) * 3, origin=(-255.0,) * 3)
    pf = p.astype(np.float32).astype(np.float64)
    x = to_gpu(np.zeros(oracle.shape_of(vol)))
    rtkb.ops.regularized_cg(gl, vd, pd, to_gpu(pf), x, weights=to_gpu(np.ones(oracle.shape_of(proj))),
                            main_loop_iterations=2, cg_iterations=4, gamma_tv=1.0, tv_iterations=3)
    got = to_np(x)
    err, psnr = _quality(got, ref)
    assert err < 0.05 and psnr > 23.0, (err, psnr)
    want = oracle.regularized_cg(g, vol, proj, pf, np.zeros(oracle.shape_of(vol)), main_iterations=2,
                                 cg_iterations=4, gamma_tv=1.0, tv_iterations=3)
    assert rel_l2(got, want) < 2e-4, rel_l2(got, want)


def test_regularized_cg_support_mask_matches_oracle(rtkb, oracle):
    gl, go, vd, vo, pd, po, p = _problem(rtkb, oracle, seed=6)
    mask = np.zeros(oracle.shape_of(vo))
    mask[2:20, 3:17, 2:22] = 1.0
    x0 = np.zeros(oracle.shape_of(vo))
    ref = oracle.regularized_cg(go, vo, po, p, x0, main_iterations=2, cg_iterations=3, gamma_tv=0.05, tv_iterations=3,
                                mask=mask)
    x = to_gpu(x0)
    rtkb.ops.regularized_cg(gl, vd, pd, to_gpu(p), x, main_loop_iterations=2, cg_iterations=3, gamma_tv=0.05,
                            tv_iterations=3, support_mask=to_gpu(mask))
    assert rel_l2(to_np(x), ref) < 2e-4, rel_l2(to_np(x), ref)

"""SART (rtkb_sart) and the ray-box lengths it normalises by
(rtkb_ray_box_lengths) against the FP64 oracle restating
include/rtkSARTConeBeamReconstructionFilter.hxx with the Joseph forward and
voxel-based back projectors, on the same processing order."""
import numpy as np
import pytest
import torch

from tests.gpu_util import pair_geometry, pair_image, rel_l2, to_gpu, to_np

pytestmark = pytest.mark.gpu


def test_ray_box_lengths_match_oracle(rtkb, oracle):
    params = [(700.0, 1100.0, i * 360.0 / 12, 25.0, -4.0, 3.0, 2.0, 1.5, -2.5) for i in range(12)]
    gl, go = pair_geometry(rtkb, oracle, params)
    c, s = np.cos(0.2), np.sin(0.2)
    rot = np.array([[c, 0.0, s], [0.0, 1.0, 0.0], [-s, 0.0, c]])
    vd, vo = pair_image(rtkb, oracle, (30, 22, 26), (3.0, 2.5, 3.5), direction=rot)
    pd, po = pair_image(rtkb, oracle, (64, 48, 12), (2.0, 2.0, 1.0), index=(-10, 3, 0))
    got = to_np(rtkb.ops.ray_box_lengths(gl, vd, pd))
    ref = oracle.ray_box(go, vo, po)
    assert ref.max() > 0 and (ref == 0).any()  # some rays miss the box
    assert rel_l2(got, ref) < 1e-6, rel_l2(got, ref)


def _problem(rtkb, oracle, n=16, offset=30.0, seed=0):
    params = [(600.0, 900.0, i * 360.0 / n, offset, 0.0) for i in range(n)]
    gl, go = pair_geometry(rtkb, oracle, params)
    vd, vo = pair_image(rtkb, oracle, (24, 20, 22), (6.0,) * 3)
    pd, po = pair_image(rtkb, oracle, (48, 40, n), (4.0, 4.0, 1.0))
    rng = np.random.default_rng(seed)
    truth = rng.uniform(0.0, 1.0, size=oracle.shape_of(vo))
    p = oracle.joseph_forward(go, vo, truth, po).astype(np.float32).astype(np.float64)
    return gl, go, vd, vo, pd, po, p, rng.permutation(n)


@pytest.mark.parametrize("subset,positivity,displaced", [(1, False, True), (4, True, True), (3, False, False)])
def test_sart_matches_oracle(rtkb, oracle, subset, positivity, displaced):
    gl, go, vd, vo, pd, po, p, order = _problem(rtkb, oracle, seed=subset)
    ref = oracle.sart(go, vo, po, p, 2, order, lam=0.3, positivity=positivity, subset=subset,
                      displaced_detector=displaced)
    x = torch.zeros(oracle.shape_of(vo), device="cuda")
    rtkb.ops.sart(gl, vd, pd, to_gpu(p), x, niter=2, lam=0.3, positivity=positivity, subset=subset,
                  displaced_detector=displaced, order=order)
    assert rtkb.ops.device_status() == 0
    assert np.abs(ref).max() > 0
    # FP32 projectors over 2 x 16 sequential updates against FP64
    assert rel_l2(to_np(x), ref) < 2e-4, rel_l2(to_np(x), ref)
    if positivity:
        assert to_np(x).min() >= 0.0


def test_sart_default_order_reduces_the_data_misfit(rtkb, oracle):
    gl, go, vd, vo, pd, po, p, _ = _problem(rtkb, oracle, seed=7)
    x = torch.zeros(oracle.shape_of(vo), device="cuda")
    rtkb.ops.sart(gl, vd, pd, to_gpu(p), x, niter=3, seed=11)
    fp = to_np(rtkb.ops.joseph_forward_project(gl, vd, pd, x, to_gpu(np.zeros(oracle.shape_of(po)))))
    assert np.linalg.norm(fp - p) < 0.3 * np.linalg.norm(p)
    with pytest.raises(rtkb.RtkbError, match="permutation"):
        rtkb.ops.sart(gl, vd, pd, to_gpu(p), x, order=np.zeros(pd.size[2], dtype=np.int32))

"""Iterative FDK (rtkb_iterative_fdk) against the oracle composed from its
restated filters (include/rtkIterativeFDKConeBeamReconstructionFilter.hxx):
displaced detector with padding, short scans, positivity; and RTK's own test
(test/rtkiterativefdktest.cxx) through the GPU path."""
import numpy as np
import pytest

from tests import phantoms
from tests.gpu_util import pair_geometry, pair_image, rel_l2, to_gpu, to_np

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("arc,offset,positivity,lam", [(360.0, 40.0, True, 0.3), (220.0, 0.0, False, 0.5),
                                                       (360.0, 0.0, False, 0.0)])
def test_iterative_fdk_matches_oracle(rtkb, oracle, arc, offset, positivity, lam):
    n = 60
    gl, go = pair_geometry(rtkb, oracle, [(700.0, 1100.0, i * arc / n, offset, 0.0) for i in range(n)])
    vd, vo = pair_image(rtkb, oracle, (48, 40, 44), (4.0,) * 3)
    pd, po = pair_image(rtkb, oracle, (96, 64, n), (3.0, 3.0, 1.0))
    ell = phantoms.random_ellipsoids(6, 3, centre_radius=30.0, axis_range=(10.0, 50.0))
    p = oracle.project_ellipsoids(go, po, ell).astype(np.float32).astype(np.float64)
    x0 = np.zeros(oracle.shape_of(vo))
    ref = oracle.iterative_fdk(go, vo, po, p, x0, niter=3, lam=lam, positivity=positivity, displaced=True,
                               short_scan=True)
    x = to_gpu(x0)
    rtkb.ops.iterative_fdk(gl, vd, pd, to_gpu(p), x, niter=3, lam=lam, positivity=positivity)
    assert rtkb.ops.device_status() == 0
    assert rel_l2(to_np(x), ref) < 1e-4, rel_l2(to_np(x), ref)
    if lam == 0.0:  # no correction: one FDK
        one = oracle.iterative_fdk(go, vo, po, p, x0, niter=1)
        assert rel_l2(ref, one) < 1e-12


def test_rtk_iterative_fdk_test_on_gpu(rtkb, oracle):
    """test/rtkiterativefdktest.cxx: 3 iterations, err/px < 0.027 and PSNR > 27 dB in the field of view."""
    n = 180
    gl, go = pair_geometry(rtkb, oracle, [(600.0, 1200.0, i * 360.0 / n, 0, 0, 0, 0, 20, 15) for i in range(n)])
    vd, vo = pair_image(rtkb, oracle, (128, 128, 128), (2.0,) * 3, origin=(-127.0,) * 3)
    pd, po = pair_image(rtkb, oracle, (128, 128, n), (4.0,) * 3, origin=(-254.0,) * 3)
    sl = phantoms.shepp_logan(116.0)
    p = oracle.project_ellipsoids(go, po, sl).astype(np.float32).astype(np.float64)
    ref = oracle.draw_ellipsoids(vo, sl)
    x = to_gpu(np.zeros(oracle.shape_of(vo)))
    rtkb.ops.iterative_fdk(gl, vd, pd, to_gpu(p), x, niter=3)
    got = to_np(x) * phantoms.fov_mask(go, vo, po)
    err, psnr, ok = phantoms.check_image_quality(got, ref, 0.027, 27.0, 2.0)
    assert ok, (err, psnr)

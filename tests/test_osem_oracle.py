"""CPU checks of the oracle's OSEM pieces (test infrastructure).

De Pierro's factor on inputs whose answer is worked out by hand, and RTK's own
OSEM test (test/rtkosemtest.cxx:27-164): a 60 mm sphere of density 1 imaged by
60 projections, reconstructed from a volume of ones, with the test's error per
pixel and PSNR thresholds (CheckImageQuality, test/rtkTest.h:39-95).  RTK
shuffles the projections with std::default_random_engine, whose sequence the
C++ standard leaves open, so a seeded permutation stands in for its order.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O


def test_de_pierro_hand_worked():
    O.build()
    vol = O.image((3, 3, 3), (1.0, 1.0, 1.0))
    xk = np.ones((3, 3, 3))
    upd = np.full((3, 3, 3), 2.0)
    norm = np.full((3, 3, 3), 5.0)
    beta = 0.01
    r = O.de_pierro(vol, xk, upd, norm, beta)
    # neighbourhood sum: 26 x the centre + the neighbours inside the image
    for idx, k in (((1, 1, 1), 26 + 26), ((0, 0, 0), 26 + 7), ((0, 1, 1), 26 + 17), ((0, 0, 1), 26 + 11)):
        a = 5.0 - beta * k
        b = 8 * beta * 26 * 2.0
        assert r[idx] == pytest.approx((a + math.sqrt(a * a + b)) / 2, rel=1e-14)
    # beta = 0: the factor is the normalisation volume itself (classic ML-EM)
    n = np.random.default_rng(0).uniform(0.0, 3.0, size=(3, 3, 3))
    np.testing.assert_allclose(O.de_pierro(vol, xk, upd, n, 0.0), n, rtol=1e-15)
    # no normalisation input: a volume of ones
    np.testing.assert_allclose(O.de_pierro(vol, xk, upd, None, 0.0), 1.0, rtol=1e-15)


def _rtk_osem_case():
    """test/rtkosemtest.cxx:39-121 at its full size."""
    n = 60
    g = O.Geometry()
    for i in range(n):
        g.add_projection(600.0, 1200.0, i * 360.0 / n)
    vol = O.image((34, 34, 34), (4.0, 4.0, 4.0), origin=(-67.0, -67.0, -67.0))
    proj = O.image((34, 34, n), (8.0, 8.0, 8.0), origin=(-135.0, -135.0, -135.0))
    sphere = np.zeros(16)
    sphere[3:6] = 60.0
    sphere[6:15] = np.eye(3).reshape(9)
    sphere[15] = 1.0
    p = O.project_ellipsoids(g, proj, sphere[None])
    ref = O.draw_ellipsoids(vol, sphere[None])
    return g, vol, proj, p, ref, np.random.default_rng(2).permutation(n)


def _quality(recon, ref, ref_value=2.0):
    err = np.abs(ref - recon).sum() / ref.size
    mse = ((ref - recon) ** 2).sum() / ref.size
    return err, 20 * math.log10(ref_value) - 10 * math.log10(mse)


@pytest.mark.parametrize("niter,subset,joseph_bp,max_err", [
    (10, 60, False, 0.047),  # case 1: ML-EM, voxel-based back projector, 10 iterations
    (3, 10, True, 0.032),    # case 2: Joseph back projector, 10 projections per subset
    (3, 10, False, 0.032),   # case 3: voxel-based back projector, 10 projections per subset
])
def test_oracle_osem_passes_rtk_osem_test(niter, subset, joseph_bp, max_err):
    O.build()
    g, vol, proj, p, ref, order = _rtk_osem_case()
    x = O.osem(g, vol, proj, p, niter, order, np.ones(O.shape_of(vol)), subset=subset, joseph_bp=joseph_bp)
    err, psnr = _quality(x, ref)
    assert err < max_err and psnr > 25.0, (err, psnr)
    assert x.min() >= 0.0  # EM updates keep a non-negative start non-negative

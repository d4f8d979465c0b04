"""CPU checks of the oracle's TV denoising and regularised CG (test
infrastructure), against RTK's own tests: test/rtktotalvariationtest.cxx
(BPDQ TV denoising of a random volume must at least halve its total
variation) and test/rtkregularizedconjugategradienttest.cxx case 1
(positivity + TV, CheckImageQuality thresholds), plus identities of the
BPDQ iteration."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.test_osem_oracle import _quality


def test_tv_denoising_halves_total_variation():
    """test/rtktotalvariationtest.cxx: 64^3 uniform(0, 1) at 4 mm, 100 iterations, gamma 0.3."""
    O.build()
    vol = O.image((64, 64, 64), (4.0, 4.0, 4.0), origin=(0.0, 0.0, 0.0))
    f = np.random.default_rng(0).uniform(0.0, 1.0, O.shape_of(vol))
    out = O.tv_denoising_bpdq(vol, f, 0.3, 100)
    before, after = O.total_variation(vol, f), O.total_variation(vol, out)
    assert after < before / 2, (before, after)


def test_tv_denoising_identities():
    O.build()
    vol = O.image((9, 7, 8), (1.0, 2.0, 0.5))
    f = np.random.default_rng(1).normal(size=O.shape_of(vol))
    # gamma = 0: every dual vector is projected to 0, the output is the input
    np.testing.assert_allclose(O.tv_denoising_bpdq(vol, f, 0.0, 5), f, rtol=0, atol=1e-15)
    # a constant image has no variation to remove
    c = np.full(O.shape_of(vol), 3.25)
    np.testing.assert_allclose(O.tv_denoising_bpdq(vol, c, 0.7, 5), c, rtol=0, atol=1e-14)
    # one processed dimension: rows along x are denoised independently of y and z
    out = O.tv_denoising_bpdq(vol, f, 0.5, 6, dims=(True, False, False))
    row = O.image((9, 1, 1), (1.0, 2.0, 0.5))
    ref = O.tv_denoising_bpdq(row, np.ascontiguousarray(f[3, 2, :]).reshape(1, 1, 9), 0.5, 6,
                              dims=(True, False, False))
    np.testing.assert_allclose(out[3, 2, :], ref.reshape(9), rtol=1e-13)


def _rtk_regularized_cg_case():
    """test/rtkregularizedconjugategradienttest.cxx:38-103 at its full size."""
    n = 90
    g = O.Geometry()
    for i in range(n):
        g.add_projection(600.0, 1200.0, i * 360.0 / n)
    vol = O.image((64, 64, 64), (4.0, 4.0, 4.0), origin=(-127.0, -127.0, -127.0))
    proj = O.image((64, 64, n), (8.0, 8.0, 8.0), origin=(-255.0, -255.0, -255.0))
    sphere = np.zeros(16)
    sphere[3:6] = 90.0
    sphere[6:15] = np.eye(3).reshape(9)
    sphere[15] = 1.0
    return g, vol, proj, O.project_ellipsoids(g, proj, sphere[None]), O.draw_ellipsoids(vol, sphere[None])


def test_oracle_regularized_cg_passes_rtk_case_1():
    """Positivity + TV: 2 main iterations of 4 CG iterations, gamma_TV 1, 3 TV iterations."""
    O.build()
    g, vol, proj, p, ref = _rtk_regularized_cg_case()
    x = O.regularized_cg(g, vol, proj, p, np.zeros(O.shape_of(vol)), main_iterations=2, cg_iterations=4,
                         gamma_tv=1.0, tv_iterations=3)
    err, psnr = _quality(x, ref)
    assert err < 0.05 and psnr > 23.0, (err, psnr)
    # the thresholds have teeth: a single CG iteration is far from the sphere
    x1 = O.regularized_cg(g, vol, proj, p, np.zeros(O.shape_of(vol)), main_iterations=1, cg_iterations=1,
                          gamma_tv=1.0, tv_iterations=3)
    assert _quality(x1, ref)[0] > 0.05


def test_cg_support_mask_identities():
    """ConjugateGradientConeBeamReconstructionFilter::SetSupportMask: a mask of ones changes nothing (bit for bit); a
    binary mask confines the solution to its support and still reduces the masked normal-equation residual."""
    O.build()
    n = 16
    g = O.Geometry()
    for i in range(n):
        g.add_projection(600.0, 900.0, i * 360.0 / n)
    vol = O.image((20, 18, 16), (6.0,) * 3)
    proj = O.image((40, 32, n), (4.0, 4.0, 1.0))
    truth = np.random.default_rng(0).uniform(0.0, 1.0, O.shape_of(vol))
    p = O.joseph_forward(g, vol, truth, proj)
    x, res = O.cg_joseph(g, vol, proj, p, 3)
    x1, res1 = O.cg_joseph(g, vol, proj, p, 3, mask=np.ones(O.shape_of(vol)))
    assert np.array_equal(x, x1) and np.array_equal(res, res1)
    m = np.zeros(O.shape_of(vol))
    m[3:13, 4:14, 5:15] = 1.0
    xm, resm = O.cg_joseph(g, vol, proj, p, 3, mask=m)
    assert np.all(xm[m == 0] == 0.0) and np.abs(xm[m == 1]).max() > 0
    assert resm[-1] < 0.5 * resm[0]

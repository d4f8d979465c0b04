"""OSEM (rtkb_osem) and De Pierro's regularisation (rtkb_de_pierro_regularization)
against the FP64 oracle restating include/rtkOSEMConeBeamReconstructionFilter.hxx
and include/rtkDePierroRegularizationImageFilter.hxx projection by projection,
on the same processing order; and RTK's own OSEM test (test/rtkosemtest.cxx)
through the GPU path with its quality thresholds."""
import numpy as np
import pytest
import torch

from tests.gpu_util import pair_geometry, pair_image, rel_l2, to_gpu, to_np
from tests.test_osem_oracle import _quality

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("beta,with_norm", [(0.0, True), (0.01, True), (0.05, False)])
def test_de_pierro_matches_oracle(rtkb, oracle, beta, with_norm):
    vd, vo = pair_image(rtkb, oracle, (21, 18, 16), (1.0, 1.0, 1.0))
    rng = np.random.default_rng(3)
    shape = oracle.shape_of(vo)
    xk = rng.uniform(0.0, 1.0, shape)
    upd = rng.uniform(0.0, 2.0, shape)
    norm = rng.uniform(1.0, 3.0, shape) if with_norm else None
    # the float32 inputs the device sees
    xk, upd = xk.astype(np.float32).astype(np.float64), upd.astype(np.float32).astype(np.float64)
    if norm is not None:
        norm = norm.astype(np.float32).astype(np.float64)
    ref = oracle.de_pierro(vo, xk, upd, norm, beta)
    got = to_np(rtkb.ops.de_pierro_regularization(vd, to_gpu(xk), to_gpu(upd),
                                                  None if norm is None else to_gpu(norm), beta=beta))
    # float32 arithmetic of the filter; with beta = 0.05 A = norm - beta K goes negative and
    # A + sqrt(A^2 + B) cancels, which costs a few more float32 ulps
    assert rel_l2(got, ref) < (1e-6 if beta <= 0.01 else 1e-5), rel_l2(got, ref)


def _problem(rtkb, oracle, n=16, first=0, extra=0, proj_direction=None, seed=0):
    params = [(600.0, 900.0, i * 360.0 / (n + extra), 20.0, -5.0) for i in range(n + extra)]
    gl, go = pair_geometry(rtkb, oracle, params)
    vd, vo = pair_image(rtkb, oracle, (24, 20, 22), (6.0,) * 3)
    pd, po = pair_image(rtkb, oracle, (48, 40, n), (4.0, 4.0, 1.0), index=(0, 0, first), direction=proj_direction)
    rng = np.random.default_rng(seed)
    truth = rng.uniform(0.2, 1.0, size=oracle.shape_of(vo))
    p = oracle.joseph_forward(go, vo, truth, po).astype(np.float32).astype(np.float64)
    return gl, go, vd, vo, pd, po, p, rng.permutation(n)


@pytest.mark.parametrize("subset,beta,bp,store", [
    (1, 0.0, "voxel", True),     # RTK's defaults (one projection per subset)
    (4, 0.0, "voxel", False),
    (5, 0.01, "voxel", True),    # ragged last subset, De Pierro term
    (4, 0.01, "joseph", True),
    (16, 0.0, "joseph", False),  # ML-EM
])
def test_osem_matches_oracle(rtkb, oracle, subset, beta, bp, store):
    gl, go, vd, vo, pd, po, p, order = _problem(rtkb, oracle, seed=subset)
    x0 = np.ones(oracle.shape_of(vo))
    ref = oracle.osem(go, vo, po, p, 2, order, x0, subset=subset, beta=beta, joseph_bp=(bp == "joseph"))
    x = to_gpu(x0)
    rtkb.ops.osem(gl, vd, pd, to_gpu(p), x, niter=2, subset=subset, beta=beta, store_normalization=store,
                  backprojector=bp, order=order)
    assert rtkb.ops.device_status() == 0
    assert ref.min() >= 0.0 and ref.max() > 0
    # FP32 projectors and multiplicative updates over 2 x 16 projections against FP64
    assert rel_l2(to_np(x), ref) < 1e-4, rel_l2(to_np(x), ref)


def test_osem_stack_offset_and_projection_direction(rtkb, oracle):
    """A stack that starts at geometry entry 3, and a projection direction that
    mixes the stack axis into v (the projection-by-projection path)."""
    gl, go, vd, vo, pd, po, p, order = _problem(rtkb, oracle, n=12, first=3, extra=5, seed=4)
    x0 = np.ones(oracle.shape_of(vo))
    ref = oracle.osem(go, vo, po, p, 2, order, x0, subset=3)
    x = to_gpu(x0)
    rtkb.ops.osem(gl, vd, pd, to_gpu(p), x, niter=2, subset=3, order=order)
    assert rel_l2(to_np(x), ref) < 1e-4, rel_l2(to_np(x), ref)

    c, s = np.cos(0.3), np.sin(0.3)
    tilt = np.array([[1.0, 0.0, 0.0], [0.0, c, -s], [0.0, s, c]])
    gl, go, vd, vo, pd, po, p, order = _problem(rtkb, oracle, n=12, first=2, extra=2, proj_direction=tilt, seed=5)
    ref = oracle.osem(go, vo, po, p, 2, order, x0, subset=4, beta=0.01)
    x = to_gpu(x0)
    rtkb.ops.osem(gl, vd, pd, to_gpu(p), x, niter=2, subset=4, beta=0.01, order=order)
    assert rel_l2(to_np(x), ref) < 1e-4, rel_l2(to_np(x), ref)


def test_osem_stored_normalisation_is_exact(rtkb, oracle):
    """Storing BP(1) per subset changes no value (the voxel-based back projector is deterministic)."""
    gl, go, vd, vo, pd, po, p, order = _problem(rtkb, oracle, seed=9)
    outs = []
    for store in (True, False):
        x = to_gpu(np.ones(oracle.shape_of(vo)))
        rtkb.ops.osem(gl, vd, pd, to_gpu(p), x, niter=3, subset=4, beta=0.01, store_normalization=store,
                      order=order)
        outs.append(to_np(x))
    assert np.array_equal(outs[0], outs[1])


def test_osem_errors(rtkb, oracle):
    gl, go, vd, vo, pd, po, p, order = _problem(rtkb, oracle, seed=1)
    x = to_gpu(np.ones(oracle.shape_of(vo)))
    bad = order.copy()
    bad[0] = bad[1]
    with pytest.raises(rtkb.RtkbError, match="permutation"):
        rtkb.ops.osem(gl, vd, pd, to_gpu(p), x, order=bad)
    with pytest.raises(ValueError, match="backprojector"):
        rtkb.ops.osem(gl, vd, pd, to_gpu(p), x, backprojector="cuda")
    with pytest.raises(rtkb.RtkbError, match="invalid OSEM parameters"):
        rtkb.ops.osem(gl, vd, pd, to_gpu(p), x, subset=0)


@pytest.mark.parametrize("niter,subset,bp,max_err", [(10, 60, "voxel", 0.047), (3, 10, "joseph", 0.032),
                                                     (3, 10, "voxel", 0.032)])
def test_rtk_osem_test_cases_on_gpu(rtkb, oracle, niter, subset, bp, max_err):
    """test/rtkosemtest.cxx cases 1-3 through rtkb_osem: RTK's thresholds, and the oracle's volume."""
    n = 60
    params = [(600.0, 1200.0, i * 360.0 / n) for i in range(n)]
    gl, go = pair_geometry(rtkb, oracle, params)
    vd, vo = pair_image(rtkb, oracle, (34, 34, 34), (4.0,) * 3, origin=(-67.0,) * 3)
    pd, po = pair_image(rtkb, oracle, (34, 34, n), (8.0,) * 3, origin=(-135.0,) * 3)
    sphere = np.zeros(16)
    sphere[3:6] = 60.0
    sphere[6:15] = np.eye(3).reshape(9)
    sphere[15] = 1.0
    p = oracle.project_ellipsoids(go, po, sphere[None]).astype(np.float32).astype(np.float64)
    ref = oracle.draw_ellipsoids(vo, sphere[None])
    order = np.random.default_rng(2).permutation(n)
    x = to_gpu(np.ones(oracle.shape_of(vo)))
    rtkb.ops.osem(gl, vd, pd, to_gpu(p), x, niter=niter, subset=subset, backprojector=bp, order=order)
    got = to_np(x)
    err, psnr = _quality(got, ref)
    assert err < max_err and psnr > 25.0, (err, psnr)
    want = oracle.osem(go, vo, po, p, niter, order, np.ones(oracle.shape_of(vo)), subset=subset,
                       joseph_bp=(bp == "joseph"))
    assert rel_l2(got, want) < 1e-4, rel_l2(got, want)

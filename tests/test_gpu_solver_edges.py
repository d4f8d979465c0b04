"""Edge cases of the solvers and filters beyond the projector pair, against the
FP64 oracle: thin and ragged volumes for TV denoising, OSEM with no iterations,
one projection and subsets larger than the stack, the regularised CG without
main or CG iterations, raw-count conversion of a single pixel, a constant image
and an unaligned buffer, and empty images refused."""
import numpy as np
import pytest
import torch

from tests.gpu_util import pair_geometry, pair_image, rel_l2, to_gpu, to_np
from tests.test_gpu_preprocess import _u16

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("size", [(1, 1, 7), (5, 1, 1), (3, 2, 1), (1, 9, 4)])
def test_tv_denoising_thin_volumes(rtkb, oracle, size):
    vd, vo = pair_image(rtkb, oracle, size, (1.0, 2.0, 0.5))
    f = np.random.default_rng(sum(size)).uniform(0.0, 1.0, oracle.shape_of(vo)).astype(np.float32).astype(np.float64)
    ref = oracle.tv_denoising_bpdq(vo, f, 0.2, 5)
    got = to_np(rtkb.ops.tv_denoising_bpdq(vd, to_gpu(f), 0.2, 5))
    assert rel_l2(got, ref) < 1e-6, rel_l2(got, ref)


def _osem_problem(rtkb, oracle, n):
    gl, go = pair_geometry(rtkb, oracle, [(600.0, 900.0, i * 360.0 / n) for i in range(n)])
    vd, vo = pair_image(rtkb, oracle, (20, 18, 16), (6.0,) * 3)
    pd, po = pair_image(rtkb, oracle, (40, 32, n), (4.0, 4.0, 1.0))
    truth = np.random.default_rng(n).uniform(0.2, 1.0, size=oracle.shape_of(vo))
    p = oracle.joseph_forward(go, vo, truth, po).astype(np.float32).astype(np.float64)
    return gl, go, vd, vo, pd, po, p


def test_osem_edges(rtkb, oracle):
    gl, go, vd, vo, pd, po, p = _osem_problem(rtkb, oracle, 12)
    x0 = np.ones(oracle.shape_of(vo))
    x = to_gpu(x0)
    rtkb.ops.osem(gl, vd, pd, to_gpu(p), x, niter=0)
    assert np.array_equal(to_np(x), x0)
    # a subset size above the stack size is one subset of the whole stack
    order = np.arange(12)[::-1].copy()
    ref = oracle.osem(go, vo, po, p, 2, order, x0, subset=12)
    x = to_gpu(x0)
    rtkb.ops.osem(gl, vd, pd, to_gpu(p), x, niter=2, subset=100, order=order)
    assert rel_l2(to_np(x), ref) < 1e-4, rel_l2(to_np(x), ref)
    # a one-projection stack
    gl, go, vd, vo, pd, po, p = _osem_problem(rtkb, oracle, 1)
    x = to_gpu(x0)
    rtkb.ops.osem(gl, vd, pd, to_gpu(p), x, niter=3, beta=0.01)
    ref = oracle.osem(go, vo, po, p, 3, np.zeros(1, dtype=int), x0, beta=0.01)
    assert rel_l2(to_np(x), ref) < 1e-4, rel_l2(to_np(x), ref)


def test_regularized_cg_edges(rtkb, oracle):
    gl, go, vd, vo, pd, po, p = _osem_problem(rtkb, oracle, 10)
    x0 = np.random.default_rng(2).normal(size=oracle.shape_of(vo))
    x = to_gpu(x0)
    rtkb.ops.regularized_cg(gl, vd, pd, to_gpu(p), x, main_loop_iterations=0)
    assert np.array_equal(to_np(x), x0.astype(np.float32))
    # no CG iterations: the restarts leave x, then positivity and TV act on it
    ref = oracle.regularized_cg(go, vo, po, p, x0.astype(np.float32).astype(np.float64), main_iterations=2,
                                cg_iterations=0, gamma_tv=0.1, tv_iterations=3)
    x = to_gpu(x0)
    rtkb.ops.regularized_cg(gl, vd, pd, to_gpu(p), x, main_loop_iterations=2, cg_iterations=0, gamma_tv=0.1,
                            tv_iterations=3)
    assert rel_l2(to_np(x), ref) < 1e-5, rel_l2(to_np(x), ref)


def test_raw_conversion_edges(rtkb, oracle):
    one = np.array([[[1234]]], dtype=np.uint16)
    d1 = rtkb.make_desc((1, 1, 1))
    assert np.array_equal(rtkb.ops.raw_to_attenuation(d1, _u16(one), 4000.0).cpu().numpy(),
                          oracle.raw_to_attenuation(one, 4000.0))
    const = np.full((2, 30, 40), 5000, dtype=np.uint16)
    dc = rtkb.make_desc((40, 30, 2))
    assert rtkb.ops.i0_estimation(dc, _u16(const)) == oracle.i0_estimation(const)
    # a buffer that starts 2 bytes past a 16-byte boundary takes the element-wise path
    raw = np.random.default_rng(4).integers(0, 65536, size=(1, 3, 101)).astype(np.uint16)
    big = _u16(np.concatenate([np.zeros(1, np.uint16), raw.ravel()]))
    sub = big[1:]
    out = torch.empty(raw.size + 1, device="cuda")[1:]
    dr = rtkb.make_desc((101, 3, 1))
    got = rtkb.ops.raw_to_attenuation(dr, sub.view(1, 3, 101), 30000.0, 10.0, out=out.view(1, 3, 101))
    assert np.array_equal(got.cpu().numpy(), oracle.raw_to_attenuation(raw, 30000.0, 10.0))


def test_empty_images_refused(rtkb):
    d0 = rtkb.make_desc((0, 4, 4))
    with pytest.raises((rtkb.RtkbError, ValueError, TypeError)):
        rtkb.ops.tv_denoising_bpdq(d0, torch.zeros((4, 4, 0), device="cuda"), 0.1, 2)
    with pytest.raises((rtkb.RtkbError, ValueError, TypeError)):
        rtkb.ops.raw_to_attenuation(d0, torch.zeros((4, 4, 0), device="cuda", dtype=torch.int16))

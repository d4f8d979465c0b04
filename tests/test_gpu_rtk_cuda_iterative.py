"""RTK's own CUDA projectors and iterative-reconstruction pieces, compiled
unchanged from the RTK sources by oracle/rtk_cuda/Makefile into
oracle/_ref/librtkcudaiter.so, on a B200 against the FP64 oracle and the
product on the same inputs.  These run the reference itself, so they pin the
oracle's conventions to RTK's GPU code:

  * the ray-casting forward projector (src/rtkCudaForwardProjectionImageFilter.cu,
    trilinear texture samples every voxel spacing) against the oracle's Joseph
    projector on a smooth volume -- two quadratures of the same line
    integrals, so they agree to about 1e-3, while a half-voxel slip of the
    volume or detector convention moves the projections by several percent
    (the test measures that margin on the oracle);
  * the voxel-based back projector (src/rtkCudaBackProjectionImageFilter.cu,
    bilinear texture reads) against the oracle's BackProjectionImageFilter,
    at the precision of the texture unit's 8-bit interpolation weights
    (about 2e-5 here, against 2.4e-3 for a half-pixel slip of the detector);
  * the Laplacian and TV denoising (BPDQ) kernels (exact FP32 finite
    differences) at 1e-6;
  * the conjugate-gradient update (src/rtkCudaConjugateGradientImageFilter.cu,
    cuBLAS FP32 dots), driven with the product's normal operator, against the
    oracle's CG: RTK's own recurrence reaches the oracle's iterate.

Skipped when the library was not built (no RTK source tree where it was
built)."""
import numpy as np
import pytest

from tests import phantoms
from tests.gpu_util import REL_L2_TOL, pair_geometry, pair_image, rel_l2, to_gpu, to_np

pytestmark = pytest.mark.gpu

# exact FP32 finite differences against FP64 (measured: 3e-8 to 5e-8)
FD_TOL = 1e-6
# CG iterates amplify rounding differences with every iteration (FP32 dots in
# RTK's update against FP64 in the oracle)
CG_TOL = 1e-4


def _need():
    from oracle import rtk_cuda

    if not rtk_cuda.iter_available():
        pytest.skip("RTK's CUDA projectors were not built (no RTK source tree)")
    return rtk_cuda


def _blobs(oracle, vol, seed, n=6):
    """Sum of Gaussian blobs (sigma 12-24 mm) inside the volume's central
    region: smooth, and negligible on the box faces."""
    rng = np.random.default_rng(seed)
    i2p = oracle.index_to_physical(vol)
    nz, ny, nx = oracle.shape_of(vol)
    zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    idx = np.stack([xx, yy, zz, np.ones_like(xx)], axis=-1).astype(np.float64)
    phys = idx @ i2p.T
    centre = (i2p @ np.array([(nx - 1) / 2, (ny - 1) / 2, (nz - 1) / 2, 1.0]))[:3]
    half = 0.25 * np.array([nx * vol.spacing[0], ny * vol.spacing[1], nz * vol.spacing[2]])
    out = np.zeros((nz, ny, nx))
    for _ in range(n):
        c = centre + rng.uniform(-1.0, 1.0, 3) * half
        s = rng.uniform(12.0, 24.0)
        d2 = ((phys[..., :3] - c) ** 2).sum(-1)
        out += rng.uniform(0.5, 1.5) * np.exp(-0.5 * d2 / (s * s))
    return out.astype(np.float32)


def _cone(n, gantry0=3.0):
    return [(600.0, 1200.0, gantry0 + i * 360.0 / n, 6.0, -4.0, 2.0, 3.0, 20.0, 15.0) for i in range(n)]


def test_rtk_cuda_forward_projector_agrees_with_oracle(rtkb, oracle):
    import torch

    rtk_cuda = _need()
    n = 60
    gl, go = pair_geometry(rtkb, oracle, _cone(n))
    vd, vo = pair_image(rtkb, oracle, (64, 64, 64), (4.0,) * 3, origin=(-126.0,) * 3)
    pd, po = pair_image(rtkb, oracle, (128, 128, n), (4.0, 4.0, 1.0), origin=(-254.0, -254.0, 0.0))
    x = _blobs(oracle, vo, seed=3)
    x64 = x.astype(np.float64)
    ref = oracle.joseph_forward(go, vo, x64, po)
    d_vol = torch.from_numpy(x).cuda()
    zeros = torch.zeros(oracle.shape_of(po), device="cuda")
    d_out = torch.empty_like(zeros)
    torch.cuda.synchronize()
    rtk_cuda.forward_project(oracle, go, vo, po, d_vol.data_ptr(), zeros.data_ptr(), d_out.data_ptr())
    torch.cuda.synchronize()
    e_rtk = rel_l2(to_np(d_out), ref)
    # the margin: the same projection with the volume half a voxel off
    vo_shift = oracle.image((64, 64, 64), (4.0,) * 3, origin=(-124.0, -126.0, -126.0))
    e_slip = rel_l2(oracle.joseph_forward(go, vo_shift, x64, po), ref)
    assert e_slip > 3e-2, e_slip
    assert e_rtk < 1e-2, (e_rtk, e_slip)
    got = to_np(rtkb.ops.joseph_forward_project(gl, vd, pd, d_vol, torch.zeros_like(zeros)))
    assert rel_l2(got, ref) < REL_L2_TOL


def test_rtk_cuda_voxel_backprojector_agrees_with_oracle(rtkb, oracle):
    import torch

    rtk_cuda = _need()
    n = 72
    gl, go = pair_geometry(rtkb, oracle, _cone(n, gantry0=1.0))
    vd, vo = pair_image(rtkb, oracle, (96, 96, 96), (2.5,) * 3, origin=(-118.75,) * 3)
    pd, po = pair_image(rtkb, oracle, (128, 128, n), (4.0, 4.0, 1.0), origin=(-254.0, -254.0, 0.0))
    sl = phantoms.shepp_logan(100.0)
    p = oracle.project_ellipsoids(go, po, sl).astype(np.float32)
    ref = oracle.backproject(go, vo, po, p.astype(np.float64), fdk=False)
    d_proj = torch.from_numpy(p).cuda()
    vin = torch.zeros(oracle.shape_of(vo), device="cuda")
    vout = torch.zeros_like(vin)
    torch.cuda.synchronize()
    rtk_cuda.back_project(oracle, go, vo, po, vin.data_ptr(), vout.data_ptr(), d_proj.data_ptr())
    torch.cuda.synchronize()
    got = to_np(rtkb.ops.voxel_backproject(gl, vd, pd, d_proj, torch.zeros_like(vin)))
    # voxels every projection sees: the texture's border mode and RTK's CPU
    # acceptance test disagree only where a voxel projects off the detector
    fov = phantoms.fov_mask(go, vo, po)
    assert fov.mean() > 0.3
    e_rtk = rel_l2(to_np(vout)[fov], ref[fov])
    # the margin: the detector half a pixel off
    po_slip = oracle.image((128, 128, n), (4.0, 4.0, 1.0), origin=(-252.0, -254.0, 0.0))
    e_slip = rel_l2(oracle.backproject(go, vo, po_slip, p.astype(np.float64), fdk=False)[fov], ref[fov])
    assert e_slip > 2e-3, e_slip
    assert e_rtk < 2e-4, (e_rtk, e_slip)
    assert rel_l2(got, ref) < REL_L2_TOL


def test_rtk_cuda_laplacian_agrees_with_oracle(rtkb, oracle):
    import torch

    rtk_cuda = _need()
    vd, vo = pair_image(rtkb, oracle, (40, 36, 32), (1.0, 1.5, 2.0))
    x = np.random.default_rng(5).uniform(-1.0, 1.0, size=oracle.shape_of(vo)).astype(np.float32)
    ref = oracle.laplacian(vo, x.astype(np.float64))
    d_in = torch.from_numpy(x).cuda()
    d_out = torch.empty_like(d_in)
    torch.cuda.synchronize()
    rtk_cuda.laplacian(vo, d_in.data_ptr(), d_out.data_ptr())
    torch.cuda.synchronize()
    assert rel_l2(to_np(d_out), ref) < FD_TOL
    assert rel_l2(to_np(rtkb.ops.laplacian(vd, d_in)), ref) < FD_TOL


@pytest.mark.parametrize("gamma,niter", [(0.05, 1), (0.2, 12)])
def test_rtk_cuda_tv_denoising_agrees_with_oracle(rtkb, oracle, gamma, niter):
    import torch

    rtk_cuda = _need()
    vd, vo = pair_image(rtkb, oracle, (48, 40, 32), (1.0, 1.25, 1.5))
    rng = np.random.default_rng(niter)
    f = (_blobs(oracle, vo, seed=niter, n=4) + 0.1 * rng.standard_normal(oracle.shape_of(vo))).astype(np.float32)
    ref = oracle.tv_denoising_bpdq(vo, f.astype(np.float64), gamma, niter)
    d_in = torch.from_numpy(f).cuda()
    d_out = torch.empty_like(d_in)
    torch.cuda.synchronize()
    rtk_cuda.total_variation_denoising(vo, d_in.data_ptr(), d_out.data_ptr(), gamma, niter)
    torch.cuda.synchronize()
    assert rel_l2(to_np(d_out), ref) < FD_TOL
    assert rel_l2(to_np(rtkb.ops.tv_denoising_bpdq(vd, d_in, gamma, niter)), ref) < FD_TOL


def test_rtk_cuda_conjugate_gradient_agrees_with_oracle(rtkb, oracle):
    """CudaConjugateGradientImageFilter's loop with RTK's CUDA update, the
    normal operator A = BP FP of the product's Joseph pair and b = BP p,
    against the oracle's CG (its own FP64 operator) and the product's CG."""
    import torch

    rtk_cuda = _need()
    n = 40
    params = [(600.0, 900.0, i * 360.0 / n, 0.0, 0.0) for i in range(n)]
    gl, go = pair_geometry(rtkb, oracle, params)
    vd, vo = pair_image(rtkb, oracle, (32, 28, 30), (8.0,) * 3)
    pd, po = pair_image(rtkb, oracle, (56, 48, n), (8.0, 8.0, 1.0))
    truth = np.random.default_rng(0).uniform(0.0, 1.0, size=oracle.shape_of(vo))
    p = oracle.joseph_forward(go, vo, truth, po).astype(np.float32).astype(np.float64)
    niter = 6
    ref_x, _ = oracle.cg_joseph(go, vo, po, p, niter)

    shape = oracle.shape_of(vo)
    d_p = to_gpu(p)
    b = rtkb.ops.joseph_back_project(gl, vd, pd, d_p, torch.zeros(shape, device="cuda"))
    plan = rtkb.ops.ConjugateGradient(gl, vd, pd, use_cuda_graph=False)
    vecs = {}

    def apply(src, dst):
        plan.apply_operator(vecs[src], vecs[dst])
        torch.cuda.synchronize()

    x, r, pk, ap = (torch.zeros(shape, device="cuda") for _ in range(4))
    for t in (b, x, r, pk, ap):
        vecs[t.data_ptr()] = t
    torch.cuda.synchronize()
    rtk_cuda.conjugate_gradient(x.numel(), apply, b.data_ptr(), x.data_ptr(), r.data_ptr(), pk.data_ptr(),
                                ap.data_ptr(), niter)
    torch.cuda.synchronize()
    x_rtk = to_np(x)
    assert rel_l2(x_rtk, ref_x) < CG_TOL, rel_l2(x_rtk, ref_x)

    x_prod = torch.zeros(shape, device="cuda")
    plan.start(d_p, x_prod, displaced_detector=False)
    plan.iterate(niter)
    assert rel_l2(to_np(x_prod), x_rtk) < CG_TOL
    plan.close()
    assert rtkb.ops.device_status() == 0


def test_rtk_cuda_ray_cast_back_projector_agrees_with_oracle(rtkb, oracle):
    """RTK's CUDA ray-cast back projector (src/rtkCudaRayCastBackProjectionImageFilter.cu,
    the back projector CUDA_ray_cast_back_project that rtkb_joseph_back_project
    replaces: steps of the smallest spacing along each ray, trilinear atomic
    splats) against the oracle's Joseph back projection of the same smooth
    projections: two discretisations of the same adjoint, so they agree to
    about 1e-2 inside the field of view, while a half-voxel slip of the volume
    convention moves the oracle's result several times more (the margin)."""
    import torch

    rtk_cuda = _need()
    n = 60
    gl, go = pair_geometry(rtkb, oracle, _cone(n))
    vd, vo = pair_image(rtkb, oracle, (64, 64, 64), (4.0,) * 3, origin=(-126.0,) * 3)
    pd, po = pair_image(rtkb, oracle, (128, 128, n), (4.0, 4.0, 1.0), origin=(-254.0, -254.0, 0.0))
    x = _blobs(oracle, vo, seed=7).astype(np.float64)
    p = oracle.joseph_forward(go, vo, x, po).astype(np.float32)
    ref = oracle.joseph_back(go, vo, po, p.astype(np.float64))
    d_p = torch.from_numpy(p).cuda()
    vin = torch.zeros(oracle.shape_of(vo), device="cuda")
    vout = torch.zeros_like(vin)
    torch.cuda.synchronize()
    rtk_cuda.ray_cast_back_project(oracle, go, vo, po, vin.data_ptr(), vout.data_ptr(), d_p.data_ptr())
    torch.cuda.synchronize()
    fov = phantoms.fov_mask(go, vo, po)
    e_rtk = rel_l2(to_np(vout)[fov], ref[fov])
    vo_shift = oracle.image((64, 64, 64), (4.0,) * 3, origin=(-124.0, -126.0, -126.0))
    e_slip = rel_l2(oracle.joseph_back(go, vo_shift, po, p.astype(np.float64))[fov], ref[fov])
    assert e_rtk < 2e-2 and e_slip > 2 * e_rtk, (e_rtk, e_slip)
    got = to_np(rtkb.ops.joseph_back_project(gl, vd, pd, d_p, torch.zeros_like(vin)))
    assert rel_l2(got, ref) < REL_L2_TOL

"""GPU conjugate gradient (rtkb_cg_*, rtkb_conjugate_gradient) against the
FP64 oracle restating include/rtkConjugateGradientImageFilter.hxx with the
Joseph operator of include/rtkReconstructionConjugateGradientOperator.hxx, and
RTK's CG reconstruction test (test/rtkconjugategradientreconstructiontest.cxx:
err/px < 0.08, PSNR > 23) on the GPU result."""
import numpy as np
import pytest

from tests import phantoms
from tests.gpu_util import pair_geometry, pair_image, rel_l2, to_gpu, to_np

pytestmark = pytest.mark.gpu

# CG iterates amplify rounding differences with every iteration; FP32 vectors
# against FP64 stay within this bound over the iteration counts tested here.
CG_TOL = 1e-4


def _problem(rtkb, oracle, n=40, vsize=(32, 28, 30), offset=0.0, seed=0):
    params = [(600.0, 900.0, i * 360.0 / n, offset, 0.0) for i in range(n)]
    gl, go = pair_geometry(rtkb, oracle, params)
    vd, vo = pair_image(rtkb, oracle, vsize, (8.0,) * 3)
    pd, po = pair_image(rtkb, oracle, (56, 48, n), (8.0, 8.0, 1.0))
    rng = np.random.default_rng(seed)
    truth = rng.uniform(0.0, 1.0, size=oracle.shape_of(vo))
    p = oracle.joseph_forward(go, vo, truth, po).astype(np.float32).astype(np.float64)
    return gl, go, vd, vo, pd, po, p


def test_cg_matches_oracle_iterates_and_residuals(rtkb, oracle):
    gl, go, vd, vo, pd, po, p = _problem(rtkb, oracle)
    niter = 6
    ref_x, ref_res = oracle.cg_joseph(go, vo, po, p, niter)
    import torch

    x = torch.zeros(oracle.shape_of(vo), device="cuda")
    cg = rtkb.ops.ConjugateGradient(gl, vd, pd)
    cg.start(to_gpu(p), x, displaced_detector=False)
    res = [cg.residual()[0]]
    for _ in range(niter):
        cg.iterate(1)
        res.append(cg.residual()[0])
    cg.close()
    assert rel_l2(to_np(x), ref_x) < CG_TOL
    np.testing.assert_allclose(res, ref_res, rtol=CG_TOL)
    assert rtkb.ops.device_status() == 0


def test_cg_graph_equals_eager(rtkb, oracle):
    gl, go, vd, vo, pd, po, p = _problem(rtkb, oracle, seed=1)
    import torch

    outs = []
    for graph in (True, False):
        x = torch.zeros(oracle.shape_of(vo), device="cuda")
        cg = rtkb.ops.ConjugateGradient(gl, vd, pd, use_cuda_graph=graph)
        cg.start(to_gpu(p), x, displaced_detector=False)
        cg.iterate(4)
        outs.append((to_np(x), cg.residual()[0]))
        cg.close()
    # the Joseph back projector accumulates with atomics, so runs agree to FP32
    # rounding rather than bitwise
    assert rel_l2(outs[0][0], outs[1][0]) < 1e-5
    assert abs(outs[0][1] / outs[1][1] - 1) < 1e-5


def test_cg_tikhonov_weights_and_warm_start(rtkb, oracle):
    gl, go, vd, vo, pd, po, p = _problem(rtkb, oracle, seed=2)
    rng = np.random.default_rng(3)
    w = rng.uniform(0.5, 2.0, size=p.shape).astype(np.float32).astype(np.float64)
    x0 = rng.uniform(0.0, 0.5, size=oracle.shape_of(vo)).astype(np.float32).astype(np.float64)
    ref_x, _ = oracle.cg_joseph(go, vo, po, p, 4, x0=x0, weights=w, tikhonov=0.3)
    x = to_gpu(x0)
    cg = rtkb.ops.ConjugateGradient(gl, vd, pd, tikhonov=0.3)
    cg.start(to_gpu(p), x, weights=to_gpu(w), displaced_detector=False)
    cg.iterate(4)
    assert rel_l2(to_np(x), ref_x) < CG_TOL
    cg.close()


def test_cg_displaced_detector_weights(rtkb, oracle):
    """W = displaced-detector weights of ones (RTK's default for CG)."""
    gl, go, vd, vo, pd, po, p = _problem(rtkb, oracle, offset=60.0, seed=4)
    ones = np.ones(p.shape)
    wref, _, _ = oracle.displaced_detector(go, po, ones, pad=False)
    ref_x, _ = oracle.cg_joseph(go, vo, po, p, 3, weights=wref)
    import torch

    x = torch.zeros(oracle.shape_of(vo), device="cuda")
    it, rel = rtkb.ops.conjugate_gradient(gl, vd, pd, to_gpu(p), x, 3, displaced_detector=True)
    assert it == 3 and 0 < rel < 1
    assert rel_l2(to_np(x), ref_x) < CG_TOL


def test_cg_early_stop_on_relative_residual(rtkb, oracle):
    gl, go, vd, vo, pd, po, p = _problem(rtkb, oracle, seed=5)
    import torch

    x = torch.zeros(oracle.shape_of(vo), device="cuda")
    it, rel = rtkb.ops.conjugate_gradient(gl, vd, pd, to_gpu(p), x, 200, rel_residual=1e-2,
                                          displaced_detector=False)
    assert rel <= 1e-2 and it < 200


@pytest.mark.parametrize("tikhonov,offset", [(0.0, 0.0), (0.3, 40.0)])
def test_cg_voxel_backprojector_matches_oracle(rtkb, oracle, tikhonov, offset):
    """RTK's default projector choice (Joseph forward, voxel-based back
    projector, include/rtkIterativeConeBeamReconstructionFilter.hxx:33-103):
    b = BP_voxel(W p), A = BP_voxel W FP_Joseph (+ tikhonov), iterates and
    residuals against the oracle's CG with the same back projector."""
    import torch

    gl, go, vd, vo, pd, po, p = _problem(rtkb, oracle, offset=offset, seed=4)
    niter = 6
    w = oracle.displaced_detector(go, po, np.ones(oracle.shape_of(po)), pad=False)[0] if offset else None
    ref_x, ref_res = oracle.cg_joseph(go, vo, po, p, niter, weights=w, tikhonov=tikhonov, backprojector="voxel")
    x = torch.zeros(oracle.shape_of(vo), device="cuda")
    cg = rtkb.ops.ConjugateGradient(gl, vd, pd, tikhonov=tikhonov, backprojector="voxel")
    cg.start(to_gpu(p), x, displaced_detector=bool(offset))
    res = [cg.residual()[0]]
    for _ in range(niter):
        cg.iterate(1)
        res.append(cg.residual()[0])
    cg.close()
    assert rel_l2(to_np(x), ref_x) < CG_TOL
    np.testing.assert_allclose(res, ref_res, rtol=CG_TOL)
    assert rtkb.ops.device_status() == 0


@pytest.mark.parametrize("backprojector", ["voxel", "joseph"])
def test_cg_sphere_like_rtkconjugategradientreconstructiontest(rtkb, oracle, backprojector):
    """Sphere of radius 90 mm, 64^3 at 4 mm, 180 projections, 5 iterations
    (RTK's test: case 1 with the voxel-based back projector, uniform input
    weights; the Joseph back projector as in its case 2 without the
    regularisation weights)."""
    n = 180
    params = [(600.0, 1200.0, i * 360.0 / n) for i in range(n)]
    gl, go = pair_geometry(rtkb, oracle, params)
    vd, vo = pair_image(rtkb, oracle, (64, 64, 64), (4.0,) * 3, origin=(-126.0,) * 3)
    pd, po = pair_image(rtkb, oracle, (64, 64, n), (8.0, 8.0, 1.0), origin=(-254.0, -254.0, 0.0))
    sphere = phantoms.ellipsoid((0.0, 0.0, 0.0), (90.0, 90.0, 90.0), np.eye(3), 1.0)[None]
    p = oracle.project_ellipsoids(go, po, sphere)
    ref = oracle.draw_ellipsoids(vo, sphere)
    import torch

    x = torch.zeros((64, 64, 64), device="cuda")
    rtkb.ops.conjugate_gradient(gl, vd, pd, to_gpu(p), x, 5, displaced_detector=True, backprojector=backprojector)
    err, psnr, ok = phantoms.check_image_quality(to_np(x), ref, 0.08, 23.0, 2.0)
    assert ok, (err, psnr)
    ref_x, _ = oracle.cg_joseph(go, vo, po, p, 5, backprojector=backprojector)
    assert rel_l2(to_np(x), ref_x) < CG_TOL


# BF16 storage of r, p, A p and the projection temporary rounds each stored
# value to 8 significant bits (relative 2^-9).  CG in reduced precision loses
# the conjugacy of its directions, so its iterates drift from the exact ones
# faster than the rounding itself (4.6e-2 after 6 iterations on this problem,
# while the residual still falls as fast as in FP32).
BF16_CG_TOL = 0.1


def test_cg_bf16_storage_precision_against_oracle(rtkb, oracle):
    """Precision study of the storage variants: FP32 and BF16 plans against
    the FP64 oracle's CG on the same problem, graph and eager BF16 alike."""
    import torch

    gl, go, vd, vo, pd, po, p = _problem(rtkb, oracle, seed=3)
    niter = 6
    ref_x, ref_res = oracle.cg_joseph(go, vo, po, p, niter)
    errs = {}
    for storage, graph in (("fp32", True), ("bf16", True), ("bf16", False), ("bf16_direction", True)):
        x = torch.zeros(oracle.shape_of(vo), device="cuda")
        cg = rtkb.ops.ConjugateGradient(gl, vd, pd, storage=storage, use_cuda_graph=graph)
        cg.start(to_gpu(p), x, displaced_detector=False)
        res = [cg.residual()[0]]
        for _ in range(niter):
            cg.iterate(1)
            res.append(cg.residual()[0])
        cg.close()
        assert rtkb.ops.device_status() == 0
        assert res[-1] < 0.1 * res[0], res
        errs[(storage, graph)] = rel_l2(to_np(x), ref_x)
        errs[(storage, graph, "residual")] = res[-1] / res[0]
    assert errs[("fp32", True)] < CG_TOL, errs
    # the BF16 plan's residual falls within a factor 2 of the FP32 plan's
    assert errs[("bf16", True, "residual")] < 2 * errs[("fp32", True, "residual")], errs
    # BF16 storage really rounds (error well above FP32's) and stays bounded
    for graph in (True, False):
        assert 10 * errs[("fp32", True)] < errs[("bf16", graph)] < BF16_CG_TOL, errs
    # a BF16 direction with an FP32 residual recurrence: converges as FP32 does
    # and stays closer to the exact iterates than all-BF16 storage
    assert errs[("bf16_direction", True, "residual")] < 2 * errs[("fp32", True, "residual")], errs
    assert errs[("bf16_direction", True)] < errs[("bf16", True)], errs


def test_cg_bf16_operator_and_preconditioner_refusal(rtkb, oracle):
    """The BF16 plan's operator rounds only its projection temporary; the
    learned preconditioner is refused (FP32 plans only)."""
    import torch

    from rtk_b200.learned import UNet

    gl, go, vd, vo, pd, po, p = _problem(rtkb, oracle, seed=4)
    rng = np.random.default_rng(4)
    e = to_gpu(rng.uniform(-1.0, 1.0, size=oracle.shape_of(vo)))
    outs = []
    for storage in ("fp32", "bf16"):
        cg = rtkb.ops.ConjugateGradient(gl, vd, pd, storage=storage)
        out = torch.empty_like(e)
        cg.apply_operator(e, out)
        outs.append(to_np(out))
        if storage == "bf16":
            with pytest.raises(Exception):
                cg.set_preconditioner(UNet(seed=0))
        cg.close()
    d = rel_l2(outs[1], outs[0])
    assert 1e-5 < d < 1e-2, d
    assert rtkb.ops.device_status() == 0


def test_cg_batch_matches_single_plans_and_oracle(rtkb, oracle):
    """Batched CG (rtkb_cg_batch_*): six uneven problems iterated as one graph
    launch (replayed twice) agree with separate plans and, for one problem,
    with the FP64 oracle's CG."""
    import torch

    rng = np.random.default_rng(7)
    probs, cases = [], []
    for i in range(6):
        n = int(rng.integers(16, 33))
        nv = int(rng.integers(18, 33))
        vsize = (nv, nv - 2, nv + 1)
        psize = (int(rng.integers(10, 17)) * 4, int(rng.integers(30, 49)), n)
        sid = float(rng.uniform(500.0, 700.0))
        gl, go = pair_geometry(rtkb, oracle, [(sid, 1.5 * sid, k * 360.0 / n, 0.0, 0.0) for k in range(n)])
        vd, vo = pair_image(rtkb, oracle, vsize, (8.0,) * 3)
        pd, po = pair_image(rtkb, oracle, psize, (8.0, 8.0, 1.0))
        truth = rng.uniform(0.0, 1.0, size=oracle.shape_of(vo))
        p = oracle.joseph_forward(go, vo, truth, po).astype(np.float32).astype(np.float64)
        x = torch.zeros(oracle.shape_of(vo), device="cuda")
        probs.append((gl, vd, pd, to_gpu(p), x, None, False))
        cases.append((gl, go, vd, vo, pd, po, p))
    batch = rtkb.ops.ConjugateGradientBatch(probs)
    batch.start()
    batch.iterate(3)
    batch.iterate(3)  # replay of the same graph
    res = [batch.residual(i) for i in range(len(probs))]
    assert rtkb.ops.device_status() == 0
    for i, (gl, go, vd, vo, pd, po, p) in enumerate(cases):
        assert res[i][2] == 6
        x1 = torch.zeros(oracle.shape_of(vo), device="cuda")
        cg = rtkb.ops.ConjugateGradient(gl, vd, pd)
        cg.start(to_gpu(p), x1, displaced_detector=False)
        cg.iterate(6)
        rr1 = cg.residual()[0]
        cg.close()
        # same kernels; only the order of the back projector's FP32 reductions differs
        assert rel_l2(to_np(probs[i][4]), to_np(x1)) < 1e-5
        np.testing.assert_allclose(res[i][0], rr1, rtol=1e-4)
    gl, go, vd, vo, pd, po, p = cases[0]
    ref_x, _ = oracle.cg_joseph(go, vo, po, p, 6)
    assert rel_l2(to_np(probs[0][4]), ref_x) < CG_TOL
    batch.close()


def test_laplacian_matches_oracle(rtkb, oracle):
    """rtkb_laplacian against RTK's LaplacianImageFilter restated (Neumann
    boundary, anisotropic spacing, a one-voxel axis)."""
    rng = np.random.default_rng(9)
    for size, sp in (((17, 12, 9), (1.0, 2.5, 0.7)), ((8, 1, 5), (2.0, 1.0, 3.0))):
        vd, vo = pair_image(rtkb, oracle, size, sp)
        x = rng.uniform(-1.0, 1.0, size=oracle.shape_of(vo)).astype(np.float32).astype(np.float64)
        got = to_np(rtkb.ops.laplacian(vd, to_gpu(x)))
        ref = oracle.laplacian(vo, x)
        assert rel_l2(got, ref) < 1e-6, rel_l2(got, ref)


def test_cg_laplacian_regularisation_matches_oracle(rtkb, oracle):
    """CG with RTK's gamma (Laplacian) and Tikhonov terms, graph and eager,
    against the FP64 oracle's CG with the same operator."""
    import torch

    gl, go, vd, vo, pd, po, p = _problem(rtkb, oracle, seed=6)
    # gamma large enough to matter: the regulariser half the size of A^T A on a random volume
    xr = to_gpu(np.random.default_rng(6).uniform(-1.0, 1.0, size=oracle.shape_of(vo)))
    plan = rtkb.ops.ConjugateGradient(gl, vd, pd)
    ax = plan.apply_operator(xr, torch.empty_like(xr))
    plan.close()
    gamma = 0.5 * float(ax.norm() / rtkb.ops.laplacian(vd, xr).norm())
    ref_x, ref_res = oracle.cg_joseph(go, vo, po, p, 5, tikhonov=0.3, gamma=gamma)
    for graph in (True, False):
        x = torch.zeros(oracle.shape_of(vo), device="cuda")
        cg = rtkb.ops.ConjugateGradient(gl, vd, pd, tikhonov=0.3, gamma=gamma, use_cuda_graph=graph)
        cg.start(to_gpu(p), x, displaced_detector=False)
        res = [cg.residual()[0]]
        for _ in range(5):
            cg.iterate(1)
            res.append(cg.residual()[0])
        cg.close()
        assert rel_l2(to_np(x), ref_x) < CG_TOL
        np.testing.assert_allclose(res, ref_res, rtol=CG_TOL)
    # the regulariser changes the solution
    plain, _ = oracle.cg_joseph(go, vo, po, p, 5, tikhonov=0.3)
    assert rel_l2(plain, ref_x) > 1e-3
    assert rtkb.ops.device_status() == 0


@pytest.mark.parametrize("kind", ["binary", "fractional"])
def test_cg_support_mask_matches_oracle(rtkb, oracle, kind):
    """SetSupportMask: b, the operator's input and output, and the result multiplied by the mask."""
    import torch

    n = 20
    gl, go = pair_geometry(rtkb, oracle, [(600.0, 900.0, i * 360.0 / n, 15.0, 0.0) for i in range(n)])
    vd, vo = pair_image(rtkb, oracle, (24, 20, 22), (6.0,) * 3)
    pd, po = pair_image(rtkb, oracle, (48, 40, n), (4.0, 4.0, 1.0))
    rng = np.random.default_rng(11)
    truth = rng.uniform(0.0, 1.0, size=oracle.shape_of(vo))
    p = oracle.joseph_forward(go, vo, truth, po).astype(np.float32).astype(np.float64)
    mask = np.zeros(oracle.shape_of(vo))
    mask[3:19, 2:18, 4:20] = 1.0
    if kind == "fractional":
        mask *= rng.uniform(0.5, 1.0, size=mask.shape)
    mask = mask.astype(np.float32).astype(np.float64)
    ref, _ = oracle.cg_joseph(go, vo, po, p, 4, tikhonov=5.0, gamma=2.0, mask=mask)
    x = torch.zeros(oracle.shape_of(vo), device="cuda")
    cg = rtkb.ops.ConjugateGradient(gl, vd, pd, tikhonov=5.0, gamma=2.0)
    cg.set_support_mask(to_gpu(mask))
    cg.start(to_gpu(p), x, displaced_detector=False)
    cg.iterate(4)
    cg.finish()
    assert rel_l2(to_np(x), ref) < 1e-4, rel_l2(to_np(x), ref)
    assert np.all(to_np(x)[mask == 0] == 0.0)


@pytest.mark.parametrize("storage,where", [("fp32", "cuda"), ("bf16_direction", "cpu")])
def test_cg_checkpoint_resume(rtkb, oracle, storage, where):
    """rtkb_cg_save_state after 3 iterations, a new plan started on the saved
    iterate and loaded from the checkpoint, 3 more iterations: the iterate and
    residuals of 6 uninterrupted iterations (the back projector's atomics
    reorder FP32 sums, hence a tolerance), unlike a warm start from the saved
    iterate, which restarts the recurrence; foreign checkpoints are refused."""
    import torch

    gl, go, vd, vo, pd, po, p = _problem(rtkb, oracle, seed=4)
    dp = to_gpu(p)

    def plan():
        return rtkb.ops.ConjugateGradient(gl, vd, pd, storage=storage)

    x = torch.zeros(oracle.shape_of(vo), device="cuda")
    a = plan().start(dp, x, displaced_detector=False)
    a.iterate(3)
    x3 = x.clone()
    state = a.save_state(device=where)
    rr3 = a.residual()
    a.iterate(3)
    rr6 = a.residual()
    x6 = to_np(x)

    xb = x3.clone()
    b = plan().start(dp, xb, displaced_detector=False)
    b.load_state(state)
    assert b.residual() == rr3
    b.iterate(3)
    rb = b.residual()
    assert rb[2] == 6 and abs(rb[0] - rr6[0]) <= 1e-4 * rr6[0]
    assert rel_l2(to_np(xb), x6) < 1e-5

    xc = x3.clone()
    c = plan().start(dp, xc, displaced_detector=False)  # warm start: a new recurrence
    c.iterate(3)
    assert rel_l2(to_np(xc), x6) > 10 * rel_l2(to_np(xb), x6)

    other = rtkb.ops.ConjugateGradient(gl, vd, pd, storage="bf16" if storage == "fp32" else "fp32")
    other.start(dp, torch.zeros_like(x), displaced_detector=False)
    with pytest.raises(rtkb.RtkbError):
        other.load_state(state)
    for q in (a, b, c, other):
        q.close()
    assert rtkb.ops.device_status() == 0

"""Flexible PCG with the learned preconditioner (rtkb_cg_set_preconditioner):
convergence of a solve with a trained network and agreement of its solution
with plain CG's and the FP64 oracle's CG solution, the fallback to plain CG
when the residual stops decreasing, graph replay, the start from a given
right-hand side and the normal operator that generates the training pairs."""
import numpy as np
import pytest

from tests.gpu_util import pair_geometry, pair_image, rel_l2, to_gpu, to_np

pytestmark = pytest.mark.gpu

TOL = 1e-3  # normal-equation relative residual the solvers run to


def _problem(rtkb, oracle, n=60, vsize=(32, 32, 32), seed=0):
    from tests import phantoms

    params = [(600.0, 900.0, i * 360.0 / n) for i in range(n)]
    gl, go = pair_geometry(rtkb, oracle, params)
    vd, vo = pair_image(rtkb, oracle, vsize, (6.0,) * 3)
    pd, po = pair_image(rtkb, oracle, (64, 56, n), (6.0, 6.0, 1.0))
    ell = phantoms.random_ellipsoids(8, seed, axis_range=(10.0, 60.0), centre_radius=40.0)
    p = oracle.project_ellipsoids(go, po, ell)
    rng = np.random.default_rng(seed)
    p = (p + rng.normal(0.0, 0.01 * p.max(), size=p.shape)).astype(np.float32).astype(np.float64)
    return gl, go, vd, vo, pd, po, p


def _solve(rtkb, gl, vd, pd, p, shape, net=None, max_iter=200, graph=True):
    import torch

    x = torch.zeros(shape, device="cuda")
    cg = rtkb.ops.ConjugateGradient(gl, vd, pd, use_cuda_graph=graph)
    if net is not None:
        cg.set_preconditioner(net)
    cg.start(to_gpu(p), x, displaced_detector=False)
    _, rr0, _ = cg.residual()
    hist = [1.0]
    it = 0
    while it < max_iter:
        cg.iterate(1)
        it += 1
        rr, _, _ = cg.residual()
        hist.append(float(np.sqrt(rr / rr0)))
        if hist[-1] <= TOL:
            break
    status = cg.preconditioner_status()
    cg.close()
    return to_np(x), it, hist, status


def _trained_net(rtkb, plan, steps=600):
    from rtk_b200 import learned

    rs, es, _ = learned.make_training_pairs(plan, 24, seed=1)
    net = learned.UNet(seed=1)
    learned.train(net, rs, es, steps=steps, batch=4, crop=32, lr=2e-3, lr_final=2e-4)
    return net


def test_learned_pcg_converges_and_agrees(rtkb, oracle):
    """A network trained by the project's own kernels on pairs from the plan's
    operator, used in flexible PCG: the solve reaches the 1e-3 tolerance (the
    fallback to plain CG guarantees it) and its solution matches plain CG's
    (which matches the FP64 oracle's).  The iteration count is not bounded
    here: after a late fallback, plain CG restarted from the current iterate
    can need more iterations than from zero.  The single-step
    quality of the network against the steepest-descent step of plain CG
    (||A (g z) - r|| / ||r|| on held-out pairs) is measured and reported; on
    this 32^3 problem and on the 256^3 one the benchmark trains on it is
    better than plain CG's step for early residuals only."""
    from rtk_b200 import learned

    gl, go, vd, vo, pd, po, p = _problem(rtkb, oracle)
    shape = oracle.shape_of(vo)
    plan = rtkb.ops.ConjugateGradient(gl, vd, pd)
    net = _trained_net(rtkb, plan)
    hr, _, _ = learned.make_krylov_pairs(plan, 1, iterations=5, every=5, seed=99)
    q = learned.preconditioner_quality(plan, net, hr, None)
    plan.close()
    assert all(np.isfinite(a) and np.isfinite(b) for a, b in q)
    x_cg, it_cg, h_cg, _ = _solve(rtkb, gl, vd, pd, p, shape)
    x_pcg, it_pcg, h_pcg, (active, fb) = _solve(rtkb, gl, vd, pd, p, shape, net=net)
    info = {"quality (net, identity)": q, "cg": it_cg, "pcg": it_pcg, "fallback": fb}
    assert h_cg[-1] <= TOL and h_pcg[-1] <= TOL, info
    # plain CG follows the oracle's FP64 iteration closely; the preconditioned
    # solve stops on a different path inside the same tolerance ball
    # (relative residual 1e-3), so it is compared with a bound of that size
    ref_x, _ = oracle.cg_joseph(go, vo, po, p, it_cg)
    e_cg, d_pcg = rel_l2(x_cg, ref_x), rel_l2(x_pcg, x_cg)
    assert e_cg < 2e-2 and d_pcg < 0.1, (e_cg, d_pcg, info)
    net.close()


def test_pcg_falls_back_to_cg_when_residual_stalls(rtkb, oracle):
    """A network with all-zero weights gives z = 0: the residual cannot
    decrease, so after two stalled iterations plain CG takes over and still
    reaches the tolerance."""
    from rtk_b200.learned import UNet

    gl, go, vd, vo, pd, po, p = _problem(rtkb, oracle, seed=2)
    shape = oracle.shape_of(vo)
    _, it_cg, _, _ = _solve(rtkb, gl, vd, pd, p, shape)
    net = UNet(seed=0)
    net.set_parameters(np.zeros(net.n, np.float32))
    x, it, hist, (active, fb) = _solve(rtkb, gl, vd, pd, p, shape, net=net)
    assert not active and fb == 2
    assert hist[1] == pytest.approx(1.0) and hist[2] == pytest.approx(1.0)
    assert hist[-1] <= TOL and it <= it_cg + 3
    net.close()


def test_pcg_graph_equals_eager(rtkb, oracle):
    """Graph replay and eager launches run the same iteration.  They agree to
    the preconditioner's BF16 noise, not to FP32 rounding: the back projector's
    atomic summation order perturbs r by ~1e-7, and BF16 rounding flips inside
    the network turn that into ~0.3 % differences of z = M(r) (eager against
    eager differs as much).  Residuals, which average that noise out, agree to
    5e-3."""
    from rtk_b200.learned import UNet

    gl, go, vd, vo, pd, po, p = _problem(rtkb, oracle, seed=3)
    shape = oracle.shape_of(vo)
    net = UNet(seed=4)
    outs = []
    for graph in (True, False):
        x, it, hist, _ = _solve(rtkb, gl, vd, pd, p, shape, net=net, max_iter=3, graph=graph)
        outs.append((x, hist))
    assert rel_l2(outs[0][0], outs[1][0]) < 0.1
    np.testing.assert_allclose(outs[0][1], outs[1][1], rtol=5e-3)
    net.close()


def test_cg_start_rhs_matches_start(rtkb, oracle):
    """rtkb_cg_start_rhs with b = BP(p) runs the same iterations as
    rtkb_cg_start with the projections p (W = 1)."""
    import torch

    gl, go, vd, vo, pd, po, p = _problem(rtkb, oracle, seed=5)
    shape = oracle.shape_of(vo)
    b = to_gpu(oracle.joseph_back(go, vo, po, p))
    xs = []
    for use_rhs in (False, True):
        x = torch.zeros(shape, device="cuda")
        cg = rtkb.ops.ConjugateGradient(gl, vd, pd)
        if use_rhs:
            cg.start_rhs(b, x)
        else:
            cg.start(to_gpu(p), x, displaced_detector=False)
        cg.iterate(5)
        xs.append(to_np(x))
        cg.close()
    assert rel_l2(xs[1], xs[0]) < 1e-4


def test_apply_operator_matches_oracle(rtkb, oracle):
    """rtkb_cg_apply_operator = BP(FP(x)) with W = 1 (the operator that
    generates the training pairs)."""
    import torch

    gl, go, vd, vo, pd, po, p = _problem(rtkb, oracle, seed=4)
    rng = np.random.default_rng(4)
    e = rng.uniform(0.0, 1.0, size=oracle.shape_of(vo))
    ref = oracle.joseph_back(go, vo, po, oracle.joseph_forward(go, vo, e, po))
    cg = rtkb.ops.ConjugateGradient(gl, vd, pd)
    out = torch.empty(oracle.shape_of(vo), device="cuda")
    cg.apply_operator(to_gpu(e), out)
    assert rel_l2(to_np(out), ref) < 1e-5
    cg.close()

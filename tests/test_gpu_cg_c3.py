"""The conjugate-gradient reconstruction at the CG configuration's full size
(256^3 at 1 mm from 360 projections of 512 x 384 at 0.8 mm, 20 random
ellipsoids, Poisson noise at I0 = 5e4) against the FP64 oracle's CG, three
iterations from zero with the Joseph pair on the FP32 plan.

The oracle needs minutes at this size, so its result is a committed fixture
(tests/golden/cg_c3_oracle.npz, written by tests/golden/make_cg_c3_fixture.py):
every 8th voxel along each axis of the iterate, its full norm and the
residual history.  The inputs are regenerated here from the same seeds and
checked against the fixture's sums first."""
import os

import numpy as np
import pytest

from tests import workloads as W
from tests.gpu_util import REL_L2_TOL, rel_l2, to_gpu

pytestmark = pytest.mark.gpu
FIXTURE = os.path.join(os.path.dirname(__file__), "golden", "cg_c3_oracle.npz")


def test_cg_c3_against_oracle_fixture(rtkb, oracle):
    import torch

    fx = np.load(FIXTURE)
    niter, stride = int(fx["iterations"]), int(fx["stride"])
    go, vo, po, p = W.c3_oracle_problem(oracle)
    assert abs(p.sum() - fx["input_sum"]) <= 1e-9 * abs(fx["input_sum"])
    assert abs((p * p).sum() - fx["input_sum_sq"]) <= 1e-9 * fx["input_sum_sq"]
    c = W.C3
    g = rtkb.geometry.circular(c["n"], c["sid"], c["sdd"])
    vd = rtkb.make_desc(c["vol"], (c["vox"],) * 3)
    pd = rtkb.make_desc((*c["det"], c["n"]), (c["pix"], c["pix"], 1.0))
    x = torch.zeros(tuple(reversed(c["vol"])), device="cuda")
    cg = rtkb.ops.ConjugateGradient(g, vd, pd)
    hist = []
    cg.start(to_gpu(p), x)
    for _ in range(niter):
        rr, rr0, _ = cg.residual()
        hist.append(rr)
        cg.iterate(1)
    rr, rr0, it = cg.residual()
    hist.append(rr)
    cg.close()
    assert it == niter and rtkb.ops.device_status() == 0
    got = x[::stride, ::stride, ::stride].cpu().numpy().astype(np.float64)
    assert rel_l2(got, fx["x_sample"].astype(np.float64)) < REL_L2_TOL
    full = float(torch.linalg.vector_norm(x.double()))
    assert abs(full - float(fx["x_norm"])) <= REL_L2_TOL * float(fx["x_norm"])
    np.testing.assert_allclose(np.array(hist), fx["residuals"], rtol=1e-4)

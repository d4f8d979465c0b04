"""Cylindrical detectors (SetRadiusCylindricalDetector) in the Joseph projector
pair and the CG plan, against the FP64 oracle restating
include/rtkProjectionsRegionConstIteratorRayBasedWithCylindricalPanel.hxx;
adjointness; RTK's cylindrical forward-projection test
(test/rtkforwardprojectiontest.cxx case 4) on the GPU; the voxel-based back
projector's path for a cylinder centred on the source; and the entry points
that model flat panels only refusing the geometry."""
import numpy as np
import pytest
import torch

from tests import phantoms
from tests.gpu_util import REL_L2_TOL, pair_geometry, pair_image, rel_l2, to_gpu, to_np

pytestmark = pytest.mark.gpu

GEOMS = {
    "centred_on_source": (lambda n: [(800.0, 1200.0, i * 360.0 / n) for i in range(n)], 1200.0),
    "radius_600": (lambda n: [(800.0, 1200.0, i * 360.0 / n) for i in range(n)], 600.0),
    "offsets_tilts": (lambda n: [(700.0, 1100.0, i * 360.0 / n + 3.0, 12.0, -7.0, 8.0, 4.0, 5.0, -3.0)
                                 for i in range(n)], 900.0),
}


def _case(rtkb, oracle, geom, n, vsize, psize, pspacing, seed=0):
    params, radius = GEOMS[geom]
    gl, go = pair_geometry(rtkb, oracle, params(n))
    gl.SetRadiusCylindricalDetector(radius)
    go.set_radius_cylindrical(radius)
    vd, vo = pair_image(rtkb, oracle, vsize, (4.0, 4.5, 3.5), index=(2, -3, 1))
    pd, po = pair_image(rtkb, oracle, psize, pspacing, index=(-4, 3, 0))
    rng = np.random.default_rng(seed)
    vol = rng.uniform(0.0, 1.0, size=oracle.shape_of(vo)).astype(np.float32).astype(np.float64)
    pr = rng.uniform(0.0, 1.0, size=oracle.shape_of(po)).astype(np.float32).astype(np.float64)
    return gl, go, vd, vo, pd, po, vol, pr


@pytest.mark.parametrize("geom", sorted(GEOMS))
@pytest.mark.parametrize("n", [3, 30])  # short stacks skip the quad copies
def test_cylindrical_forward_matches_oracle(rtkb, oracle, geom, n):
    gl, go, vd, vo, pd, po, vol, pr = _case(rtkb, oracle, geom, n, (40, 36, 44), (72, 64, n), (5.0, 5.0, 1.0))
    ref = oracle.joseph_forward(go, vo, vol, po, pr)
    got = to_np(rtkb.ops.joseph_forward_project(gl, vd, pd, to_gpu(vol), to_gpu(pr)))
    assert rel_l2(got, ref) < REL_L2_TOL, rel_l2(got, ref)


@pytest.mark.parametrize("geom", sorted(GEOMS))
def test_cylindrical_back_matches_oracle(rtkb, oracle, geom):
    gl, go, vd, vo, pd, po, vol, pr = _case(rtkb, oracle, geom, 24, (36, 32, 40), (64, 56, 24), (5.0, 5.0, 1.0))
    ref = oracle.joseph_back(go, vo, po, pr, vol)
    got = to_np(rtkb.ops.joseph_back_project(gl, vd, pd, to_gpu(pr), to_gpu(vol)))
    assert rel_l2(got, ref) < REL_L2_TOL, rel_l2(got, ref)


def test_cylindrical_adjoint(rtkb, oracle):
    gl, go, vd, vo, pd, po, vol, pr = _case(rtkb, oracle, "radius_600", 40, (48, 40, 44), (80, 70, 40),
                                            (6.0, 6.0, 1.0), seed=5)
    fp = to_np(rtkb.ops.joseph_forward_project(gl, vd, pd, to_gpu(vol), torch.zeros(pr.shape, device="cuda")))
    bp = to_np(rtkb.ops.joseph_back_project(gl, vd, pd, to_gpu(pr), torch.zeros(vol.shape, device="cuda")))
    a, b = np.vdot(fp, pr), np.vdot(vol, bp)
    assert abs(a / b - 1) < 1e-5, (a, b)


def test_cylindrical_cg_matches_oracle(rtkb, oracle):
    gl, go, vd, vo, pd, po, vol, pr = _case(rtkb, oracle, "centred_on_source", 20, (24, 20, 22), (48, 40, 20),
                                            (6.0, 6.0, 1.0), seed=2)
    p = oracle.joseph_forward(go, vo, vol, po).astype(np.float32).astype(np.float64)
    ref, _ = oracle.cg_joseph(go, vo, po, p, 4)
    x = torch.zeros(oracle.shape_of(vo), device="cuda")
    cg = rtkb.ops.ConjugateGradient(gl, vd, pd)
    cg.start(to_gpu(p), x, displaced_detector=False)
    cg.iterate(4)
    assert rel_l2(to_np(x), ref) < 1e-4, rel_l2(to_np(x), ref)


def test_rtk_cylindrical_forward_projection_test_on_gpu(rtkb, oracle):
    """test/rtkforwardprojectiontest.cxx case 4: Joseph projection of a 128^3 Shepp-Logan at 2 mm, 45 projections
    (SID 500, SDD 1000, 8 deg steps), cylindrical detector of radius 600, against the analytic projections."""
    n = 45
    gl, go = pair_geometry(rtkb, oracle, [(500.0, 1000.0, i * 8.0) for i in range(n)])
    gl.SetRadiusCylindricalDetector(600.0)
    go.set_radius_cylindrical(600.0)
    vd, vo = pair_image(rtkb, oracle, (128, 128, 128), (2.0,) * 3, origin=(-127.0,) * 3)
    pd, po = pair_image(rtkb, oracle, (64, 64, n), (4.0,) * 3, origin=(-126.0,) * 3)
    sl = phantoms.shepp_logan(128.0)
    ref = oracle.project_ellipsoids(go, po, sl)
    vol = oracle.draw_ellipsoids(vo, sl)
    got = to_np(rtkb.ops.joseph_forward_project(gl, vd, pd, to_gpu(vol), torch.zeros((n, 64, 64), device="cuda")))
    err, psnr, ok = phantoms.check_image_quality(got, ref, 1.28, 44.0, 255.0)
    assert ok, (err, psnr)
    want = oracle.joseph_forward(go, vo, vol, po)
    assert rel_l2(got, want) < REL_L2_TOL


def test_flat_panel_only_entry_points_refuse(rtkb, oracle):
    gl, go, vd, vo, pd, po, vol, pr = _case(rtkb, oracle, "radius_600", 4, (16, 16, 16), (24, 20, 4), (5.0, 5.0, 1.0))
    with pytest.raises(rtkb.RtkbError, match="flat panels only"):
        rtkb.ops.ray_box_lengths(gl, vd, pd)
    with pytest.raises(rtkb.RtkbError, match="flat panels only"):
        rtkb.ops.project_ellipsoids(gl, pd, phantoms.shepp_logan(10.0))


@pytest.mark.parametrize("params,radius", [
    ([(800.0, 1200.0, i * 360.0 / 24) for i in range(24)], 1200.0),
    ([(700.0, 1100.0, i * 360.0 / 24 + 3.0, 12.0, -7.0, 8.0, 4.0, 5.0, -3.0) for i in range(24)], 1100.0),
])
def test_cylindrical_voxel_backprojection_matches_oracle(rtkb, oracle, params, radius):
    """BackProjectionImageFilter's path for a cylinder centred on the source (radius = SDD)."""
    gl, go = pair_geometry(rtkb, oracle, params + [(700.0, 1100.0, 0.0)] * 2)
    gl.SetRadiusCylindricalDetector(radius)
    go.set_radius_cylindrical(radius)
    vd, vo = pair_image(rtkb, oracle, (36, 32, 40), (4.0, 4.5, 3.5), index=(2, -3, 1))
    pd, po = pair_image(rtkb, oracle, (64, 56, 24), (5.0, 5.0, 1.0), index=(-4, 3, 1))
    rng = np.random.default_rng(7)
    vol = rng.uniform(0.0, 1.0, size=oracle.shape_of(vo)).astype(np.float32).astype(np.float64)
    pr = rng.uniform(0.0, 1.0, size=oracle.shape_of(po)).astype(np.float32).astype(np.float64)
    ref = oracle.backproject(go, vo, po, pr, vol, fdk=False)
    got = to_np(rtkb.ops.voxel_backproject(gl, vd, pd, to_gpu(pr), to_gpu(vol)))
    assert rel_l2(got, ref) < REL_L2_TOL, rel_l2(got, ref)


def test_cylindrical_voxel_backprojection_refusals(rtkb, oracle):
    gl, go, vd, vo, pd, po, vol, pr = _case(rtkb, oracle, "radius_600", 4, (16, 16, 16), (24, 20, 4), (5.0, 5.0, 1.0))
    with pytest.raises(rtkb.RtkbError, match="centered on the source"):
        rtkb.ops.voxel_backproject(gl, vd, pd, to_gpu(pr), to_gpu(vol))
    gl.SetRadiusCylindricalDetector(1200.0)
    with pytest.raises(rtkb.RtkbError, match="FDK back projector"):
        rtkb.ops.fdk_backproject(gl, vd, pd, to_gpu(pr), to_gpu(vol))

"""GPU parity of the Joseph projector pair (rtkb_joseph_forward_project,
rtkb_joseph_back_project) against the FP64 oracle restating
include/rtkJosephForwardProjectionImageFilter.hxx and
include/rtkJosephBackProjectionImageFilter.hxx, RTK's box test
(test/rtkforwardprojectiontest.cxx) on the GPU, and adjointness
(test/rtkadjointoperatorstest.cxx).  Tolerance: relative L2 < 1e-5."""
import numpy as np
import pytest

from tests import phantoms
from tests.gpu_util import REL_L2_TOL, pair_geometry, pair_image, rel_l2, to_gpu, to_np

pytestmark = pytest.mark.gpu


def _case(rtkb, oracle, params, vsize, vspacing, psize, pspacing, vindex=(0, 0, 0), pindex=(0, 0, 0), seed=0):
    gl, go = pair_geometry(rtkb, oracle, params)
    vd, vo = pair_image(rtkb, oracle, vsize, vspacing, index=vindex)
    pd, po = pair_image(rtkb, oracle, psize, pspacing, index=pindex)
    rng = np.random.default_rng(seed)
    vol = rng.uniform(0.0, 1.0, size=oracle.shape_of(vo)).astype(np.float32).astype(np.float64)
    pr = rng.uniform(0.0, 1.0, size=oracle.shape_of(po)).astype(np.float32).astype(np.float64)
    return gl, go, vd, vo, pd, po, vol, pr


GEOMS = {
    "circular": lambda n: [(800.0, 1200.0, i * 360.0 / n) for i in range(n)],
    "offsets_tilts": lambda n: [(700.0, 1100.0, i * 360.0 / n + 3.0, 12.0, -7.0, 8.0, 4.0, 5.0, -3.0) for i in range(n)],
    "parallel": lambda n: [(500.0, 0.0, i * 180.0 / n, 3.0, -2.0) for i in range(n)],
    "steep_cone": lambda n: [(120.0, 300.0, i * 360.0 / n, 0.0, 0.0, 35.0) for i in range(n)],
}


@pytest.mark.parametrize("geom", sorted(GEOMS))
def test_joseph_forward_matches_oracle(rtkb, oracle, geom):
    gl, go, vd, vo, pd, po, vol, pr = _case(rtkb, oracle, GEOMS[geom](30), (40, 36, 44), (4.0, 4.5, 3.5),
                                            (72, 64, 30), (5.0, 5.0, 1.0), vindex=(2, -3, 1), pindex=(-4, 3, 0))
    ref = oracle.joseph_forward(go, vo, vol, po, pr)
    got = to_np(rtkb.ops.joseph_forward_project(gl, vd, pd, to_gpu(vol), to_gpu(pr)))
    assert rel_l2(got, ref) < REL_L2_TOL


@pytest.mark.parametrize("geom", sorted(GEOMS))
def test_joseph_back_matches_oracle(rtkb, oracle, geom):
    gl, go, vd, vo, pd, po, vol, pr = _case(rtkb, oracle, GEOMS[geom](24), (36, 32, 40), (4.0, 4.5, 3.5),
                                            (64, 56, 24), (5.0, 5.0, 1.0), vindex=(-1, 2, 0), pindex=(3, -2, 0))
    ref = oracle.joseph_back(go, vo, po, pr, vol)
    got = to_np(rtkb.ops.joseph_back_project(gl, vd, pd, to_gpu(pr), to_gpu(vol)))
    assert rel_l2(got, ref) < REL_L2_TOL


def test_joseph_adjoint_on_gpu(rtkb, oracle):
    gl, go, vd, vo, pd, po, vol, pr = _case(rtkb, oracle, GEOMS["offsets_tilts"](40), (48, 40, 44), (4.0,) * 3,
                                            (80, 70, 40), (6.0, 6.0, 1.0), seed=5)
    import torch

    fp = to_np(rtkb.ops.joseph_forward_project(gl, vd, pd, to_gpu(vol), torch.zeros(pr.shape, device="cuda")))
    bp = to_np(rtkb.ops.joseph_back_project(gl, vd, pd, to_gpu(pr), torch.zeros(vol.shape, device="cuda")))
    a, b = np.vdot(fp, pr), np.vdot(vol, bp)
    assert abs(a / b - 1) < 1e-5, (a, b)


def test_joseph_box_like_rtkforwardprojectiontest_on_gpu(rtkb, oracle):
    """RTK's inner-source box test with RTK's thresholds, on the GPU result."""
    import torch

    n = 45
    ones = np.ones((64, 64, 64))
    pd, po = pair_image(rtkb, oracle, (64, 64, n), (4.0,) * 3, origin=(-126.0,) * 3)
    vd = rtkb.make_desc((64, 64, 64), (4.0,) * 3, origin=(-126.0,) * 3)
    from tests.test_oracle_pins import _ray_box_lengths

    ref = None
    for q in range(4):
        params = [(47.6 / np.cos(np.deg2rad(-45.0 + i * 2.0)), 1000.0, q * 90 + (-45.0 + i * 2.0)) for i in range(n)]
        gl, go = pair_geometry(rtkb, oracle, params)
        if q == 0:
            ref = _ray_box_lengths(oracle, go, po, (-126.0, -126.0, -126.0), (126.0, 126.0, 47.6))
        got = to_np(rtkb.ops.joseph_forward_project(gl, vd, pd, to_gpu(ones),
                                                    torch.zeros((n, 64, 64), device="cuda")))
        err, psnr, ok = phantoms.check_image_quality(got, ref, 1.28, 44.0, 255.0)
        assert ok, (q, err, psnr)


def test_joseph_in_place(rtkb, oracle):
    gl, go, vd, vo, pd, po, vol, pr = _case(rtkb, oracle, GEOMS["circular"](20), (30, 30, 30), (4.0,) * 3,
                                            (50, 40, 20), (5.0, 5.0, 1.0), seed=9)
    ref_fp = oracle.joseph_forward(go, vo, vol, po, pr)
    t = to_gpu(pr)
    rtkb.ops.joseph_forward_project(gl, vd, pd, to_gpu(vol), t, out=t)
    assert rel_l2(to_np(t), ref_fp) < REL_L2_TOL
    ref_bp = oracle.joseph_back(go, vo, po, pr, vol)
    tv = to_gpu(vol)
    rtkb.ops.joseph_back_project(gl, vd, pd, to_gpu(pr), tv, out=tv)
    assert rel_l2(to_np(tv), ref_bp) < REL_L2_TOL


def test_joseph_cg_size_projection_subset(rtkb, oracle):
    """256^3 at 1 mm onto 512x384 pixels at 0.8 mm (the CG configuration):
    two stack slices (index offset into the geometry) against the oracle."""
    import torch

    n = 360
    params = [(1000.0, 1536.0, i * 360.0 / n) for i in range(n)]
    gl, go = pair_geometry(rtkb, oracle, params)
    vd, vo = pair_image(rtkb, oracle, (256, 256, 256), (1.0,) * 3)
    rng = np.random.default_rng(2)
    vol = rng.uniform(0, 1, size=(256, 256, 256)).astype(np.float32)
    for first in (0, 45):
        pd, po = pair_image(rtkb, oracle, (512, 384, 2), (0.8, 0.8, 1.0), index=(0, 0, first))
        ref = oracle.joseph_forward(go, vo, vol.astype(np.float64), po)
        got = to_np(rtkb.ops.joseph_forward_project(gl, vd, pd, to_gpu(vol), torch.zeros((2, 384, 512),
                                                                                          device="cuda")))
        assert rel_l2(got, ref) < REL_L2_TOL


@pytest.mark.parametrize("geom", sorted(GEOMS))
def test_joseph_sample_count_matches_oracle(rtkb, oracle, geom):
    """rtkb_joseph_sample_count (the work unit of the ray-cast throughput
    figure) equals the oracle's count from the same FP64 ray set-up."""
    gl, go, vd, vo, pd, po, vol, pr = _case(rtkb, oracle, GEOMS[geom](30), (40, 36, 44), (4.0, 4.5, 3.5),
                                            (72, 64, 30), (5.0, 5.0, 1.0), vindex=(2, -3, 1), pindex=(-4, 3, 0))
    assert rtkb.ops.joseph_sample_count(gl, vd, pd) == oracle.joseph_sample_count(go, vo, po)


def test_joseph_forward_short_stack_without_quads(rtkb, oracle):
    """Stacks of fewer than four projections (SART's subsets) take the four-tap
    loop without the quad copies: main-z (0 deg) and main-x (95 deg) rays."""
    params = [(700.0, 1100.0, 0.0, 6.0, -3.0), (700.0, 1100.0, 95.0, 6.0, -3.0)]
    gl, go, vd, vo, pd, po, vol, pr = _case(rtkb, oracle, params, (40, 32, 36), (4.0,) * 3, (72, 60, 2),
                                            (3.0, 3.0, 1.0))
    ref = oracle.joseph_forward(go, vo, vol, po, pr)
    got = to_np(rtkb.ops.joseph_forward_project(gl, vd, pd, to_gpu(vol), to_gpu(pr)))
    assert rtkb.ops.device_status() == 0
    assert rel_l2(got, ref) < REL_L2_TOL, rel_l2(got, ref)


def test_joseph_band_rows_and_autotune(rtkb, oracle, tmp_path):
    """Bands of 16, 32 and 64 detector rows regroup the projectors' blocks
    only: the forward projection is bit-identical to 8-row bands (each ray is
    one thread), the back projection equal up to the FP32 order of its
    reductions, both within the oracle's tolerance on a ragged detector
    (rows not a multiple of the band); the autotuner restores the setting it
    found when apply=False and caches its result."""
    import torch

    gl, go, vd, vo, pd, po, vol, pr = _case(rtkb, oracle, GEOMS["offsets_tilts"](30), (40, 36, 44), (4.0, 4.5, 3.5),
                                            (72, 100, 30), (5.0, 5.0, 1.0), vindex=(2, -3, 1), pindex=(-4, 3, 0))
    dv, dp = to_gpu(vol), to_gpu(pr)
    zp, zv = torch.zeros(pr.shape, device="cuda"), torch.zeros(vol.shape, device="cuda")
    out = {}
    try:
        for rows in (8, 16, 32, 64):
            assert rtkb.ops.joseph_band_rows(rows, rows) == (rows, rows)
            out[rows] = (to_np(rtkb.ops.joseph_forward_project(gl, vd, pd, dv, zp)),
                         to_np(rtkb.ops.joseph_back_project(gl, vd, pd, dp, zv)))
    finally:
        rtkb.ops.joseph_band_rows(8, 8)
    for rows in (16, 32, 64):
        assert np.array_equal(out[rows][0], out[8][0])
        assert rel_l2(out[rows][1], out[8][1]) < 1e-6
    assert rel_l2(out[64][0], oracle.joseph_forward(go, vo, vol, po)) < REL_L2_TOL
    assert rel_l2(out[64][1], oracle.joseph_back(go, vo, po, pr)) < REL_L2_TOL
    with pytest.raises(rtkb.RtkbError):
        rtkb.ops.joseph_band_rows(12, 8)
    path = str(tmp_path / "tune.json")
    res = rtkb.ops.joseph_autotune(gl, vd, pd, dv, dp, repeats=1, cache=path, apply=False)
    assert res["forward"] in (8, 16, 32, 64) and res["back"] in (8, 16, 32, 64)
    assert len(res["forward_ms"]) == 4 and len(res["back_ms"]) == 4
    assert rtkb.ops.joseph_band_rows() == (8, 8)
    assert rtkb.ops.joseph_autotune(gl, vd, pd, dv, dp, cache=path, apply=False) == res
    assert np.array_equal(to_np(dv), vol.astype(np.float32)) and np.array_equal(to_np(dp), pr.astype(np.float32))
    assert rtkb.ops.device_status() == 0

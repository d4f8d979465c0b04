"""GPU parity of the projection-domain filters (FDK weighting, Parker short
scan, displaced detector, ramp filter and their fused form) against the FP64
oracle.  The irregular 4-projection geometry and the 1e-5 / 95 dB thresholds
are those of RTK's CPU-vs-CUDA comparisons (test/rtkfdkprojweightcompcudatest.cxx:37-75,
test/rtkshortscancompcudatest.cxx, test/rtkdisplaceddetectorcompcudatest.cxx)."""
import numpy as np
import pytest

from tests import phantoms
from tests.gpu_util import REL_L2_TOL, pair_geometry, pair_image, rel_l2, to_gpu, to_np

pytestmark = pytest.mark.gpu

IRREGULAR = [(600., 700., 0., 84., 35, 23, 15, 21, 26), (500., 800., 45., 21., 12, 16, 546, 14, 41),
             (700., 900., 90., 68., 68, 54, 38, 35, 56), (900., 1000., 135., 48., 35, 84, 10, 84, 59)]


def _sl_projections(oracle, go, po):
    return oracle.project_ellipsoids(go, po, phantoms.shepp_logan(116.0))


def _rtk_cuda_cpu_check(got, ref):
    err, psnr, ok = phantoms.check_image_quality(got, ref, 1e-5, 95.0, 1.0)
    assert ok, (err, psnr)


def test_fdk_weight_irregular_geometry(rtkb, oracle):
    gl, go = pair_geometry(rtkb, oracle, IRREGULAR)
    pd, po = pair_image(rtkb, oracle, (128, 4, 4), (2.0, 2.0, 2.0), origin=(-127.0, -3.0, 0.0))
    p = _sl_projections(oracle, go, po).astype(np.float32).astype(np.float64)
    ref = oracle.fdk_weight(go, po, p)
    got = to_np(rtkb.ops.fdk_weight(gl, pd, to_gpu(p)))
    assert rel_l2(got, ref) < 1e-6
    _rtk_cuda_cpu_check(got, ref)


def test_fdk_weight_in_place_and_subset_index(rtkb, oracle):
    params = [(1000.0, 1536.0, i * 3.0, 5.0, -4.0, 2.0, 1.0, 3.0, 1.0) for i in range(30)]
    gl, go = pair_geometry(rtkb, oracle, params)
    pd, po = pair_image(rtkb, oracle, (96, 40, 12), (0.8, 0.8, 1.0), index=(-3, 2, 10))
    p = np.random.default_rng(1).uniform(0, 2, size=oracle.shape_of(po))
    ref = oracle.fdk_weight(go, po, p)
    t = to_gpu(p)
    rtkb.ops.fdk_weight(gl, pd, t, out=t)
    assert rel_l2(to_np(t), ref) < 1e-6


def test_parker_short_scan(rtkb, oracle):
    params = [(1000.0, 1536.0, i * 200.0 / 120, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0) for i in range(120)]
    gl, go = pair_geometry(rtkb, oracle, params)
    pd, po = pair_image(rtkb, oracle, (256, 8, 120), (1.0, 1.0, 1.0))
    p = np.random.default_rng(2).uniform(0, 1, size=oracle.shape_of(po))
    ref, short = oracle.parker_weight(go, po, p)
    got, gshort = rtkb.ops.parker_short_scan(gl, pd, to_gpu(p))
    assert short and gshort
    assert rel_l2(to_np(got), ref) < 1e-6


def test_parker_full_scan_is_a_copy(rtkb, oracle):
    params = [(1000.0, 1536.0, i * 3.0) for i in range(120)]
    gl, go = pair_geometry(rtkb, oracle, params)
    pd, po = pair_image(rtkb, oracle, (64, 4, 120), (1.0, 1.0, 1.0))
    p = np.random.default_rng(3).uniform(0, 1, size=oracle.shape_of(po)).astype(np.float32)
    got, short = rtkb.ops.parker_short_scan(gl, pd, to_gpu(p))
    assert not short
    assert np.array_equal(to_np(got), p.astype(np.float64))


def test_parker_irregular_like_rtkshortscancompcudatest(rtkb, oracle):
    gl, go = pair_geometry(rtkb, oracle, IRREGULAR)
    pd, po = pair_image(rtkb, oracle, (128, 4, 4), (2.0, 2.0, 2.0), origin=(-127.0, -3.0, 0.0))
    p = _sl_projections(oracle, go, po).astype(np.float32).astype(np.float64)
    ref, short = oracle.parker_weight(go, po, p)
    got, gshort = rtkb.ops.parker_short_scan(gl, pd, to_gpu(p))
    assert short == gshort
    _rtk_cuda_cpu_check(to_np(got), ref)


@pytest.mark.parametrize("offset", [80.0, -60.0])
def test_displaced_detector(rtkb, oracle, offset):
    params = [(1000.0, 1536.0, i * 6.0, offset, 0.0) for i in range(60)]
    gl, go = pair_geometry(rtkb, oracle, params)
    pd, po = pair_image(rtkb, oracle, (256, 6, 60), (0.8, 0.8, 1.0))
    p = np.random.default_rng(4).uniform(0, 1, size=oracle.shape_of(po))
    ref, i0, s0 = oracle.displaced_detector(go, po, p)
    got, od = rtkb.ops.displaced_detector(gl, pd, to_gpu(p))
    assert (od.index[0], od.size[0]) == (i0, s0)
    assert rel_l2(to_np(got), ref) < 1e-6


def test_displaced_irregular_like_rtkdisplaceddetectorcompcudatest(rtkb, oracle):
    gl, go = pair_geometry(rtkb, oracle, IRREGULAR)
    pd, po = pair_image(rtkb, oracle, (128, 4, 4), (2.0, 2.0, 2.0), origin=(-127.0, -3.0, 0.0))
    p = _sl_projections(oracle, go, po).astype(np.float32).astype(np.float64)
    ref, i0, s0 = oracle.displaced_detector(go, po, p)
    got, od = rtkb.ops.displaced_detector(gl, pd, to_gpu(p))
    assert (od.index[0], od.size[0]) == (i0, s0)
    _rtk_cuda_cpu_check(to_np(got), ref)


@pytest.mark.parametrize("offset,irregular", [(60.0, False), (-45.0, False), (50.0, True)])
def test_displaced_detector_offset_fov(rtkb, oracle, offset, irregular):
    """DisplacedDetectorForOffsetFieldOfViewImageFilter (the variant RTK's CPU
    rtkfdk chains) on detectors displaced to either side and on an irregular
    geometry (per-projection distances, offsets and source offsets): padded
    region and weights (from the field of view's disc) against the oracle."""
    if irregular:
        params = [(900.0 + 3 * (i % 7), 1400.0 + 5 * (i % 5), i * 3.7 + 1.0, offset + (i % 3), 2.0, 0.0, 0.0, 4.0, 1.0)
                  for i in range(97)]
    else:
        params = [(1000.0, 1536.0, i * 6.0, offset, 0.0) for i in range(60)]
    gl, go = pair_geometry(rtkb, oracle, params)
    pd, po = pair_image(rtkb, oracle, (256, 6, len(params)), (0.8, 0.8, 1.0))
    p = np.random.default_rng(5).uniform(0, 1, size=oracle.shape_of(po))
    ref, i0, s0 = oracle.displaced_detector_offset_fov(go, po, p)
    got, od = rtkb.ops.displaced_detector_offset_fov(gl, pd, to_gpu(p))
    assert (od.index[0], od.size[0]) == (i0, s0) and s0 == 512
    assert rel_l2(to_np(got), ref) < 1e-6


def test_offset_fov_like_rtkdisplaceddetectorcompoffsettest(rtkb, oracle):
    """RTK's test/rtkdisplaceddetectorcompoffsettest.cxx: on its four-projection
    geometry and Shepp-Logan stack the offset-field-of-view variant equals
    DisplacedDetectorImageFilter (CheckImageQuality 1e-6, 100 dB, reference 1)."""
    params = [(600., 560., 0., 3., 0., 0., 0., 2., 0.), (500., 545., 90., 2., 0., 0., 0., 4., 0.),
              (700., 790., 180., 8., 0., 0., 0., 5., 0.), (900., 935., 270., 4., 0., 0., 0., 8., 0.)]
    gl, go = pair_geometry(rtkb, oracle, params)
    pd, po = pair_image(rtkb, oracle, (128, 4, 4), (8.0, 2.0, 2.0), origin=(-508.0, -3.0, 0.0))
    p = _sl_projections(oracle, go, po).astype(np.float32)
    a, oda = rtkb.ops.displaced_detector_offset_fov(gl, pd, to_gpu(p))
    b, odb = rtkb.ops.displaced_detector(gl, pd, to_gpu(p))
    assert (oda.index[0], oda.size[0]) == (odb.index[0], odb.size[0])
    err, psnr, ok = phantoms.check_image_quality(to_np(a), to_np(b), 1e-6, 100.0, 1.0)
    assert ok, (err, psnr)


def test_fdk_preprocess_offset_fov(rtkb, oracle):
    """The fused FDK preprocessing with the offset-field-of-view displaced
    detector (rtkfdk's CPU chain: displaced detector, Parker, FDK weights,
    ramp) against the oracle's filters in sequence."""
    params = [(1000.0, 1536.0, i * 4.0, 70.0, 1.0) for i in range(90)]
    gl, go = pair_geometry(rtkb, oracle, params)
    pd, po = pair_image(rtkb, oracle, (200, 9, 90), (0.8, 0.8, 1.0))
    p = np.random.default_rng(6).uniform(0, 1, size=oracle.shape_of(po))
    q, i0, s0 = oracle.displaced_detector_offset_fov(go, po, p)
    qo = oracle.image((s0, 9, 90), (0.8, 0.8, 1.0), origin=tuple(po.origin), index=(i0, 0, 0))
    ref = oracle.ramp_filter(qo, oracle.fdk_weight(go, qo, q), oracle.ramp_params(hann=0.9))
    got, od = rtkb.ops.fdk_preprocess(gl, pd, to_gpu(p), rtkb.ops.ramp_params(hann=0.9), displaced="offset_fov")
    assert (od.index[0], od.size[0]) == (i0, s0)
    assert rel_l2(to_np(got), ref) < REL_L2_TOL


@pytest.mark.parametrize("nu,window", [(256, {}), (1024, {"hann": 1.0}), (300, {"hann": 0.8}),
                                       (128, {"cosine": 0.7}), (512, {"hamming": 0.9}),
                                       (200, {"ramlak": 0.6}), (256, {"shepplogan": 0.8}),
                                       (256, {"truncation": 0.1}), (2048, {"hann": 0.5}),
                                       (600, {"pad": 1}), (700, {"truncation": 0.3}),
                                       (600, {"truncation": 0.9, "pad": 1}), (4096, {"hann": 0.9}),
                                       (300, {"gpf": 13}), (99, {"gpf": 13, "pad": 1, "hann": 0.9}),
                                       (700, {"gpf": 13, "truncation": 0.3}), (1000, {"gpf": 13, "cosine": 0.8})])
def test_ramp_filter(rtkb, oracle, nu, window):
    """Every form of the ramp kernel: shared-memory passes (N < 1024), the
    register-resident first and last passes with the upper-zero form (row in
    the lower half, no mirror: 300, 1024, 2048, 4096 columns), without it (600
    columns padded to 1024 only) and with the truncation mirror (700 columns;
    600 with an extent wider than the zero padding); with a greatest prime
    factor of 13 (RTK built with FFTW) the padded lengths 600, 99, 1400 and
    2000, whose period-P convolution runs embedded in a power-of-two FFT of
    length >= 2P - 1."""
    pd, po = pair_image(rtkb, oracle, (nu, 7, 3), (0.5, 0.5, 1.0))
    rng = np.random.default_rng(nu)
    p = rng.uniform(0, 1, size=oracle.shape_of(po))
    ref = oracle.ramp_filter(po, p, oracle.ramp_params(**window))
    got = to_np(rtkb.ops.ramp_filter(pd, to_gpu(p), rtkb.ops.ramp_params(**window)))
    assert rel_l2(got, ref) < REL_L2_TOL


@pytest.mark.parametrize("nu,nv,n,window", [(300, 200, 2, {"hann_y": 0.8}), (1024, 768, 2, {"hann": 1.0, "hann_y": 0.6}),
                                            (128, 40, 3, {"hann_y": 1.0, "pad_y": 1}),
                                            (700, 33, 3, {"cosine": 0.8, "hann_y": 0.4, "truncation": 0.3}),
                                            (57, 1, 4, {"hann_y": 0.9}),
                                            (300, 200, 2, {"hann_y": 0.8, "gpf": 13, "truncation": 0.2})])
def test_ramp_filter_2d_kernel(rtkb, oracle, nu, nv, n, window):
    """HannCutFrequencyY: the 2-D kernel (the row filter, then every column
    zero-padded to the padded height and filtered with the vertical window by
    the same FFT kernel on a transposed copy) against the oracle's literal 2-D
    path; padded heights 512, 2048 (register-resident passes), 64 (zero pad 1),
    128 and 2 (one detector row)."""
    pd, po = pair_image(rtkb, oracle, (nu, nv, n), (0.5, 0.5, 1.0))
    p = np.random.default_rng(nu + nv).uniform(0, 1, size=oracle.shape_of(po))
    ref = oracle.ramp_filter(po, p, oracle.ramp_params(**window))
    got = to_np(rtkb.ops.ramp_filter(pd, to_gpu(p), rtkb.ops.ramp_params(**window)))
    assert rel_l2(got, ref) < REL_L2_TOL, rel_l2(got, ref)
    flat = {k: v for k, v in window.items() if k not in ("hann_y", "pad_y")}
    # the window acts (with one row, padded to two, it scales the row by 0.75)
    assert rel_l2(got, oracle.ramp_filter(po, p, oracle.ramp_params(**flat))) > 1e-3


def test_fdk_preprocess_2d_kernel_single_and_batched(rtkb, oracle):
    """The fused FDK preprocessing with HannCutFrequencyY, one stack against
    the oracle (weights, then the 2-D ramp), and the batched call with one
    stack using the 2-D kernel beside one that does not: each output
    bit-identical to its own single call."""
    cases = []
    for k, (nu, nv, n) in enumerate([(200, 40, 30), (120, 24, 20)]):
        params = [(1000.0, 1500.0, i * 360.0 / n, 3.0 * k, 1.0) for i in range(n)]
        gl, go = pair_geometry(rtkb, oracle, params)
        pd, po = pair_image(rtkb, oracle, (nu, nv, n), (0.8, 0.8, 1.0))
        p = np.random.default_rng(30 + k).uniform(0, 1, size=oracle.shape_of(po)).astype(np.float32)
        cases.append((gl, go, pd, po, p))
    ramp2 = rtkb.ops.ramp_params(hann=0.8, hann_y=0.7)
    gl, go, pd, po, p = cases[0]
    one, _ = rtkb.ops.fdk_preprocess(gl, pd, to_gpu(p), ramp2)
    ref = oracle.ramp_filter(po, oracle.fdk_weight(go, po, p.astype(np.float64)),
                             oracle.ramp_params(hann=0.8, hann_y=0.7))
    assert rel_l2(to_np(one), ref) < REL_L2_TOL
    batch = rtkb.ops.fdk_preprocess_batch([(c[0], c[2], to_gpu(c[4]), None) for c in cases], ramp2)
    for (gl, go, pd, po, p), (got, od) in zip(cases, batch):
        single, _ = rtkb.ops.fdk_preprocess(gl, pd, to_gpu(p), ramp2)
        assert np.array_equal(to_np(got), to_np(single))
    assert rtkb.ops.device_status() == 0


def test_ramp_kernel_matches_oracle(rtkb, oracle):
    for nu, kw in ((256, {}), (1000, {"hann": 0.7}), (513, {"shepplogan": 1.0})):
        n, k = rtkb.ops.ramp_kernel(nu, 0.388, rtkb.ops.ramp_params(**kw))
        assert n == oracle.ramp_padded_size(nu, oracle.ramp_params(**kw))
        np.testing.assert_allclose(k, oracle.ramp_kernel(n, 0.388, oracle.ramp_params(**kw)), rtol=1e-12,
                                   atol=1e-12)


@pytest.mark.parametrize("displaced,short", [(False, False), (True, False), (False, True), (True, True)])
def test_fdk_preprocess_fused(rtkb, oracle, displaced, short):
    arc = 220.0 if short else 360.0
    params = [(1000.0, 1536.0, i * arc / 90, 60.0 if displaced else 0.0, 2.0) for i in range(90)]
    gl, go = pair_geometry(rtkb, oracle, params)
    pd, po = pair_image(rtkb, oracle, (200, 9, 90), (0.8, 0.8, 1.0))
    p = np.random.default_rng(5).uniform(0, 1, size=oracle.shape_of(po))
    q, qo = p, po
    if displaced:
        q, i0, s0 = oracle.displaced_detector(go, po, q)
        qo = oracle.image((s0, 9, 90), (0.8, 0.8, 1.0), origin=tuple(po.origin), index=(i0, 0, 0))
    if short:
        q, _ = oracle.parker_weight(go, qo, q)
    q = oracle.fdk_weight(go, qo, q)
    ref = oracle.ramp_filter(qo, q, oracle.ramp_params(hann=0.9))
    got, od = rtkb.ops.fdk_preprocess(gl, pd, to_gpu(p), rtkb.ops.ramp_params(hann=0.9), displaced=displaced,
                                      short_scan=short)
    assert (od.index[0], od.size[0]) == (qo.index[0], qo.size[0])
    assert rel_l2(to_np(got), ref) < REL_L2_TOL


def test_fdk_gpu_shepp_logan_like_rtkfdktest(rtkb, oracle):
    """Full GPU FDK (fused preprocessing + backprojection) against the oracle
    FDK, and against the phantom with rtkfdktest's thresholds."""
    n = 180
    params = [(600.0, 1200.0, i * 360.0 / n, 0, 0, 0, 0, 20, 15) for i in range(n)]
    gl, go = pair_geometry(rtkb, oracle, params)
    vd, vo = pair_image(rtkb, oracle, (128, 128, 128), (2.0,) * 3, origin=(-127.0,) * 3)
    pd, po = pair_image(rtkb, oracle, (128, 128, n), (4.0,) * 3, origin=(-254.0,) * 3)
    sl = phantoms.shepp_logan(116.0)
    p = oracle.project_ellipsoids(go, po, sl).astype(np.float32).astype(np.float64)
    ref_img = oracle.draw_ellipsoids(vo, sl)
    filt = oracle.ramp_filter(po, oracle.fdk_weight(go, po, p), oracle.ramp_params())
    ref = oracle.backproject(go, vo, po, filt, fdk=True)
    import torch

    f, _ = rtkb.ops.fdk_preprocess(gl, pd, to_gpu(p))
    rec = to_np(rtkb.ops.fdk_backproject(gl, vd, pd, f, torch.zeros((128, 128, 128), device="cuda")))
    assert rel_l2(rec, ref) < REL_L2_TOL
    err, psnr, ok = phantoms.check_image_quality(rec * phantoms.fov_mask(go, vo, po), ref_img, 0.03, 26.0, 2.0)
    assert ok, (err, psnr)


def test_fdk_gpu_like_rtkrampfiltertest(rtkb, oracle):
    """RTK's rtkrampfiltertest (test/rtkrampfiltertest.cxx) on the GPU FDK:
    Shepp-Logan (scale 128) projected onto 180 x 128^2 at 4 mm (SID 600, SDD
    1200), reconstructed on 128^3 at 2 mm and compared over the whole volume
    with its CheckImageQuality thresholds: (1) Gaussian noise of standard
    deviation 1 (seeded here) with the Hann window at 0.8, error per pixel
    <= 0.72 and PSNR >= 22.4; (1.5) the same with HannCutFrequencyY 0.8 (the
    2-D kernel), 0.74 and 21.8, and within 1e-5 of the oracle's FDK; (2) no
    noise, the detector cut to 114 columns and truncation correction 0.1,
    0.12 and 20.8."""
    import torch

    n = 180
    params = [(600.0, 1200.0, i * 360.0 / n) for i in range(n)]
    gl, go = pair_geometry(rtkb, oracle, params)
    vd, vo = pair_image(rtkb, oracle, (128, 128, 128), (2.0,) * 3, origin=(-127.0,) * 3)
    pd, po = pair_image(rtkb, oracle, (128, 128, n), (4.0,) * 3, origin=(-254.0,) * 3)
    sl = phantoms.shepp_logan(128.0)
    ref_img = oracle.draw_ellipsoids(vo, sl)
    p = oracle.project_ellipsoids(go, po, sl)
    noisy = (p + np.random.default_rng(1).normal(0.0, 1.0, size=p.shape)).astype(np.float32)

    def fdk(desc, proj, **ramp):
        f, fd = rtkb.ops.fdk_preprocess(gl, desc, to_gpu(proj), rtkb.ops.ramp_params(**ramp))
        return to_np(rtkb.ops.fdk_backproject(gl, vd, fd, f, torch.zeros((128, 128, 128), device="cuda")))

    rec = fdk(pd, noisy, hann=0.8)
    err, psnr, ok = phantoms.check_image_quality(rec, ref_img, 0.72, 22.4, 2.0)
    assert ok, (err, psnr)
    rec = fdk(pd, noisy, hann=0.8, hann_y=0.8)
    err, psnr, ok = phantoms.check_image_quality(rec, ref_img, 0.74, 21.8, 2.0)
    assert ok, (err, psnr)
    n64 = noisy.astype(np.float64)
    filt = oracle.ramp_filter(po, oracle.fdk_weight(go, po, n64), oracle.ramp_params(hann=0.8, hann_y=0.8))
    assert rel_l2(rec, oracle.backproject(go, vo, po, filt, fdk=True)) < REL_L2_TOL
    pdc, poc = pair_image(rtkb, oracle, (114, 128, n), (4.0,) * 3, origin=(-254.0,) * 3)
    cropped = oracle.project_ellipsoids(go, poc, sl).astype(np.float32)
    rec = fdk(pdc, cropped, truncation=0.1)
    err, psnr, ok = phantoms.check_image_quality(rec, ref_img, 0.12, 20.8, 2.0)
    assert ok, (err, psnr)
    assert rtkb.ops.device_status() == 0


def test_project_ellipsoids_matches_oracle(rtkb, oracle):
    params = [(1000.0, 1536.0, i * 12.0, 5.0, -3.0, 2.0, 1.0, 4.0, 2.0) for i in range(30)]
    gl, go = pair_geometry(rtkb, oracle, params)
    pd, po = pair_image(rtkb, oracle, (160, 120, 30), (1.5, 1.5, 1.0), index=(-3, 2, 0))
    ell = np.concatenate([phantoms.random_ellipsoids(12, 3, centre_radius=40.0), phantoms.shepp_logan(60.0)])
    ref = oracle.project_ellipsoids(go, po, ell)
    got = to_np(rtkb.ops.project_ellipsoids(gl, pd, ell))
    assert rel_l2(got, ref) < 1e-6


@pytest.mark.parametrize("displaced", [False, True])
def test_fdk_preprocess_batch_equals_one_call_per_stack(rtkb, oracle, displaced):
    """rtkb_fdk_preprocess_batch on stacks of different widths (three padded
    row lengths, one of them shared by two stacks), projection counts, index
    offsets and geometries: every output bit-identical to its own
    rtkb_fdk_preprocess call (the same kernel over a one-stack table), one
    within the oracle's tolerance; an invalid problem fails the whole call."""
    rng = np.random.default_rng(21)
    cases = []
    for k, (nu, nv, n) in enumerate([(200, 9, 90), (120, 17, 47), (230, 5, 61), (500, 12, 33)]):
        params = [(900.0 + 50 * k, 1400.0 + 40 * k, i * 360.0 / n, (40.0 if displaced else 0.0) + k, 1.0)
                  for i in range(n)]
        gl, go = pair_geometry(rtkb, oracle, params)
        pd, po = pair_image(rtkb, oracle, (nu, nv, n), (0.8, 0.8, 1.0), index=(-k, k, 0))
        p = rng.uniform(0, 1, size=oracle.shape_of(po)).astype(np.float32)
        cases.append((gl, go, pd, po, p))
    ramp = rtkb.ops.ramp_params(hann=0.7)
    batch = rtkb.ops.fdk_preprocess_batch([(gl, pd, to_gpu(p), None) for gl, go, pd, po, p in cases], ramp,
                                          displaced=displaced)
    for (gl, go, pd, po, p), (got, od) in zip(cases, batch):
        one, od1 = rtkb.ops.fdk_preprocess(gl, pd, to_gpu(p), ramp, displaced=displaced)
        assert (od.index[0], od.size[0]) == (od1.index[0], od1.size[0])
        assert np.array_equal(to_np(got), to_np(one))
    gl, go, pd, po, p = cases[1]
    q, qo = p.astype(np.float64), po
    if displaced:
        q, i0, s0 = oracle.displaced_detector(go, po, q)
        qo = oracle.image((s0, po.size[1], po.size[2]), (0.8, 0.8, 1.0), origin=tuple(po.origin),
                          index=(i0, po.index[1], 0))
    ref = oracle.ramp_filter(qo, oracle.fdk_weight(go, qo, q), oracle.ramp_params(hann=0.7))
    assert rel_l2(to_np(batch[1][0]), ref) < REL_L2_TOL
    bad = rtkb.make_desc((120, 17, 500), (0.8, 0.8, 1.0))  # more projections than the geometry has
    with pytest.raises(rtkb.RtkbError):
        rtkb.ops.fdk_preprocess_batch([(cases[0][0], cases[0][2], to_gpu(cases[0][4]), None),
                                       (cases[1][0], bad, to_gpu(np.zeros((500, 17, 120), np.float32)), None)],
                                      ramp)
    assert rtkb.ops.device_status() == 0

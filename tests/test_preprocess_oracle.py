"""CPU checks of the oracle's raw-to-line-integral pieces (test
infrastructure): rtk::LUTbasedVariableI0RawToAttenuationImageFilter against
its closed form, and rtk::I0EstimationProjectionFilter on images whose
background mode and dynamic range are known.  RTK's own tests of these filters
(test/rtklutbasedvarI0rawtoatttest.cxx, test/rtkI0estimationtest.cxx) run them
without checking values; their inputs are reused below."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.mark.parametrize("i0,idark", [(65535.0, 0.0), (4000.0, 100.0), (51.0, 0.0), (5.0, 10.0)])
def test_raw_to_attenuation_closed_form(i0, idark):
    O.build()
    raw = np.arange(65536, dtype=np.uint16)
    got = O.raw_to_attenuation(raw, i0, idark).astype(np.float64)
    want = np.log(max(i0 - idark, 1.0)) - np.log(np.maximum(raw.astype(np.float64) - idark, 1.0))
    np.testing.assert_allclose(got, want, rtol=2e-6, atol=2e-6)
    # counts at or below IDark + 1 read as one count above the dark level
    low = raw.astype(np.float64) - idark <= 1.0
    assert np.all(got[low] == np.float32(np.log(max(i0 - idark, 1.0))))


def test_raw_to_attenuation_like_rtklutbasedvarI0rawtoatttest():
    """test/rtklutbasedvarI0rawtoatttest.cxx: 10x10 raw images filled with 0..I0, converted with I0 / 2."""
    O.build()
    for i in range(10):
        i0 = 10 * i + 1
        raw = (np.arange(100) % (i0 + 1)).astype(np.uint16).reshape(10, 10)
        got = O.raw_to_attenuation(raw, i0 // 2, 0.0)
        assert np.all(np.isfinite(got))
        assert got.max() == np.float32(np.log(max(i0 // 2, 1)))  # raw values of 0 and 1


def test_i0_estimation_finds_the_background_mode():
    O.build()
    rng = np.random.default_rng(0)
    # 150x150: an object of counts 1000-1399 (about 63 per 4-count bin, above the dynamic threshold of 20) on a
    # background of 4000 +- 6 counts
    img = rng.integers(3994, 4007, size=(150, 150)).astype(np.uint16)
    img[40:110, 30:120] = rng.integers(1000, 1400, size=(70, 90))
    est = O.i0_estimation(img, bit_shift=2, dyn_threshold=20)
    assert 3992 <= est["i0"] <= 4004 and est["i0"] % 4 == 0
    assert est["imin"] == 1000 and est["imax"] == 4004
    # the background spans bins 998-1001; the half-maximum walk stops at the first bin on each side at or below
    # half the mode's count, at most bins 997 and 1002
    assert 0 < est["i0_fwhm"] <= (1002 - 997) * 4
    # bit shift 0: the mode is one of the background values
    est0 = O.i0_estimation(img, bit_shift=0, dyn_threshold=20)
    assert 3994 <= est0["i0"] <= 4006


def test_i0_estimation_like_rtkI0estimationtest():
    """test/rtkI0estimationtest.cxx's inputs (150x150 uniform images, minimum 3200, maximum 3800 + 400 i, bit shift
    3): the estimate lies in the upper quarter of each image's range."""
    O.build()
    rng = np.random.default_rng(1)
    for i in range(10):
        hi = 3800 + 400 * i
        img = rng.integers(3200, hi + 1, size=(150, 150)).astype(np.uint16)
        est = O.i0_estimation(img, bit_shift=3, dyn_threshold=20)
        assert 3 * est["imax"] // 4 - 8 <= est["i0"] <= hi
        assert est["imin"] <= 3200 + 8 and est["imax"] >= hi - 16


@pytest.mark.parametrize("c", [[2.0, 2.0], [0.05, 0.3, 2.0], [0.0687, 2.5, 0.6, -0.2, 0.1]])
def test_water_precorrection_like_rtkwaterprecorrectiontest(c):
    """test/rtkwaterprecorrectiontest.cxx: orders 2, 3 and 5 map a constant 1.5 to 5."""
    out = O.water_precorrection(np.full((16, 16), 1.5, dtype=np.float32), c)
    np.testing.assert_allclose(out, 5.0, atol=1e-4)


def test_water_precorrection_pass_through():
    v = np.random.default_rng(0).normal(size=(3, 5)).astype(np.float32)
    for c in ([], [0.0, 1.0], [0.0]):
        assert np.array_equal(O.water_precorrection(v, c), v)
    assert np.all(O.water_precorrection(v, [2.5]) == np.float32(2.5))

"""Raw 16-bit projections to line integrals on the GPU (rtkb_i0_estimation,
rtkb_raw_to_attenuation) against the oracle restating
include/rtkI0EstimationProjectionFilter.hxx and
include/rtkLUTbasedVariableI0RawToAttenuationImageFilter.hxx: bit-exact, as
both are integer histograms and table look-ups."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _u16(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint16).view(np.int16)).cuda().view(torch.uint16)


@pytest.mark.parametrize("shape,i0,idark", [((7, 64, 80), 65535.0, 0.0), ((3, 33, 45), 4000.0, 100.0),
                                            ((1, 10, 10), 5.0, 10.0), ((2, 1, 9), 30000.0, 2.5)])
def test_raw_to_attenuation_bit_exact(rtkb, oracle, shape, i0, idark):
    raw = np.random.default_rng(3).integers(0, 65536, size=shape).astype(np.uint16)
    desc = rtkb.make_desc((shape[2], shape[1], shape[0]))
    got = rtkb.ops.raw_to_attenuation(desc, _u16(raw), i0, idark).cpu().numpy()
    want = oracle.raw_to_attenuation(raw, i0, idark)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("bit_shift", [0, 2, 3])
def test_i0_estimation_matches_oracle(rtkb, oracle, bit_shift):
    rng = np.random.default_rng(bit_shift)
    img = rng.integers(3994, 4007, size=(4, 150, 150)).astype(np.uint16)
    img[:, 40:110, 30:120] = rng.integers(1000, 1400, size=(4, 70, 90))
    desc = rtkb.make_desc((150, 150, 4))
    assert rtkb.ops.i0_estimation(desc, _u16(img), bit_shift, 20) == oracle.i0_estimation(img, bit_shift, 20)


def test_i0_estimation_like_rtkI0estimationtest_on_gpu(rtkb, oracle):
    """test/rtkI0estimationtest.cxx's inputs: 150x150 uniform images between 3200 and 3800 + 400 i, bit shift 3."""
    rng = np.random.default_rng(1)
    desc = rtkb.make_desc((150, 150, 1))
    for i in range(10):
        img = rng.integers(3200, 3800 + 400 * i + 1, size=(1, 150, 150)).astype(np.uint16)
        assert rtkb.ops.i0_estimation(desc, _u16(img), 3, 20) == oracle.i0_estimation(img, 3, 20)


def test_estimated_i0_into_the_conversion(rtkb, oracle):
    """ProjectionsReader's chain: the estimated I0 configures the look-up table."""
    rng = np.random.default_rng(9)
    img = rng.integers(3994, 4007, size=(2, 120, 100)).astype(np.uint16)
    img[:, 30:90, 20:80] = rng.integers(500, 3000, size=(2, 60, 60))
    desc = rtkb.make_desc((100, 120, 2))
    est = rtkb.ops.i0_estimation(desc, _u16(img))
    got = rtkb.ops.raw_to_attenuation(desc, _u16(img), est["i0"]).cpu().numpy()
    assert np.array_equal(got, oracle.raw_to_attenuation(img, oracle.i0_estimation(img)["i0"]))
    assert abs(float(np.median(got[:, :5, :5]))) < 0.01  # the background reads as no attenuation

"""Water precorrection (rtkb_water_precorrection) against the oracle restating
include/rtkWaterPrecorrectionImageFilter.hxx: bit-exact, as both evaluate the
polynomial with the filter's float and double operations in the same order."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("c", [[], [0.0], [3.0], [0.0, 1.0], [0.5, 1.2], [0.05, 0.3, 2.0],
                               [0.0687, 2.5, 0.6, -0.2, 0.1], list(np.linspace(-1.0, 1.0, 16))])
def test_water_precorrection_bit_exact(rtkb, oracle, c):
    v = np.random.default_rng(len(c)).uniform(0.0, 4.0, size=(5, 33, 47)).astype(np.float32)
    desc = rtkb.make_desc((47, 33, 5))
    got = rtkb.ops.water_precorrection(desc, torch.from_numpy(v).cuda(), c).cpu().numpy()
    assert np.array_equal(got, oracle.water_precorrection(v, c))
    # in place
    x = torch.from_numpy(v).cuda()
    rtkb.ops.water_precorrection(desc, x, c, out=x)
    assert np.array_equal(x.cpu().numpy(), got)


def test_water_precorrection_rtk_cases_and_limits(rtkb):
    desc = rtkb.make_desc((16, 16, 1))
    for c in ([2.0, 2.0], [0.05, 0.3, 2.0], [0.0687, 2.5, 0.6, -0.2, 0.1]):
        out = rtkb.ops.water_precorrection(desc, torch.full((1, 16, 16), 1.5, device="cuda"), c)
        assert torch.allclose(out, torch.full_like(out, 5.0), atol=1e-4)
    with pytest.raises(rtkb.RtkbError, match="at most 16"):
        rtkb.ops.water_precorrection(desc, torch.zeros((1, 16, 16), device="cuda"), [0.1] * 17)

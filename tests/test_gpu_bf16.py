"""BF16 storage variant of the FDK and voxel-based backprojectors
(rtkb_fdk_backproject_bf16, rtkb_voxel_backproject_bf16, rtkb_convert_to_bf16).

Parity: the FP64 oracle (include/rtkFDKBackProjectionImageFilter.hxx,
include/rtkBackProjectionImageFilter.hxx restated) is fed the same
BF16-rounded projection values, so the only remaining difference is the FP32
interpolation and accumulation: relative L2 < 1e-5, as for FP32 stacks.
Precision cost: against the FP32 stack, BF16 storage (8-bit mantissa,
relative rounding 2^-9) changes the backprojection by ~1e-3 relative L2."""
import numpy as np
import pytest

from tests.gpu_util import REL_L2_TOL, pair_geometry, pair_image, rel_l2, to_gpu, to_np

pytestmark = pytest.mark.gpu


def _circular(n, sid, sdd, arc=360.0, pox=0.0, poy=0.0):
    return [(sid, sdd, i * arc / n, pox, poy) for i in range(n)]


CASES = {
    # name: (params, vsize, vspacing, psize, pspacing, fdk, pindex)
    "fdk_c1": (_circular(180, 1000.0, 1500.0), (128, 128, 128), (1.6,) * 3, (256, 256, 180), (1.0,) * 3, True,
               (0, 0, 0)),
    "voxel": (_circular(90, 1000.0, 1500.0), (96, 80, 72), (2.0,) * 3, (256, 200, 90), (1.0,) * 3, False, (0, 0, 0)),
    "displaced_ragged": (_circular(64, 1000.0, 1536.0, pox=40.0, poy=-3.0), (61, 37, 45), (3.0, 2.5, 3.5),
                         (512, 120, 64), (1.0, 1.2, 1.0), True, (-256, 4, 0)),
    # 250 columns: rows of 500 bytes cannot be described to TMA, the plain-load path stages the boxes
    "plain_load_rows": (_circular(48, 900.0, 1400.0), (64, 48, 64), (2.0,) * 3, (250, 130, 48), (1.1,) * 3, True,
                        (0, 0, 0)),
    "generic_tilted": ([(1000.0, 1500.0, i * 9.0, 3.0, -2.0, 10.0, 5.0, 0.0, 0.0) for i in range(40)], (48, 40, 44),
                       (2.5,) * 3, (160, 150, 40), (1.0,) * 3, True, (0, 0, 0)),
}


def _bf16_round(a):
    import torch

    return torch.from_numpy(np.asarray(a, np.float32)).to(torch.bfloat16).double().numpy()


@pytest.mark.parametrize("name", sorted(CASES))
def test_bf16_backprojection_matches_oracle_on_bf16_values(rtkb, oracle, name):
    params, vsize, vsp, psize, psp, fdk, pindex = CASES[name]
    gl, go = pair_geometry(rtkb, oracle, params)
    vd, vo = pair_image(rtkb, oracle, vsize, vsp)
    pd, po = pair_image(rtkb, oracle, psize, psp, index=pindex)
    rng = np.random.default_rng(len(name))
    p32 = rng.uniform(-1.0, 1.0, size=oracle.shape_of(po)).astype(np.float32)
    pb = _bf16_round(p32)
    ref = oracle.backproject(go, vo, po, pb, np.zeros(oracle.shape_of(vo)), fdk=fdk)
    dpb = rtkb.ops.to_bf16(to_gpu(p32))
    z = to_gpu(np.zeros(oracle.shape_of(vo)))
    fn = rtkb.ops.fdk_backproject if fdk else rtkb.ops.voxel_backproject
    got = to_np(fn(gl, vd, pd, dpb, z))
    assert rtkb.ops.device_status() == 0
    assert rel_l2(got, ref) < REL_L2_TOL, rel_l2(got, ref)


def test_bf16_conversion_is_round_to_nearest_even(rtkb):
    import torch

    rng = np.random.default_rng(3)
    x = np.concatenate([rng.standard_normal(100000).astype(np.float32) * 10 ** rng.uniform(-20, 20, 100000),
                        np.array([0.0, -0.0, 1.0, 1.00390625, 1.01171875, 3.0e38, -1e-40], np.float32)])
    got = rtkb.ops.to_bf16(to_gpu(x)).view(torch.int16).cpu().numpy()
    ref = torch.from_numpy(x).to(torch.bfloat16).view(torch.int16).numpy()
    assert np.array_equal(got, ref)


def test_bf16_storage_precision_cost(rtkb, oracle):
    """What BF16 storage costs against the FP32 stack on smooth, realistic
    projections (a phantom's line integrals): ~1e-3 relative L2."""
    from tests import phantoms

    params, vsize, vsp, psize, psp, fdk, pindex = CASES["fdk_c1"]
    gl, go = pair_geometry(rtkb, oracle, params)
    vd, vo = pair_image(rtkb, oracle, vsize, vsp, origin=(-101.6,) * 3)
    pd, po = pair_image(rtkb, oracle, psize, psp, origin=(-127.5, -127.5, 0.0))
    p = oracle.project_ellipsoids(go, po, phantoms.shepp_logan(90.0))
    ref = oracle.backproject(go, vo, po, p.astype(np.float32).astype(np.float64), np.zeros(oracle.shape_of(vo)))
    z = to_gpu(np.zeros(oracle.shape_of(vo)))
    got32 = to_np(rtkb.ops.fdk_backproject(gl, vd, pd, to_gpu(p), z))
    got16 = to_np(rtkb.ops.fdk_backproject(gl, vd, pd, rtkb.ops.to_bf16(to_gpu(p)), z))
    e32, e16 = rel_l2(got32, ref), rel_l2(got16, ref)
    assert e32 < REL_L2_TOL
    assert 1e-5 < e16 < 1e-2, e16

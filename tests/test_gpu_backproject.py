"""GPU parity of the FDK and voxel-based backprojectors (rtkb_fdk_backproject,
rtkb_voxel_backproject through the C ABI) against the FP64 oracle, which
restates include/rtkFDKBackProjectionImageFilter.hxx and
include/rtkBackProjectionImageFilter.hxx.  Tolerance: relative L2 < 1e-5."""
import numpy as np
import pytest

from tests.gpu_util import REL_L2_TOL, pair_geometry, pair_image, rel_l2, to_gpu, to_np

pytestmark = pytest.mark.gpu


def _circular(n, sid, sdd, arc=360.0, **kw):
    keys = ("pox", "poy", "oop", "ip", "sox", "soy")
    extra = [kw.get(k, 0.0) for k in keys]
    return [(sid, sdd, i * arc / n, *extra) for i in range(n)]


def _run(rtkb, oracle, params, vsize, vspacing, psize, pspacing, fdk=True, vindex=(0, 0, 0), pindex=(0, 0, 0),
         vorigin=None, porigin=None, direction=None, seed=0, vol_init=False, inplace=False):
    gl, go = pair_geometry(rtkb, oracle, params)
    vd, vo = pair_image(rtkb, oracle, vsize, vspacing, vorigin, vindex, direction)
    pd, po = pair_image(rtkb, oracle, psize, pspacing, porigin, pindex)
    rng = np.random.default_rng(seed)
    p = rng.uniform(-1.0, 1.0, size=oracle.shape_of(po))
    v0 = rng.uniform(-1.0, 1.0, size=oracle.shape_of(vo)) if vol_init else np.zeros(oracle.shape_of(vo))
    p = p.astype(np.float32).astype(np.float64)
    v0 = v0.astype(np.float32).astype(np.float64)
    ref = oracle.backproject(go, vo, po, p, v0, fdk=fdk)
    dp, dv = to_gpu(p), to_gpu(v0)
    fn = rtkb.ops.fdk_backproject if fdk else rtkb.ops.voxel_backproject
    out = fn(gl, vd, pd, dp, dv, out=dv if inplace else None)
    assert rtkb.ops.device_status() == 0
    return rel_l2(to_np(out), ref), ref


def test_fdk_bp_c1_geometry(rtkb, oracle):
    err, ref = _run(rtkb, oracle, _circular(180, 1000.0, 1500.0), (128, 128, 128), (1.6,) * 3, (256, 256, 180),
                    (1.0, 1.0, 1.0))
    assert np.abs(ref).max() > 0
    assert err < REL_L2_TOL, err


def test_voxel_bp_c1_geometry(rtkb, oracle):
    err, _ = _run(rtkb, oracle, _circular(90, 1000.0, 1500.0), (96, 80, 72), (2.0,) * 3, (256, 200, 90),
                  (1.0, 1.0, 1.0), fdk=False)
    assert err < REL_L2_TOL, err


def test_fdk_bp_displaced_offsets_and_indices(rtkb, oracle):
    """Displaced detector stack (negative u index after padding), source and
    projection offsets, volume index offsets and ragged tile sizes."""
    params = _circular(64, 1000.0, 1536.0, pox=40.0, poy=-3.0, sox=2.0, soy=1.5)
    err, _ = _run(rtkb, oracle, params, (61, 37, 45), (3.0, 2.5, 3.5), (512, 120, 64), (1.0, 1.2, 1.0),
                  vindex=(5, -7, 3), pindex=(-256, 4, 0), porigin=(-100.0, -80.0, 0.0), vol_init=True)
    assert err < REL_L2_TOL, err


def test_fdk_bp_parker_short_scan_arc(rtkb, oracle):
    err, _ = _run(rtkb, oracle, _circular(100, 1000.0, 1536.0, arc=200.0), (64, 64, 64), (2.0,) * 3,
                  (200, 160, 100), (1.2, 1.2, 1.0))
    assert err < REL_L2_TOL, err


def test_fdk_bp_generic_path_out_of_plane(rtkb, oracle):
    """A tilted detector takes RTK's generic interpolator path (mode 0)."""
    params = [(1000.0, 1500.0, i * 9.0, 3.0, -2.0, 10.0, 5.0, 0.0, 0.0) for i in range(40)]
    err, _ = _run(rtkb, oracle, params, (48, 40, 44), (2.5,) * 3, (160, 150, 40), (1.0, 1.0, 1.0))
    assert err < REL_L2_TOL, err


def test_fdk_bp_rotated_volume_direction(rtkb, oracle):
    c, s = np.cos(np.pi / 4), np.sin(np.pi / 4)
    direction = np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]])
    err, _ = _run(rtkb, oracle, _circular(36, 800.0, 1200.0), (40, 40, 40), (2.0,) * 3, (128, 128, 36),
                  (1.0, 1.0, 1.0), direction=direction)
    assert err < REL_L2_TOL, err


def test_fdk_bp_in_place(rtkb, oracle):
    err, _ = _run(rtkb, oracle, _circular(45, 1000.0, 1500.0), (50, 34, 50), (2.0,) * 3, (160, 120, 45),
                  (1.0, 1.0, 1.0), vol_init=True, inplace=True)
    assert err < REL_L2_TOL, err


def test_fdk_bp_unaligned_rows_without_tma(rtkb, oracle):
    """Rows of 254 floats are not 16-byte multiples: the footprint is staged
    with plain loads instead of TMA."""
    err, _ = _run(rtkb, oracle, _circular(60, 1000.0, 1500.0), (64, 48, 64), (2.0,) * 3, (254, 203, 60),
                  (1.0, 1.0, 1.0))
    assert err < REL_L2_TOL, err


def test_fdk_bp_large_magnification_slow_tiles(rtkb, oracle):
    """Source close to the volume: corner tiles overflow the footprint box and
    take the FP64 per-projection fallback."""
    err, _ = _run(rtkb, oracle, _circular(40, 300.0, 600.0), (96, 64, 96), (2.0,) * 3, (512, 384, 40),
                  (1.0, 1.0, 1.0))
    assert err < REL_L2_TOL, err


def test_fdk_bp_parallel_geometry(rtkb, oracle):
    err, _ = _run(rtkb, oracle, _circular(60, 1000.0, 0.0, arc=180.0), (48, 32, 48), (2.0,) * 3, (128, 80, 60),
                  (1.0, 1.0, 1.0))
    assert err < REL_L2_TOL, err


def test_fdk_bp_single_voxel_and_empty_stack(rtkb, oracle):
    err, _ = _run(rtkb, oracle, _circular(8, 1000.0, 1500.0), (1, 1, 1), (1.0,) * 3, (16, 16, 8), (1.0, 1.0, 1.0),
                  vol_init=True)
    assert err < REL_L2_TOL, err


def test_fdk_bp_full_size_c2_region_and_linearity(rtkb, oracle):
    """512^3 from 720 projections of 1024x768 (the benchmark configuration):
    a y-slab of the GPU volume against the oracle computing only that region
    (region index semantics), and linearity of the full-size operator."""
    import torch

    n = 720
    params = _circular(n, 1000.0, 1536.0)
    gl, go = pair_geometry(rtkb, oracle, params)
    vd = rtkb.make_desc((512, 512, 512), (0.5,) * 3)
    pd, po = pair_image(rtkb, oracle, (1024, 768, n), (0.388, 0.388, 1.0))
    gen = torch.Generator(device="cuda").manual_seed(11)
    p1 = torch.rand((n, 768, 1024), device="cuda", generator=gen) * 2 - 1
    zero = torch.zeros((512, 512, 512), device="cuda")
    v1 = rtkb.ops.fdk_backproject(gl, vd, pd, p1, zero)
    # region y in [250, 254): same origin, index offset selects the slab
    full_origin = tuple(vd.origin)
    vo_region = oracle.image((512, 4, 512), (0.5,) * 3, origin=full_origin, index=(0, 250, 0))
    ref = oracle.backproject(go, vo_region, po, p1.cpu().numpy().astype(np.float64), fdk=True)
    got = v1[:, 250:254, :].cpu().numpy()
    assert rel_l2(got, ref) < REL_L2_TOL
    # linearity: BP(a p1 + b p2) = a BP(p1) + b BP(p2)
    p2 = torch.rand((n, 768, 1024), device="cuda", generator=gen)
    v2 = rtkb.ops.fdk_backproject(gl, vd, pd, p2, zero)
    v12 = rtkb.ops.fdk_backproject(gl, vd, pd, 0.5 * p1 + 2.0 * p2, zero)
    lin = torch.linalg.vector_norm(v12 - (0.5 * v1 + 2.0 * v2)) / torch.linalg.vector_norm(v12)
    assert lin.item() < 1e-5
    assert rtkb.ops.device_status() == 0


@pytest.mark.parametrize("chunk,vol_init,nz", [(0, False, 44), (7, True, 44), (1000, True, 100), (1, False, 44),
                                               (0, True, 137)])
def test_fdk_bp_host_buffers_streamed_in_chunks(rtkb, oracle, chunk, vol_init, nz):
    """rtkb_fdk_backproject_host: host stack and volume, the stack streamed in
    chunks (ragged last chunk with 7, one chunk with 1000, one projection per
    chunk with 1), projection indices offset as in a subset of a longer scan;
    the last subset's slabs of halving size over 3, 7 and 9 tile layers."""
    import torch

    params = _circular(50, 1000.0, 1536.0, pox=12.0)
    gl, go = pair_geometry(rtkb, oracle, params)
    vd, vo = pair_image(rtkb, oracle, (40, 36, nz), (2.5,) * 3, index=(2, -3, 1))
    pd, po = pair_image(rtkb, oracle, (160, 120, 45), (1.0,) * 3, index=(-80, 0, 3))
    rng = np.random.default_rng(11 + chunk)
    p = rng.uniform(-1.0, 1.0, size=oracle.shape_of(po)).astype(np.float32).astype(np.float64)
    v0 = (rng.uniform(-1.0, 1.0, size=oracle.shape_of(vo)) if vol_init else np.zeros(oracle.shape_of(vo)))
    v0 = v0.astype(np.float32).astype(np.float64)
    ref = oracle.backproject(go, vo, po, p, v0, fdk=True)
    hp = torch.from_numpy(p.astype(np.float32)).pin_memory()
    hv = torch.from_numpy(v0.astype(np.float32)).pin_memory() if vol_init else None
    out = rtkb.ops.fdk_backproject_host(gl, vd, pd, hp, hv, chunk=chunk)
    torch.cuda.synchronize()
    assert rtkb.ops.device_status() == 0
    got = out.numpy().astype(np.float64)
    dev = to_np(rtkb.ops.fdk_backproject(gl, vd, pd, to_gpu(p), to_gpu(v0)))
    assert rel_l2(got, ref) < REL_L2_TOL, rel_l2(got, ref)
    # chunking only regroups the FP32 sums per voxel: the running volume is
    # rounded to FP32 once per chunk (45 times with chunk=1, ~1.7e-6)
    assert rel_l2(got, dev) < 5e-6, rel_l2(got, dev)


def test_fdk_bp_host_rejects_device_tensors(rtkb, oracle):
    import torch

    gl, go = pair_geometry(rtkb, oracle, _circular(4, 1000.0, 1500.0))
    vd, vo = pair_image(rtkb, oracle, (8, 8, 8), (1.0,) * 3)
    pd, po = pair_image(rtkb, oracle, (16, 16, 4), (1.0,) * 3)
    with pytest.raises(TypeError):
        rtkb.ops.fdk_backproject_host(gl, vd, pd, torch.zeros((4, 16, 16), device="cuda"))


@pytest.mark.parametrize("fdk", [True, False])
def test_bp_projection_sweep_schedule(rtkb, oracle, fdk):
    """Tile schedule 1 (the projection sweep: tiles start at the projection the
    resident CTAs have reached and wrap around the stack) sums the same terms
    in another order: within FP32 rounding of schedule 0, and both within the
    oracle's tolerance.  Schedule 0 is identical from run to run."""
    import torch

    params = _circular(240, 1000.0, 1536.0, pox=7.0, sox=3.0)
    gl, go = pair_geometry(rtkb, oracle, params)
    vd, vo = pair_image(rtkb, oracle, (160, 144, 128), (1.0,) * 3, index=(2, -3, 1))
    pd, po = pair_image(rtkb, oracle, (256, 192, 240), (1.2, 1.2, 1.0))
    p = np.random.default_rng(3).uniform(-1.0, 1.0, size=oracle.shape_of(po)).astype(np.float32)
    dp = torch.from_numpy(p).cuda()
    zero = torch.zeros(oracle.shape_of(vo), device="cuda")
    fn = rtkb.ops.fdk_backproject if fdk else rtkb.ops.voxel_backproject
    outs = {}
    try:
        for sched in (0, 1, 0):
            rtkb.ops.backproject_schedule(sched, 2)
            outs.setdefault(sched, []).append(to_np(fn(gl, vd, pd, dp, zero)))
    finally:
        rtkb.ops.backproject_schedule(0)
    assert rtkb.ops.device_status() == 0
    a, b = outs[0]
    assert np.array_equal(a, b)
    assert rel_l2(outs[1][0], a) < 1e-6
    ref = oracle.backproject(go, vo, po, p.astype(np.float64), fdk=fdk)
    assert rel_l2(outs[1][0], ref) < REL_L2_TOL
    with pytest.raises(rtkb.RtkbError):
        rtkb.ops.backproject_schedule(2)

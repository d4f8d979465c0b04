"""Batched backprojection of uneven problems in one persistent launch
(rtkb_fdk_backproject_batch, rtkb_voxel_backproject_batch) and the
configuration autotuner (rtkb_backproject_autotune): every problem of the
batch against the FP64 oracle (include/rtkFDKBackProjectionImageFilter.hxx
restated), relative L2 < 1e-5, whatever configuration runs the batch."""
import numpy as np
import pytest

from tests.gpu_util import REL_L2_TOL, pair_geometry, pair_image, rel_l2, to_gpu, to_np

pytestmark = pytest.mark.gpu


def _problems(rtkb, oracle, n=7, seed=11):
    """Seeded uneven problems: volumes 24-72 voxels per side, 20-60
    projections, detectors 64-200 pixels, SID 800-1200 mm; one with a tilted
    detector (RTK's generic path), one with a detector width that TMA cannot
    describe (plain loads), one with index offsets and a non-zero input."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        sid = float(rng.uniform(800, 1200))
        sdd = sid * float(rng.uniform(1.3, 1.6))
        npj = int(rng.integers(20, 61))
        oop = 8.0 if k == 2 else 0.0
        params = [(sid, sdd, i * 360.0 / npj, float(rng.uniform(-5, 5)), 0.0, oop) for i in range(npj)]
        vsize = tuple(int(v) for v in rng.integers(24, 73, size=3))
        vsp = float(rng.uniform(1.5, 3.0))
        nu = 130 if k == 3 else int(rng.integers(16, 51)) * 4
        nv = int(rng.integers(64, 201))
        gl, go = pair_geometry(rtkb, oracle, params)
        vindex = (3, -2, 1) if k == 4 else (0, 0, 0)
        vd, vo = pair_image(rtkb, oracle, vsize, (vsp,) * 3, index=vindex)
        pd, po = pair_image(rtkb, oracle, (nu, nv, npj), (1.2, 1.2, 1.0))
        p = rng.uniform(-1, 1, size=oracle.shape_of(po)).astype(np.float32).astype(np.float64)
        v0 = (rng.uniform(-1, 1, size=oracle.shape_of(vo)) if k == 4 else np.zeros(oracle.shape_of(vo)))
        v0 = v0.astype(np.float32).astype(np.float64)
        out.append((gl, go, vd, vo, pd, po, p, v0))
    return out


@pytest.mark.parametrize("fdk", [True, False])
def test_batch_matches_oracle_per_problem(rtkb, oracle, fdk):
    probs = _problems(rtkb, oracle)
    refs = [oracle.backproject(go, vo, po, p, v0, fdk=fdk) for (gl, go, vd, vo, pd, po, p, v0) in probs]
    for config in (-1, 2):
        args, outs = [], []
        for (gl, go, vd, vo, pd, po, p, v0) in probs:
            out = to_gpu(np.zeros(oracle.shape_of(vo)))
            args.append((gl, vd, pd, to_gpu(p), to_gpu(v0), out))
            outs.append(out)
        used = rtkb.ops.backproject_batch(args, fdk=fdk, config=config)
        assert 0 <= used < 6
        assert rtkb.ops.device_status() == 0
        for k, (out, ref) in enumerate(zip(outs, refs)):
            assert rel_l2(to_np(out), ref) < REL_L2_TOL, (config, k, rel_l2(to_np(out), ref))


def test_autotune_picks_a_configuration_and_results_are_unchanged(rtkb, oracle):
    probs = _problems(rtkb, oracle, n=5, seed=3)
    args, outs = [], []
    for (gl, go, vd, vo, pd, po, p, v0) in probs:
        out = to_gpu(np.zeros(oracle.shape_of(vo)))
        args.append((gl, vd, pd, to_gpu(p), to_gpu(v0), out))
        outs.append(out)
    best, best_ms, times = rtkb.ops.backproject_autotune(args, repeats=1)
    assert len(times) == 6 and 0 <= best < 6 and best_ms == min(times) and best_ms > 0
    rtkb.ops.backproject_batch(args, config=best)
    for (gl, go, vd, vo, pd, po, p, v0), out in zip(probs, outs):
        ref = oracle.backproject(go, vo, po, p, v0)
        assert rel_l2(to_np(out), ref) < REL_L2_TOL


def test_autotune_rejects_in_place_outputs(rtkb, oracle):
    (gl, go, vd, vo, pd, po, p, v0), = _problems(rtkb, oracle, n=1, seed=5)
    v = to_gpu(v0)
    with pytest.raises(rtkb.RtkbError):
        rtkb.ops.backproject_autotune([(gl, vd, pd, to_gpu(p), v, v)])


def test_prepared_batch_repeats_the_one_shot_result(rtkb, oracle):
    """A prepared batch executed twice writes the same volumes as the one-shot
    call (out = in + backprojection, so repeated executes do not accumulate)."""
    probs = _problems(rtkb, oracle, n=4, seed=9)
    args, outs = [], []
    for (gl, go, vd, vo, pd, po, p, v0) in probs:
        out = to_gpu(np.zeros(oracle.shape_of(vo)))
        args.append((gl, vd, pd, to_gpu(p), to_gpu(v0), out))
        outs.append(out)
    b = rtkb.ops.BackprojectionBatch(args)
    b.execute()
    b.execute()
    first = [to_np(o) for o in outs]
    b.close()
    rtkb.ops.backproject_batch(args, config=b.config)
    for f, o in zip(first, outs):
        assert rel_l2(f, to_np(o)) < 1e-6


def test_single_problem_autotune_and_forced_configuration(rtkb, oracle):
    """n == 1: the autotuner times the single-problem path; forcing its choice
    keeps the results at the oracle's."""
    (gl, go, vd, vo, pd, po, p, v0), = _problems(rtkb, oracle, n=1, seed=21)
    out = to_gpu(np.zeros(oracle.shape_of(vo)))
    best, best_ms, times = rtkb.ops.backproject_autotune([(gl, vd, pd, to_gpu(p), to_gpu(v0), out)], repeats=1)
    assert len(times) == 6 and 0 <= best < 6
    try:
        rtkb.ops.backproject_config(best)
        got = to_np(rtkb.ops.fdk_backproject(gl, vd, pd, to_gpu(p), to_gpu(v0)))
        last, count = rtkb.ops.backproject_config(-1)
    finally:
        rtkb.ops.backproject_config(-1)
    assert count == 6 and last in (best, -1)
    assert rel_l2(got, oracle.backproject(go, vo, po, p, v0)) < REL_L2_TOL


def test_autotune_cache_hit_returns_the_stored_result(rtkb, oracle, tmp_path):
    """With a cache file, the first call times the configurations and stores
    the result under (kernel, device, problem sizes); the second call returns
    it without timing (identical per-configuration times), another kernel
    choice misses."""
    probs = _problems(rtkb, oracle, n=3, seed=8)
    args = [(gl, vd, pd, to_gpu(p), to_gpu(v0), to_gpu(np.zeros(oracle.shape_of(vo))))
            for (gl, go, vd, vo, pd, po, p, v0) in probs]
    path = str(tmp_path / "autotune.json")
    first = rtkb.ops.backproject_autotune(args, repeats=1, cache=path)
    second = rtkb.ops.backproject_autotune(args, repeats=1, cache=path)
    assert second == first
    other = rtkb.ops.backproject_autotune(args, fdk=False, repeats=1, cache=path)
    assert len(other[2]) == 6
    import json

    with open(path) as f:
        assert len(json.load(f)) == 2

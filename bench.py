"""Benchmark: FDK backprojection throughput (GUPS) on one B200.

Workload (the projector-pair throughput configuration): a 512^3 float32 volume
at 0.5 mm from 720 projections over 360 deg of 1024x768 float32 pixels at
0.388 mm, SID 1000 mm, SDD 1536 mm.  One step = one FDK backprojection of the
whole stack into the volume (9.66e10 voxel-projection updates).  The metric is
giga voxel-projection updates per second (GUPS).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Multi-GPU: replicas only (each rank backprojects its own stack; there is no
data-path collective), value = all ranks' updates / max-over-ranks time.
The reference arm times RTK's CPU FDK backprojector (the oracle's restatement
with RTK's data types and loop order, oracle/rtk_oracle.c) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "backproj GUPS (FDK voxel-projection updates/s, 1e9)"
UNIT = "GUPS"
NX = NY = NZ = 512
VOX = 0.5
NU, NV, NP = 1024, 768, 720
PIX = 0.388
SID, SDD = 1000.0, 1536.0
SEED = 20261203 + 1
L1_BYTES_PER_UPDATE = 16  # four 4-byte taps of one bilinear interpolation
# DRAM bytes (read + write) of one backprojection launch of this workload under each tile schedule,
# recorded from a 1-pass ncu capture (dram__bytes_read.sum + dram__bytes_write.sum) of the kernel as of
# BP_TRAFFIC_COMMIT; recorded figures, not measurements of the build that runs.
BP_DRAM_BYTES_BY_SCHEDULE = {0: 70.3237e9 + 0.5960e9, 1: 13.6485e9 + 0.5856e9}
BP_TRAFFIC_COMMIT = "e17605a"
WORKLOAD = {"workload": "FDK backprojection 512^3 @0.5mm <- 720 x 1024x768 @0.388mm, SID 1000, SDD 1536, 360 deg",
            "volume": [NX, NY, NZ], "projections": [NU, NV, NP], "dtype_storage": "float32",
            "l2_policy": "inputs larger than L2 (2.26 GB projection stack, 0.54 GB volume)"}


def updates_per_step() -> float:
    return float(NX) * NY * NZ * NP


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return json.load(f)
    except Exception:
        return {}


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.out.close()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    mhz.append(float(parts[1]))
                    mx = float(parts[2])
                except ValueError:
                    continue
                for name, val in zip(names, parts[5:9]):
                    if val.lower() == "active":
                        reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx, "samples": len(mhz),
                "reasons": sorted(reasons)}


def dist_setup(n_gpus: int):
    """One process per GPU (NCCL); without a GPU (the CPU tests of the
    multi-process path) the same plumbing runs over gloo."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def make_geometry():
    import rtk_b200 as rtkb

    return rtkb.geometry.circular(NP, SID, SDD)


def make_projections(torch, g, gen):
    """Seeded synthetic projections with the workload's shape: analytic line
    integrals (on the GPU, rtkb_project_ellipsoids) of 20 random ellipsoids with
    semi-axes 5-80 mm, centres in a 200 mm sphere, random rotations and
    densities 0.1-1 (no public dataset is named for this configuration)."""
    import rtk_b200 as rtkb
    from tests import phantoms

    pd = rtkb.make_desc((NU, NV, NP), (PIX, PIX, 1.0))
    ell = phantoms.random_ellipsoids(20, SEED)
    p = rtkb.ops.project_ellipsoids(g, pd, ell)
    return pd, p, "analytic line integrals of 20 seeded random ellipsoids (semi-axes 5-80 mm)"


def fdk_pipeline_ms(torch, rtkb, g, vd, pd, proj, stream, reps=3):
    """Whole FDK (fused weighting + Hann ramp filter, then backprojection) on the
    benchmark stack, device time per reconstruction."""
    zero = torch.zeros(tuple(reversed(list(vd.size))), device="cuda")
    ramp = rtkb.ops.ramp_params(hann=1.0)

    def run():
        f, fd = rtkb.ops.fdk_preprocess(g, pd, proj, ramp, stream=stream)
        rtkb.ops.fdk_backproject(g, vd, fd, f, zero, out=zero, stream=stream)

    run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        run()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def ramp_leg(torch, rtkb, g, pd, proj, reps=5) -> dict:
    """The projection filter of the headline's stack (720 x 768 rows of 1024,
    zero-padded to 2048): FDK weighting + Hann ramp filter in one kernel, and
    the ramp filter alone.  Device time (median of `reps`, current stream), the
    HBM roofline (the stack read once and written once) and the transforms'
    arithmetic (per row pair one forward and one inverse complex FFT of the
    padded length, 5 N log2 N flops each)."""
    import math

    rp = rtkb.ops.ramp_params(hann=1.0)
    out = torch.empty_like(proj)
    ms_pre, _ = _event_median_ms(torch, lambda: rtkb.ops.fdk_preprocess(g, pd, proj, rp, out=out), reps)
    ms_ramp, _ = _event_median_ms(torch, lambda: rtkb.ops.ramp_filter(pd, proj, rp, out=out), reps)
    n_pad = rtkb.ops.ramp_kernel(NU, PIX, rp)[0]
    pairs = (NP * NV + 1) // 2
    algo_bytes = 2 * proj.numel() * 4
    flops = pairs * 2 * 5 * n_pad * math.log2(n_pad)
    hbm = peaks().get("hbm_gbs")
    gbs = algo_bytes / (ms_ramp * 1e-3) / 1e9
    return {"workload": f"720 x 768 rows of {NU} columns, padded to {n_pad}; Hann ramp (cut 1.0)",
            "weights_and_ramp_ms": ms_pre, "ramp_ms": ms_ramp,
            "roofline": {"bound": "hbm", "algorithmic_bytes": algo_bytes, "achieved_gbs": gbs, "peak_gbs": hbm,
                         "frac": gbs / hbm if hbm else None,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"},
            "fft_gflops": flops / (ms_ramp * 1e-3) / 1e9}


def draw_ellipsoids(torch, vd, ell):
    """Voxelised ellipsoids (rtk::DrawEllipsoidImageFilter semantics: a voxel
    whose centre lies inside adds the density) on a volume description with
    identity direction: synthetic input of the forward-projection leg."""
    nx, ny, nz = vd.size
    ax = [vd.origin[a] + vd.spacing[a] * torch.arange(vd.size[a], device="cuda", dtype=torch.float64) for a in range(3)]
    out = torch.zeros((nz, ny, nx), device="cuda", dtype=torch.float32)
    for e in ell:
        c, semi, R, dens = e[0:3], e[3:6], e[6:15].reshape(3, 3), e[15]
        acc = 0.0
        for k in range(3):  # local coordinate k = (R^T (p - c))_k / semi_k
            col = R[:, k]
            lk = ((ax[0] - c[0])[None, None, :] * col[0] + (ax[1] - c[1])[None, :, None] * col[1] +
                  (ax[2] - c[2])[:, None, None] * col[2]) / semi[k]
            acc = acc + lk * lk
        out += float(dens) * (acc <= 1.0).float()
    return out


def joseph_forward_leg(torch, rtkb, lib, stream, reps=2):
    """Joseph forward projection of the projector-pair configuration: a 512^3
    volume at 0.5 mm holding the 20 seeded random ellipsoids, projected onto
    720 x 1024x768 at 0.388 mm.  Ray samples per second (device time, inputs
    resident) with the L1 roofline: one bilinear sample gathers 4 taps x 4 B."""
    from tests import phantoms

    g = make_geometry()
    vd = rtkb.make_desc((NX, NY, NZ), (VOX, VOX, VOX))
    pd = rtkb.make_desc((NU, NV, NP), (PIX, PIX, 1.0))
    vol = draw_ellipsoids(torch, vd, phantoms.random_ellipsoids(20, SEED))
    zero = torch.zeros((NP, NV, NU), device="cuda")
    out = torch.empty_like(zero)
    n = rtkb.ops.joseph_sample_count(g, vd, pd, stream=stream)
    rtkb.ops.joseph_forward_project(g, vd, pd, vol, zero, out=out, stream=stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        rtkb.ops.joseph_forward_project(g, vd, pd, vol, zero, out=out, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / reps
    peak = smem_peak_gbs(torch, lib, stream)
    achieved = n * 16 / t / 1e9
    out_leg = {"workload": "Joseph forward projection 512^3 @0.5mm -> 720 x 1024x768 @0.388mm, 20 random ellipsoids",
               "samples_per_launch": n, "ms_per_launch": t * 1e3, "gsamples_per_s": n / t / 1e9,
               "roofline": {"bound": "l1", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": achieved / peak, "bytes_per_sample": 16,
                            "peak_source": "shared-memory bilinear-gather probe (the taps are L1-cached global loads)"}}
    out_leg["rtk_cuda_reference"] = rtk_cuda_forward_leg(torch, vol, out, t * 1e3)
    return out_leg


def joseph_back_leg(torch, rtkb, lib, stream, reps=3):
    """Joseph back projection of the CG configuration (360 x 512x384 @0.8 mm
    -> 256^3 @1 mm, seeded uniform projections), device time, samples per
    second and the L1-gather roofline (one bilinear splat moves 4 taps x 4 B;
    the kernel is bound by its atomic reductions instead), beside RTK's own
    CUDA ray-cast back projector (kernel_ray_cast_back_project, built
    unchanged, 16-projection slabs; steps of the smallest spacing, trilinear
    atomic splats) on the same projections, with the two outputs' relative L2
    distance (different discretisations of the same adjoint)."""
    from oracle import oracle as O
    from oracle import rtk_cuda
    from tests import workloads as W

    c = W.C3
    n = c["n"]
    g = rtkb.geometry.circular(n, c["sid"], c["sdd"])
    vd = rtkb.make_desc(c["vol"], (c["vox"],) * 3)
    pd = rtkb.make_desc((*c["det"], n), (c["pix"], c["pix"], 1.0))
    gen = torch.Generator(device="cuda").manual_seed(SEED + 5)
    p = torch.rand((n, c["det"][1], c["det"][0]), device="cuda", generator=gen)
    vin = torch.zeros(tuple(reversed(c["vol"])), device="cuda")
    vout = torch.empty_like(vin)
    samples = rtkb.ops.joseph_sample_count(g, vd, pd, stream=stream)
    ms, _ = _event_median_ms(torch, lambda: rtkb.ops.joseph_back_project(g, vd, pd, p, vin, out=vout), reps)
    peak = smem_peak_gbs(torch, lib, stream)
    achieved = samples * 16 / (ms * 1e-3) / 1e9
    leg = {"workload": "Joseph back projection 360 x 512x384 @0.8mm -> 256^3 @1mm, seeded uniform projections",
           "samples_per_launch": samples, "ms_per_launch": ms, "gsamples_per_s": samples / (ms * 1e-3) / 1e9,
           "roofline": {"bound": "l1", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "bytes_per_sample": 16,
                        "peak_source": "shared-memory bilinear-gather probe (the bound is the atomic reductions)"}}
    if not rtk_cuda.iter_available():
        leg["rtk_cuda_reference"] = {"unavailable": "RTK's CUDA projectors were not built"}
        return leg
    prod = vout.clone()
    go = O.Geometry()
    for i in range(n):
        go.add_projection(c["sid"], c["sdd"], i * 360.0 / n)
    vo = O.image(c["vol"], (c["vox"],) * 3)
    po = O.image((*c["det"], n), (c["pix"], c["pix"], 1.0))

    def run_rtk():
        rtk_cuda.ray_cast_back_project(O, go, vo, po, vin.data_ptr(), vout.data_ptr(), p.data_ptr())

    ms_rtk, _ = _event_median_ms(torch, run_rtk, reps)
    leg["rtk_cuda_reference"] = {
        "ms_per_back_projection": ms_rtk, "product_speedup": ms_rtk / ms,
        "rel_l2_to_product": float((vout - prod).double().norm() / prod.double().norm()),
        "kernel": "RTK kernel_ray_cast_back_project, SLAB_SIZE 16, trilinear atomic splats every smallest spacing"}
    return leg


def _event_median_ms(torch, run, reps):
    """Median device time of run() over reps calls (one warm-up call first);
    run() may issue work on the legacy default stream, so each call is
    bracketed by events on the current stream and a synchronise."""
    torch.cuda.synchronize()
    run()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    times = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run()
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    return statistics.median(times), times


def rtk_cuda_forward_leg(torch, vol, product_out, product_ms, reps=3) -> dict:
    """RTK's own CUDA forward projector (kernel_forwardProject of
    src/rtkCudaForwardProjectionImageFilter.cu, compiled unchanged into
    oracle/_ref) on the same volume and geometry, driven in 16-projection slabs
    as CudaForwardProjectionImageFilter runs it (each slab copies the volume
    into a 3-D texture array; trilinear samples every 0.5 mm along the ray).
    A different quadrature of the same line integrals than Joseph's: its
    relative L2 distance to the product's projections is reported, not a
    parity figure.  The reference's GPU code, timed beside the product."""
    from oracle import oracle as O
    from oracle import rtk_cuda

    if not rtk_cuda.iter_available():
        return {"unavailable": "RTK's CUDA projectors were not built (no RTK source tree where the library was built)"}
    go = oracle_geometry()
    vo = O.image((NX, NY, NZ), (VOX,) * 3)
    po = O.image((NU, NV, NP), (PIX, PIX, 1.0))
    zero = torch.zeros((NP, NV, NU), device="cuda")
    res = torch.empty_like(zero)

    def run():
        rtk_cuda.forward_project(O, go, vo, po, vol.data_ptr(), zero.data_ptr(), res.data_ptr())

    ms, times = _event_median_ms(torch, run, reps)
    d = (res - product_out).double().norm() / product_out.double().norm()
    # every slab allocates, fills and frees a 512^3 texture array, whose cost varies with the device's
    # allocation state: the fastest run is reported beside the median
    return {"ms_per_projection": ms, "ms_min": min(times), "ms_each": [round(x, 1) for x in times],
            "product_speedup": ms / product_ms, "product_speedup_vs_fastest": min(times) / product_ms,
            "rel_l2_to_product_joseph": float(d),
            "kernel": "RTK kernel_forwardProject, SLAB_SIZE 16, 3-D texture trilinear samples every 0.5 mm"}


def sweep_leg(torch, rtkb, g, vd, pd, proj, vol_ref, stream, schedule_timed, reps=5) -> dict:
    """The headline backprojection under the other tile schedule: the
    projection sweep (schedule 1: tiles start where the resident CTAs are in
    the stack and wrap around, so the tiles in flight share projections in L2)
    against every tile from projection 0 (schedule 0).  Median device time of
    `reps` steps, its relative L2 distance to the timed output (summation
    order only), and the DRAM bytes of one launch recorded from a 1-pass ncu
    capture of each schedule."""
    other = 1 - schedule_timed
    zero = torch.zeros((NZ, NY, NX), device="cuda")
    out = torch.empty_like(zero)
    rtkb.ops.backproject_schedule(other)
    try:
        ms, times = _event_median_ms(
            torch, lambda: rtkb.ops.fdk_backproject(g, vd, pd, proj, zero, out=out, stream=stream), reps)
    finally:
        rtkb.ops.backproject_schedule(schedule_timed)
    d = float((out - vol_ref).double().norm() / vol_ref.double().norm())
    return {"schedule": other, "ms_per_backprojection": ms, "gups": updates_per_step() / ms / 1e6,
            "rel_l2_to_timed_output": d, "dram_bytes_per_launch_recorded": BP_DRAM_BYTES_BY_SCHEDULE[other],
            "dram_bytes_commit": BP_TRAFFIC_COMMIT}


def voxel_bp_leg(torch, rtkb, g, vd, pd, proj, stream, reps=3) -> dict:
    """Voxel-based back projection (rtk::BackProjectionImageFilter, RTK's
    default back projector of its iterative filters) of the headline's stack
    into the 512^3 volume: the product's kernel against RTK's own CUDA back
    projector (kernel_backProject of src/rtkCudaBackProjectionImageFilter.cu,
    compiled unchanged, 16-projection layered-texture slabs), device time with
    inputs resident, and the two outputs' relative L2 distance."""
    from oracle import oracle as O
    from oracle import rtk_cuda

    zero = torch.zeros((NZ, NY, NX), device="cuda")
    out = torch.empty_like(zero)

    def run_product():
        rtkb.ops.voxel_backproject(g, vd, pd, proj, zero, out=out, stream=stream)

    ms, times = _event_median_ms(torch, run_product, reps)
    leg = {"workload": "voxel-based back projection 720 x 1024x768 @0.388mm -> 512^3 @0.5mm",
           "updates": updates_per_step(), "ms_per_backprojection": ms, "gups": updates_per_step() / ms / 1e6}
    if not rtk_cuda.iter_available():
        leg["rtk_cuda_reference"] = {"unavailable": "RTK's CUDA back projector was not built"}
        return leg
    go = oracle_geometry()
    vo = O.image((NX, NY, NZ), (VOX,) * 3)
    po = O.image((NU, NV, NP), (PIX, PIX, 1.0))
    res = torch.empty_like(zero)

    def run_rtk():
        rtk_cuda.back_project(O, go, vo, po, zero.data_ptr(), res.data_ptr(), proj.data_ptr())

    rms, rtimes = _event_median_ms(torch, run_rtk, reps)
    d = (res - out).double().norm() / out.double().norm()
    leg["rtk_cuda_reference"] = {"ms_per_backprojection": rms, "ms_each": [round(x, 1) for x in rtimes],
                                 "gups": updates_per_step() / rms / 1e6, "product_speedup": rms / ms,
                                 "rel_l2_to_product": float(d),
                                 "kernel": "RTK kernel_backProject, SLAB_SIZE 16, layered-texture bilinear"}
    return leg


def bf16_storage_leg(torch, rtkb, g, vd, pd, proj, vol_fp32, stream, peak_smem, reps=5):
    """BF16 storage variant of the headline backprojection: the same stack
    converted once (outside the timed region) to bfloat16, backprojected with
    FP32 interpolation and accumulation.  GUPS, the roofline at 8 B per update
    (four 2-byte taps) and the change against the FP32 stack's volume."""
    pb = rtkb.ops.to_bf16(proj, stream=stream)
    zero = torch.zeros_like(vol_fp32)
    out = torch.empty_like(vol_fp32)
    for _ in range(2):
        rtkb.ops.fdk_backproject(g, vd, pd, pb, zero, out=out, stream=stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        rtkb.ops.fdk_backproject(g, vd, pd, pb, zero, out=out, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / reps
    gups = updates_per_step() / t / 1e9
    diff = float((out.double() - vol_fp32.double()).norm() / vol_fp32.double().norm())
    achieved = gups * 8.0
    return {"value": gups, "unit": UNIT, "ms_per_step": t * 1e3, "stack_bytes": pb.numel() * 2,
            "rel_l2_vs_fp32_stack": diff,
            "roofline": {"bound": "l1", "achieved": achieved, "peak": peak_smem, "unit": "GB/s",
                         "frac": achieved / peak_smem if peak_smem else None, "bytes_per_update": 8}}


def batch_leg(torch, rtkb, stream, n=64, reps=3):
    """Batched uneven reconstructions: n seeded FDK backprojection problems
    (volumes 64^3-256^3 with voxels of at most 1.5 detector pixels, 90-360
    projections, detectors 128^2-512^2, SID 800-1200 mm) in one persistent
    launch with the autotuner's configuration,
    against the same problems launched one by one.  GUPS over all problems;
    the persistent figure times prepared-batch executions (host preparation
    done once, outside the timed region)."""
    import numpy as np

    rng = np.random.default_rng(SEED + 7)
    args, updates = [], 0.0
    for _ in range(n):
        nv_ = int(rng.integers(64, 257))
        npj = int(rng.integers(90, 361))
        nu = int(rng.integers(32, 129)) * 4
        nvd = int(rng.integers(128, 513))
        sid = float(rng.uniform(800, 1200))
        sdd = 1.5 * sid
        g = rtkb.geometry.circular(npj, sid, sdd)
        # a voxel projects onto at most ~1.5 pixels (magnification 1.5, 1 mm pixels), as in the projector-pair
        # configuration; smaller volumes are shrunk further so that they fit the detector width
        vsp = min(1.0, 0.9 * nu / (nv_ * 1.5))
        vd = rtkb.make_desc((nv_, nv_, nv_), (vsp,) * 3)
        pd = rtkb.make_desc((nu, nvd, npj), (1.0, 1.0, 1.0))
        proj = torch.rand((npj, nvd, nu), device="cuda")
        zero = torch.zeros((nv_, nv_, nv_), device="cuda")
        args.append((g, vd, pd, proj, zero, torch.empty_like(zero)))
        updates += float(nv_) ** 3 * npj
    best, best_ms, times = rtkb.ops.backproject_autotune(args, repeats=1, stream=stream)
    batch = rtkb.ops.BackprojectionBatch(args, config=best)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    batch.execute(stream)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        batch.execute(stream)
    e1.record(stream)
    torch.cuda.synchronize()
    t_batch = e0.elapsed_time(e1) / reps
    batch.close()
    e0.record(stream)
    for _ in range(reps):
        for (g, vd, pd, proj, zero, out) in args:
            rtkb.ops.fdk_backproject(g, vd, pd, proj, zero, out=out, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    t_seq = e0.elapsed_time(e1) / reps
    return {"workload": f"{n} FDK backprojections, volumes 64^3-256^3, 90-360 projections, detectors 128^2-512^2, "
                        "SID 800-1200 mm (seeded)",
            "updates": updates, "persistent_ms": t_batch, "gups": updates / (t_batch / 1e3) / 1e9,
            "one_launch_per_problem_ms": t_seq,
            "one_launch_per_problem_gups": updates / (t_seq / 1e3) / 1e9, "autotuned_config": best,
            "autotune_ms_per_config": [round(t, 3) for t in times],
            "note": "FDK backprojection part of the batched configuration; its CG part is the batched_cg entry"}


def c4_leg(torch, rtkb, stream, n=64, niter=10):
    """The batched configuration end to end: n seeded problems (volumes
    64^3-256^3, 90-360 projections, detectors 128^2-512^2, SID 800-1200 mm) of
    random-ellipsoid phantoms, each reconstructed by FDK (weights + Hann ramp,
    then backprojection) followed by niter CG iterations (Joseph pair) started
    from the FDK volume.  Batched: the preprocessing of every stack in one
    launch per padded row length, every backprojection in one persistent launch (autotuned
    configuration), every problem's CG start and iterations in one CUDA graph
    launch (a branch per problem).  Against the same work problem after problem
    (the same CG plans, one after another).  Plans and the backprojection batch
    are prepared outside both timed regions.  The two smallest problems' FDK
    volumes are checked against the FP64 oracle's FDK, and their CG results
    (from that FDK volume) against the oracle's CG from the same start."""
    import numpy as np

    from rtk_b200._capi import check
    from tests import phantoms

    rng = np.random.default_rng(SEED + 8)
    probs = []
    for _ in range(n):
        nv_ = int(rng.integers(64, 257))
        npj = int(rng.integers(90, 361))
        nu = int(rng.integers(32, 129)) * 4
        nvd = int(rng.integers(128, 513))
        sid = float(rng.uniform(800, 1200))
        vsp = min(1.0, 0.9 * nu / (nv_ * 1.5))
        P = {"nv": nv_, "np": npj, "nu": nu, "nvd": nvd, "sid": sid, "vsp": vsp,
             "ell": phantoms.random_ellipsoids(8, int(rng.integers(1 << 30)), axis_range=(0.05 * nv_ * vsp, 0.25 * nv_ * vsp),
                                               centre_radius=0.2 * nv_ * vsp, density_range=(0.002, 0.02))}
        P["g"] = rtkb.geometry.circular(npj, sid, 1.5 * sid)
        P["vd"] = rtkb.make_desc((nv_,) * 3, (vsp,) * 3)
        P["pd"] = rtkb.make_desc((nu, nvd, npj), (1.0, 1.0, 1.0))
        P["p"] = rtkb.ops.project_ellipsoids(P["g"], P["pd"], P["ell"], stream=stream)
        P["f"] = torch.empty_like(P["p"])
        P["zero"] = torch.zeros((nv_,) * 3, device="cuda")
        P["x"] = torch.zeros_like(P["zero"])
        probs.append(P)
    ramp = rtkb.ops.ramp_params(hann=1.0)

    def preprocess(P):
        rtkb.ops.fdk_preprocess(P["g"], P["pd"], P["p"], ramp, stream=stream, out=P["f"])

    for P in probs:
        preprocess(P)
    bp_args = [(P["g"], P["vd"], P["pd"], P["f"], P["zero"], P["x"]) for P in probs]
    best, _, _ = rtkb.ops.backproject_autotune(bp_args, repeats=1, stream=stream)
    bpb = rtkb.ops.BackprojectionBatch(bp_args, config=best)
    # the Joseph pair's band heights from the autotuner, timed on the largest problem
    big = max(probs, key=lambda P: P["nv"] ** 3 * P["np"])
    bands = rtkb.ops.joseph_autotune(big["g"], big["vd"], big["pd"], torch.ones_like(big["zero"]), big["p"],
                                     repeats=1, stream=stream)
    cgb = rtkb.ops.ConjugateGradientBatch([(P["g"], P["vd"], P["pd"], P["p"], P["x"], None, False) for P in probs])
    lib = rtkb.load()
    plans = [lib.rtkb_cg_batch_plan(cgb._h, i) for i in range(n)]

    pre_batch = [(P["g"], P["pd"], P["p"], P["f"]) for P in probs]

    def batched():
        rtkb.ops.fdk_preprocess_batch(pre_batch, ramp, stream=stream)
        bpb.execute(stream)
        cgb.start(stream)
        cgb.iterate(niter, stream)

    def one_after_another():
        for P, plan in zip(probs, plans):
            preprocess(P)
            rtkb.ops.fdk_backproject(P["g"], P["vd"], P["pd"], P["f"], P["zero"], out=P["x"], stream=stream)
            check(lib.rtkb_cg_start(plan, rtkb.ops._ptr(P["p"]), None, 0, rtkb.ops._ptr(P["x"]), stream.cuda_stream))
            check(lib.rtkb_cg_iterate(plan, niter, stream.cuda_stream))

    batched()  # captures the CG graph
    torch.cuda.synchronize()
    times = {}
    for name, fn in (("batched", batched), ("one_after_another", one_after_another)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        times[name] = e0.elapsed_time(e1)
    assert rtkb.ops.device_status(stream) == 0
    # the FP64 oracle's FDK of the two smallest problems (the batched backprojection's volumes), then
    # its CG from that volume
    errs, cg_errs = {}, {}
    try:
        from oracle import oracle as O

        bpb.execute(stream)
        torch.cuda.synchronize()
        order = sorted(range(n), key=lambda i: probs[i]["nv"] ** 3 * probs[i]["np"])[:2]
        for i in order:
            P = probs[i]
            go = O.Geometry()
            for k in range(P["np"]):
                go.add_projection(P["sid"], 1.5 * P["sid"], k * 360.0 / P["np"])
            vo = O.image((P["nv"],) * 3, (P["vsp"],) * 3)
            po = O.image((P["nu"], P["nvd"], P["np"]), (1.0, 1.0, 1.0))
            pr = P["p"].double().cpu().numpy()
            ref = O.backproject(go, vo, po, O.ramp_filter(po, O.fdk_weight(go, po, pr), O.ramp_params(hann=1.0)),
                                fdk=True)
            got = P["x"].double().cpu().numpy()
            errs[f"problem_{i}_{P['nv']}^3_{P['np']}x{P['nu']}x{P['nvd']}"] = float(
                np.linalg.norm(got - ref) / np.linalg.norm(ref))
            # the problem's CG from its FDK volume, on the GPU (its batch plan)
            # and in the oracle (FP64 CG, Joseph pair) from the same FP32 start
            check(lib.rtkb_cg_start(plans[i], rtkb.ops._ptr(P["p"]), None, 0, rtkb.ops._ptr(P["x"]),
                                    stream.cuda_stream))
            check(lib.rtkb_cg_iterate(plans[i], niter, stream.cuda_stream))
            torch.cuda.synchronize()
            ref_cg, _ = O.cg_joseph(go, vo, po, pr, niter, x0=got)
            got_cg = P["x"].double().cpu().numpy()
            cg_errs[f"problem_{i}"] = float(np.linalg.norm(got_cg - ref_cg) / np.linalg.norm(ref_cg))
    except Exception as ex:
        errs = {"error": str(ex)}
    rtkb.ops.joseph_band_rows(8, 8)
    bpb.close()
    cgb.close()
    return {"workload": f"{n} problems: FDK (weights + Hann ramp + backprojection) then {niter} CG iterations "
                        "(Joseph pair) from the FDK volume; volumes 64^3-256^3, 90-360 projections, detectors "
                        "128^2-512^2, SID 800-1200 mm (seeded ellipsoid phantoms)",
            "batched_ms": times["batched"], "one_problem_after_another_ms": times["one_after_another"],
            "speedup": times["one_after_another"] / times["batched"],
            "autotuned_config": best, "joseph_band_rows": {"forward": bands["forward"], "back": bands["back"]},
            "fdk_oracle_rel_l2": errs,
            f"cg_{niter}_iterations_oracle_rel_l2": cg_errs,
            "launches_batched": "one preprocessing launch per padded row length, one persistent backprojection "
                                "launch, one CUDA graph launch for every problem's CG start and iterations"}

def sart_leg(torch, rtkb, stream, niter=1):
    """SART (RTK's defaults: lambda 0.3, one projection per subset, Joseph
    forward and voxel-based back projection) on the CG configuration's problem:
    256^3 at 1 mm from 360 projections of 512x384 at 0.8 mm, seeded order."""
    from tests import phantoms

    n = 360
    g = rtkb.geometry.circular(n, SID, SDD)
    vd = rtkb.make_desc((256, 256, 256), (1.0, 1.0, 1.0))
    pd = rtkb.make_desc((512, 384, n), (0.8, 0.8, 1.0))
    ell = phantoms.random_ellipsoids(20, SEED + 2, centre_radius=60.0, axis_range=(5.0, 60.0))
    ell[:, 15] *= 0.02
    p = rtkb.ops.project_ellipsoids(g, pd, ell, stream=stream)
    x = torch.zeros((256, 256, 256), device="cuda")
    rtkb.ops.sart(g, vd, pd, p, x, niter=1, seed=1, stream=stream)  # warm-up (allocations, host tables)
    x.zero_()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    rtkb.ops.sart(g, vd, pd, p, x, niter=niter, seed=1, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    fp = rtkb.ops.joseph_forward_project(g, vd, pd, x, torch.zeros_like(p), stream=stream)
    misfit = float((fp - p).double().norm() / p.double().norm())
    return {"workload": "SART, 256^3 @1mm <- 360 x 512x384 @0.8mm, lambda 0.3, 1 projection per subset",
            "iterations": niter, "seconds_per_iteration_device": e0.elapsed_time(e1) / 1e3 / niter,
            "seconds_per_iteration_wall": wall / niter, "relative_projection_misfit_after": misfit}


def osem_leg(torch, rtkb, stream, niter=3, subset=10):
    """OSEM (RTK's default niter 3 and back projector, voxel-based; 10
    projections per subset as in RTK's OSEM test; Joseph forward projection)
    on the CG configuration's problem: 256^3 at 1 mm from 360 projections of
    512x384 at 0.8 mm, seeded order, from a constant volume of 0.01.  Timed
    without (beta 0, ML-EM updates) and with De Pierro's term (beta 0.01)."""
    from tests import phantoms

    n = 360
    g = rtkb.geometry.circular(n, SID, SDD)
    vd = rtkb.make_desc((256, 256, 256), (1.0, 1.0, 1.0))
    pd = rtkb.make_desc((512, 384, n), (0.8, 0.8, 1.0))
    ell = phantoms.random_ellipsoids(20, SEED + 2, centre_radius=60.0, axis_range=(5.0, 60.0))
    ell[:, 15] *= 0.02
    p = rtkb.ops.project_ellipsoids(g, pd, ell, stream=stream)
    x = torch.full((256, 256, 256), 0.01, device="cuda")
    for beta in (0.0, 0.01):  # warm-up of both update kernels (allocations, host tables, module loading)
        rtkb.ops.osem(g, vd, pd, p, x, niter=2, subset=subset, beta=beta, seed=1, stream=stream)
    out = {"workload": f"OSEM, 256^3 @1mm <- 360 x 512x384 @0.8mm, {subset} projections per subset, "
                       "Joseph forward / voxel-based back projection", "iterations": niter}
    for beta in (0.0, 0.01):
        x.fill_(0.01)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rtkb.ops.osem(g, vd, pd, p, x, niter=niter, subset=subset, beta=beta, seed=1, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        fp = rtkb.ops.joseph_forward_project(g, vd, pd, x, torch.zeros_like(p), stream=stream)
        misfit = float((fp - p).double().norm() / p.double().norm())
        out[f"beta_{beta:g}"] = {"seconds_device": e0.elapsed_time(e1) / 1e3, "seconds_wall": wall,
                                 "relative_projection_misfit_after": misfit}
    return out


def regularized_cg_leg(torch, rtkb, stream, main_iterations=3):
    """Regularised CG with RTK's defaults (4 CG iterations per main iteration,
    positivity, TV denoising gamma 5e-5 x 10 BPDQ iterations) on the CG
    configuration's problem (noise-free projections), 3 main iterations; and
    the TV denoiser alone on the 256^3 volume against the HBM roofline: one
    BPDQ run of n iterations must move (28 n + 8) bytes per voxel (first
    iteration: f in, the three-component dual field z out; each later one:
    f and z in, z out; final pass: f and z in, the volume out)."""
    from tests import phantoms

    n = 360
    g = rtkb.geometry.circular(n, SID, SDD)
    vd = rtkb.make_desc((256, 256, 256), (1.0, 1.0, 1.0))
    pd = rtkb.make_desc((512, 384, n), (0.8, 0.8, 1.0))
    ell = phantoms.random_ellipsoids(20, SEED + 2, centre_radius=60.0, axis_range=(5.0, 60.0))
    ell[:, 15] *= 0.02
    p = rtkb.ops.project_ellipsoids(g, pd, ell, stream=stream)
    x = torch.zeros((256, 256, 256), device="cuda")
    # warm-up with the timed call's iteration count: its first run captures and allocates per main iteration
    rtkb.ops.regularized_cg(g, vd, pd, p, x, main_loop_iterations=main_iterations, stream=stream)
    x.zero_()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    rtkb.ops.regularized_cg(g, vd, pd, p, x, main_loop_iterations=main_iterations, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    total = e0.elapsed_time(e1) / 1e3
    niter, reps = 10, 10
    out = torch.empty_like(x)
    rtkb.ops.tv_denoising_bpdq(vd, x, 5e-5, niter, out=out, stream=stream)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(reps):
        rtkb.ops.tv_denoising_bpdq(vd, x, 5e-5, niter, out=out, stream=stream)
    t1.record(stream)
    torch.cuda.synchronize()
    tv_s = t0.elapsed_time(t1) / 1e3 / reps
    tv_bytes = (28 * niter + 8) * 256 ** 3
    hbm = peaks().get("hbm_gbs")
    return {"workload": "regularised CG, 256^3 @1mm <- 360 x 512x384 @0.8mm, 4 CG iterations + positivity + "
                        "TV (gamma 5e-5, 10 BPDQ iterations) per main iteration",
            "main_iterations": main_iterations, "seconds_device": total,
            "seconds_per_main_iteration": total / main_iterations,
            "tv_denoising": {"volume": [256, 256, 256], "iterations": niter, "ms": tv_s * 1e3,
                             "roofline": {"bound": "hbm", "algorithmic_bytes": tv_bytes,
                                          "achieved_gbs": tv_bytes / tv_s / 1e9, "peak_gbs": hbm,
                                          "frac": (tv_bytes / tv_s / 1e9) / hbm if hbm else None,
                                          "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"}}}


def preprocess_leg(torch, rtkb, stream, reps=5):
    """Raw 16-bit counts to line integrals for a stack the size of the
    backprojection configuration's (720 x 768 x 1024): I0 estimation over the
    stack, then the lookup-table conversion, against the HBM roofline (the
    conversion moves 6 bytes per pixel: 2 in, 4 out; the estimation reads 2)."""
    n = 720 * 768 * 1024
    gen = torch.Generator(device="cuda").manual_seed(SEED + 4)
    raw = torch.randint(-32768, 32768, (720, 768, 1024), device="cuda", dtype=torch.int32, generator=gen)
    raw = raw.to(torch.int16).view(torch.uint16)
    desc = rtkb.make_desc((1024, 768, 720))
    out = torch.empty((720, 768, 1024), device="cuda", dtype=torch.float32)
    est = rtkb.ops.i0_estimation(desc, raw, stream=stream)
    rtkb.ops.raw_to_attenuation(desc, raw, est["i0"], out=out, stream=stream)
    torch.cuda.synchronize()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record(stream)
    for _ in range(reps):
        rtkb.ops.raw_to_attenuation(desc, raw, est["i0"], out=out, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    t_conv = e0.elapsed_time(e1) / 1e3 / reps
    t0 = time.perf_counter()
    for _ in range(reps):
        rtkb.ops.i0_estimation(desc, raw, stream=stream)  # waits for its histogram on the host
    t_est = (time.perf_counter() - t0) / reps
    hbm = peaks().get("hbm_gbs")
    gbs = 6 * n / t_conv / 1e9
    return {"workload": "720 x 768 x 1024 uniform random 16-bit counts", "i0_estimate": est["i0"],
            "conversion_ms": t_conv * 1e3,
            "conversion_roofline": {"bound": "hbm", "algorithmic_bytes": 6 * n, "achieved_gbs": gbs, "peak_gbs": hbm,
                                    "frac": gbs / hbm if hbm else None,
                                    "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"},
            "i0_estimation_ms_wall": t_est * 1e3}


def cg_seconds_to_residual(torch, rtkb, stream, tol=1e-3, max_iter=300, learned_pcg=True):
    """CG configuration: 256^3 at 1 mm, 360 projections of 512x384 at 0.8 mm
    (SID 1000, SDD 1536) of 20 seeded random ellipsoids with pre-log Poisson
    noise at I0 = 5e4; Joseph pair, FP32 vectors, FP64 scalars, one CUDA graph
    per iteration.  Seconds until the normal-equation residual falls to
    tol * ||r_0||, device time from the start of CG to convergence.  The
    learned-PCG leg trains the U-Net preconditioner on the same geometry
    (training pairs from the plan's own normal operator, hand-written
    forward/backward kernels, Adam) and solves the same problem with
    flexible PCG; training time is reported separately."""
    import numpy as np

    from tests import workloads as W

    c = W.C3
    n = c["n"]
    g = rtkb.geometry.circular(n, c["sid"], c["sdd"])
    vd = rtkb.make_desc(c["vol"], (c["vox"],) * 3)
    pd = rtkb.make_desc((*c["det"], n), (c["pix"], c["pix"], 1.0))
    # the CG configuration's inputs (tests/workloads.py): analytic projections
    # of its ellipsoids (on the GPU), seeded pre-log Poisson noise at I0 = 5e4
    clean = rtkb.ops.project_ellipsoids(g, pd, W.c3_ellipsoids(), stream=stream)
    p = torch.from_numpy(W.c3_noise(clean.double().cpu().numpy())).cuda()
    del clean

    def solve(net, storage="fp32", max_it=max_iter, backprojector="joseph"):
        x = torch.zeros((256, 256, 256), device="cuda")
        cg = rtkb.ops.ConjugateGradient(g, vd, pd, storage=storage, backprojector=backprojector)
        if net is not None:
            cg.set_preconditioner(net, history=8)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        cg.start(p, x, stream=stream)
        rr, rr0, it = cg.residual(stream)
        hist = [1.0]
        while rr > tol * tol * rr0 and it < max_it:
            cg.iterate(1, stream)
            rr, rr0, it = cg.residual(stream)
            hist.append(round((rr / rr0) ** 0.5, 6))
        e1.record(stream)
        torch.cuda.synchronize()
        secs = e0.elapsed_time(e1) / 1e3
        status = cg.preconditioner_status()
        cg.close()
        solve.hist = hist
        return (secs if rr <= tol * tol * rr0 else None), it, (rr / rr0) ** 0.5, secs / max(it, 1), status, x

    # the Joseph pair's band heights from the autotuner, timed on this problem
    bands = rtkb.ops.joseph_autotune(g, vd, pd, torch.zeros((256, 256, 256), device="cuda").add_(0.01), p,
                                     repeats=2, stream=stream)
    secs, it, rel, per_it, _, x_cg = solve(None)
    cg_hist = solve.hist
    # roofline of one iteration, the sum of its components' bounds (they run one after another): the
    # Joseph forward and back projections at the measured shared-memory gather peak (16 B per bilinear
    # sample, gathered or scattered), and the HBM traffic they cannot avoid (the volume read and the
    # projections written by the forward projector, the projections read and the volume written by
    # the back projector) plus the vector updates (about 10 volume reads and writes) at the HBM peak
    ns = rtkb.ops.joseph_sample_count(g, vd, pd, stream=stream)
    l1_peak = smem_peak_gbs(torch, rtkb.load(), stream)
    hbm_peak = peaks().get("hbm_gbs")
    nvox, npix = 256 ** 3, n * c["det"][0] * c["det"][1]
    hbm_bytes = 2 * npix * 4 + 12 * nvox * 4
    t_l1 = 2 * ns * 16 / (l1_peak * 1e9)
    t_hbm = hbm_bytes / (hbm_peak * 1e9) if hbm_peak else 0.0
    roofline = {"samples_per_projector_call": ns, "l1_bytes_per_iteration": 2 * ns * 16, "l1_peak_gbs": l1_peak,
                "hbm_bytes_per_iteration": hbm_bytes, "hbm_peak_gbs": hbm_peak,
                "seconds_per_iteration_bound": t_l1 + t_hbm,
                "seconds_to_rel_residual_1e-3_bound": (t_l1 + t_hbm) * it,
                "frac": (t_l1 + t_hbm) / per_it if per_it else None,
                "peak_source": "shared-memory gather probe of this run; MEASURED_PEAKS.json hbm_gbs (of measured)"}
    out = {"seconds_to_rel_residual_1e-3": secs, "iterations": it, "relative_residual": rel,
           "seconds_per_iteration": per_it, "roofline": roofline, "joseph_band_rows": bands,
           "residual_history": cg_hist,
           "config": "256^3 @1mm <- 360 x 512x384 @0.8mm, SID 1000, SDD 1536, 20 random ellipsoids, "
                     "Poisson I0=5e4, Joseph pair, FP32 vectors / FP64 scalars, CUDA graph per iteration",
           "learned_pcg": None}
    # RTK's default projector choice: Joseph forward, voxel-based back projector
    # (not the forward projector's adjoint, so CG solves a non-symmetric system)
    vsecs, vit, vrel, vper, _, x_vox = solve(None, backprojector="voxel", max_it=100)
    out["voxel_backprojector"] = {"seconds_to_rel_residual_1e-3": vsecs, "iterations": vit, "relative_residual": vrel,
                                  "seconds_per_iteration": vper, "residual_history": solve.hist}
    del x_vox

    # precision study: 30 iterations in one graph replay loop per storage
    # variant (FP32, or BF16 r, p, A p and projection temporary), and each
    # variant's seconds to the residual target
    def fixed(storage, niter=30):
        x = torch.zeros((256, 256, 256), device="cuda")
        cg = rtkb.ops.ConjugateGradient(g, vd, pd, storage=storage)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        cg.start(p, x, stream=stream)
        cg.iterate(niter, stream)
        e1.record(stream)
        torch.cuda.synchronize()
        rr, rr0, it = cg.residual(stream)
        cg.close()
        return e0.elapsed_time(e1) / 1e3, (rr / rr0) ** 0.5, x

    study = {"iterations": 30}
    t32, r32, x32 = fixed("fp32")
    study["fp32"] = {"seconds": t32, "relative_residual": r32}
    for variant in ("bf16", "bf16_direction"):
        tv, rv, xv = fixed(variant)
        bsecs, bit, brel, bper, _, _ = solve(None, storage=variant, max_it=100)
        study[variant] = {"seconds": tv, "relative_residual": rv,
                          "rel_diff_to_fp32": float((xv - x32).double().norm() / x32.double().norm()),
                          "seconds_to_rel_residual_1e-3": bsecs, "iterations_to_1e-3": bit if bsecs else None,
                          "residual_history": solve.hist}
        del xv
    del x32
    study["storage"] = {"bf16": "r, p, A p and the projection temporary in BF16",
                        "bf16_direction": "p and the projection temporary in BF16; r, A p and x in FP32"}
    # each variant after 3 iterations against the FP64 oracle's CG of the same
    # problem (a committed fixture: every 8th voxel of its iterate)
    try:
        fx = np.load(os.path.join(ROOT, "tests", "golden", "cg_c3_oracle.npz"))
        k, stride = int(fx["iterations"]), int(fx["stride"])
        ref = fx["x_sample"].astype(np.float64)
        errs = {}
        for variant in ("fp32", "bf16", "bf16_direction"):
            x = torch.zeros((256, 256, 256), device="cuda")
            cg = rtkb.ops.ConjugateGradient(g, vd, pd, storage=variant)
            cg.start(p, x, stream=stream)
            cg.iterate(k, stream)
            torch.cuda.synchronize()
            cg.close()
            got = x[::stride, ::stride, ::stride].double().cpu().numpy()
            errs[variant] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
        study["oracle_rel_l2_after_3_iterations"] = errs
    except Exception as ex:
        study["oracle_rel_l2_after_3_iterations"] = {"error": str(ex)}
    out["precision_study"] = study
    if not learned_pcg:
        return out
    from rtk_b200 import learned

    plan = rtkb.ops.ConjugateGradient(g, vd, pd)
    t0 = time.perf_counter()
    rs, es, _ = learned.make_training_pairs(plan, 32, seed=SEED + 5)
    torch.cuda.synchronize()
    t_pairs = time.perf_counter() - t0
    net = learned.UNet(seed=1)
    hist, t_train = learned.train(net, rs, es, steps=3000, batch=4, crop=64, lr=2e-3, lr_final=2e-4, log_every=500)
    del rs, es
    plan.close()
    psecs, pit, prel, pper, (active, fb), x_pcg = solve(net)
    net.close()
    diff = float((x_pcg - x_cg).double().norm() / x_cg.double().norm())
    out["learned_pcg"] = {
        "seconds_to_rel_residual_1e-3": psecs, "iterations": pit, "relative_residual": prel,
        "seconds_per_iteration": pper, "speedup_vs_cg": (secs / psecs) if (secs and psecs) else None,
        "fallback_to_cg_at_iteration": fb if fb >= 0 else None, "rel_diff_to_cg_solution": diff,
        "residual_history": solve.hist,
        "training": {"pairs": 32, "pairs_seconds": t_pairs, "steps": 3000, "batch": 4, "crop": 64,
                     "train_seconds": t_train, "final_loss": hist[-1][1] if hist else None},
        "method": "flexible PCG, history 8, 3-level 3D U-Net 16/32/64 (BF16 convolutions: tcgen05 forward "
                  "and data gradient, mma.sync weight gradient; FP32 accumulation), fallback to plain CG after 2 "
                  "non-improving iterations"}
    rtkb.ops.joseph_band_rows(8, 8)
    return out


def smem_peak_gbs(torch, lib, stream) -> float:
    """Measured shared-memory gather bandwidth (GB/s), best of 5."""
    import ctypes as C

    sms = torch.cuda.get_device_properties(0).multi_processor_count
    blocks, iters = sms * 8, 4096
    sink = torch.zeros(blocks, device="cuda")
    best = 0.0
    for _ in range(6):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rc = lib.rtkb_probe_smem_gather(blocks, iters, C.c_void_p(sink.data_ptr()), C.c_void_p(stream.cuda_stream))
        e1.record(stream)
        e1.synchronize()
        if rc != 0:
            return float("nan")
        t = e0.elapsed_time(e1) / 1e3
        best = max(best, blocks * 256.0 * iters * 16 / t / 1e9)
    return best


def cpu_baseline_gups(g_oracle_factory, n_proj_sample: int, threads: int):
    """RTK's CPU FDK backprojector (oracle restatement, FP32 data, FP64 coords)
    on a bounded sample: the 512^3 volume from the first n_proj_sample projections."""
    import numpy as np

    from oracle import oracle as O

    go = g_oracle_factory()
    vo = O.image((NX, NY, NZ), (VOX,) * 3)
    po = O.image((NU, NV, n_proj_sample), (PIX, PIX, 1.0))
    rng = np.random.default_rng(SEED)
    p = rng.random((n_proj_sample, NV, NU), dtype=np.float32)
    vol = np.zeros((NZ, NY, NX), dtype=np.float32)
    t0 = time.perf_counter()
    O.fdk_backproject_f32_rtk(go, vo, po, p, vol, threads=threads)
    dt = time.perf_counter() - t0
    return float(NX) * NY * NZ * n_proj_sample / dt / 1e9, dt


def oracle_slab_error(torch, proj, vol, y0=250, ny=4, r0=360, nr=40, threads=None) -> dict:
    """The checker on the timed output: relative L2 error of the volume's
    y-slab [y0, y0 + ny) against the FP64 oracle's FDK backprojection of the
    same stack.  The slab projects onto detector rows ~370-392 of every
    projection; the oracle reads rows [r0, r0 + nr) of the stack (with margin)
    and never the rest."""
    import numpy as np

    from oracle import oracle as O

    O.build()
    go = oracle_geometry()
    po = O.image((NU, NV, NP), (PIX, PIX, 1.0))
    rows = O.image((NU, nr, NP), (PIX, PIX, 1.0), origin=tuple(po.origin), index=(0, r0, 0))
    vfull = O.image((NX, NY, NZ), (VOX,) * 3)
    slab = O.image((NX, ny, NZ), (VOX,) * 3, origin=tuple(vfull.origin), index=(0, y0, 0))
    t0 = time.perf_counter()
    ref = O.backproject(go, slab, rows, proj[:, r0:r0 + nr, :].cpu().numpy().astype(np.float64), fdk=True,
                        threads=threads)
    got = vol[:, y0:y0 + ny, :].cpu().numpy().astype(np.float64)
    err = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    return {"oracle_rel_l2": err, "region": f"y-slab {y0}..{y0 + ny - 1} of the last timed step's volume",
            "oracle": "FP64 CPU restatement, ray/detector-plane voxel map", "seconds": time.perf_counter() - t0}


def legs_summary(legs: dict) -> dict:
    """The headline's compact copy of the extra legs: their numeric fields (one
    nesting level deep, 4 significant digits); the full records are the 'leg'
    lines printed before the headline."""
    def num(v):
        return isinstance(v, (int, float)) and not isinstance(v, bool)

    out = {}
    for name, d in legs.items():
        if num(d):
            out[name] = float(f"{d:.4g}")
            continue
        if not isinstance(d, dict):
            continue
        flat = {}
        for k, v in d.items():
            if num(v):
                flat[k] = float(f"{v:.4g}")
            elif isinstance(v, dict):
                for k2, v2 in v.items():
                    if num(v2):
                        flat[f"{k}.{k2}"] = float(f"{v2:.4g}")
            elif k == "error":
                flat[k] = str(v)[:120]
        out[name] = flat
    return out


def rtk_cuda_leg(torch, proj, product_ms, reps=5) -> dict:
    """RTK's own CUDA FDK back projector on the same stack: CUDA_reconstruct_conebeam
    (src/rtkCudaFDKBackProjectionImageFilter.cu, compiled unchanged from RTK's
    sources into oracle/_ref) driven in 16-projection slabs as
    CudaFDKBackProjectionImageFilter runs it, each slab copying its projections
    into a layered texture array.  Device time per backprojection, GUPS, and
    its error against the oracle on the same y-slab as the headline's check.
    The reference's GPU kernel, timed beside the product; never the product."""
    from oracle import oracle as O
    from oracle import rtk_cuda

    if not rtk_cuda.available():
        return {"unavailable": "RTK's CUDA back projector was not built (no RTK source tree where the library was built)"}
    go = oracle_geometry()
    vo = O.image((NX, NY, NZ), (VOX,) * 3)
    po = O.image((NU, NV, NP), (PIX, PIX, 1.0))
    mats = rtk_cuda.filter_matrices(O, go, vo, po)
    vin = torch.zeros((NZ, NY, NX), device="cuda")
    vout = torch.empty_like(vin)

    def run():
        rtk_cuda.fdk_backproject((NU, NV, NP), (NX, NY, NZ), mats, vin.data_ptr(), vout.data_ptr(), proj.data_ptr())

    torch.cuda.synchronize()
    run()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    times = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run()
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = statistics.median(times)
    check = oracle_slab_error(torch, proj, vout)
    return {"ms_per_backprojection": ms, "ms_each": [round(t, 1) for t in times],
            "gups": updates_per_step() / (ms / 1e3) / 1e9,
            "product_speedup": ms / product_ms, "oracle_rel_l2": check["oracle_rel_l2"],
            "kernel": "RTK kernel_fdk_3Dgrid, SLAB_SIZE 16, layered-texture bilinear (8-bit weight fractions)"}


def emit_leg(name: str, data) -> None:
    """One extra measurement as its own line, 'leg <name> <json>', printed as
    soon as it is measured (not a JSON line, so the headline stays the only
    one)."""
    print(f"leg {name} " + json.dumps(data, separators=(",", ":")), flush=True)


def oracle_geometry():
    from oracle import oracle as O

    go = O.Geometry()
    for i in range(NP):
        go.add_projection(SID, SDD, i * 360.0 / NP)
    return go


def run_reference(args, world, rank):
    """--impl reference: RTK's CPU FDK backprojector on the host cores."""
    if rank != 0:
        return 0
    from oracle import oracle as O

    O.build()
    threads = os.cpu_count() or 1
    sample = 8  # projections per step: a bounded sample of the workload
    for _ in range(args.warmup):
        cpu_baseline_gups(oracle_geometry, sample, threads)
    vals, tot = [], 0.0
    for _ in range(args.steps):
        v, dt = cpu_baseline_gups(oracle_geometry, sample, threads)
        vals.append(v)
        tot += dt
    value = float(NX) * NY * NZ * sample * args.steps / tot / 1e9
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded uniform projections)", "config": WORKLOAD,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"512^3 volume from {sample} of the 720 projections per step"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def profile_cg():
    """CG configuration kernels, each launched a few times outside any graph
    (targets for ncu --set full captures; prints a JSON line of device times).
    The Joseph band heights are autotuned first, as in the CG leg; the CG
    iterations run inside the NVTX range "rtkb_cg_iterate" (ncu --nvtx
    --nvtx-include "rtkb_cg_iterate/" selects exactly their kernels)."""
    import torch

    import rtk_b200 as rtkb
    from rtk_b200 import learned
    from tests import phantoms

    rtkb.load()
    n = 360
    g = rtkb.geometry.circular(n, SID, SDD)
    vd = rtkb.make_desc((256, 256, 256), (1.0, 1.0, 1.0))
    pd = rtkb.make_desc((512, 384, n), (0.8, 0.8, 1.0))
    ell = phantoms.random_ellipsoids(20, SEED + 2, centre_radius=60.0, axis_range=(5.0, 60.0))
    ell[:, 15] *= 0.02
    p = rtkb.ops.project_ellipsoids(g, pd, ell)
    x = torch.zeros((256, 256, 256), device="cuda")
    # the Joseph pair's band heights from the autotuner, as the CG leg runs it
    bands = rtkb.ops.joseph_autotune(g, vd, pd, torch.full_like(x, 0.01), p, repeats=1)
    cg = rtkb.ops.ConjugateGradient(g, vd, pd, use_cuda_graph=False)
    cg.start(p, x)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    cg.iterate(2)
    e1.record()
    torch.cuda.synchronize()
    t_it = e0.elapsed_time(e1) / 2
    cg.close()
    net = learned.UNet(seed=1)
    r = torch.randn((256, 256, 256), device="cuda")
    z = net.forward(r)
    torch.cuda.synchronize()
    e0.record()
    net.forward(r, z)
    e1.record()
    torch.cuda.synchronize()
    t_fwd = e0.elapsed_time(e1)
    xb = torch.randn((4, 64, 64, 64), device="cuda")
    net.train_step(xb, xb, lr=1e-3, margin=16)
    net.close()
    rtkb.ops.joseph_band_rows(8, 8)
    print(json.dumps({"profile_cg": {"cg_iteration_ms": t_it, "unet_forward_ms_256": t_fwd,
                                     "joseph_band_rows": [bands["forward"], bands["back"]],
                                     "workload": "256^3 @1mm <- 360 x 512x384 @0.8mm"}}), flush=True)
    return 0


def profile_fdk():
    """FDK preprocessing of the projector-pair stack (720 x 1024x768), twice:
    target of ncu captures of the fused weighting + ramp-filter kernel."""
    import torch

    import rtk_b200 as rtkb

    rtkb.load()
    g = make_geometry()
    pd = rtkb.make_desc((NU, NV, NP), (PIX, PIX, 1.0))
    p = torch.rand((NP, NV, NU), device="cuda", generator=torch.Generator(device="cuda").manual_seed(SEED))
    rp = rtkb.ops.ramp_params(hann=1.0)
    rtkb.ops.fdk_preprocess(g, pd, p, rp)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    rtkb.ops.fdk_preprocess(g, pd, p, rp)
    e1.record()
    torch.cuda.synchronize()
    print(json.dumps({"profile_fdk": {"preprocess_ms": e0.elapsed_time(e1),
                                      "workload": "weights + Hann ramp of 720 x 768 rows of 1024 (padded 2048)"}}))
    return 0


def profile_osem():
    """OSEM (10 projections per subset, beta 0.01) on the CG configuration's
    problem: 256^3 at 1 mm from 360 projections of 512x384; one warm-up
    iteration, then one iteration (36 subsets), for ncu launch lists."""
    import torch

    import rtk_b200 as rtkb
    from tests import phantoms

    rtkb.load()
    n = 360
    g = rtkb.geometry.circular(n, SID, SDD)
    vd = rtkb.make_desc((256, 256, 256), (1.0, 1.0, 1.0))
    pd = rtkb.make_desc((512, 384, n), (0.8, 0.8, 1.0))
    ell = phantoms.random_ellipsoids(20, SEED + 2, centre_radius=60.0, axis_range=(5.0, 60.0))
    ell[:, 15] *= 0.02
    p = rtkb.ops.project_ellipsoids(g, pd, ell)
    x = torch.full((256, 256, 256), 0.01, device="cuda")
    for _ in range(2):
        rtkb.ops.osem(g, vd, pd, p, x, niter=1, subset=10, beta=0.01, seed=1)
    torch.cuda.synchronize()
    print(json.dumps({"profile_osem": "256^3 <- 360 x 512x384, 10 per subset, beta 0.01, 2 x 1 iteration"}),
          flush=True)


def profile_tv():
    """TV denoising (BPDQ, gamma 5e-5, 3 iterations) of a uniform random 256^3
    volume, run twice: one first-iteration, two fused-iteration and one final
    launch each, for ncu captures of the TV kernels."""
    import torch

    import rtk_b200 as rtkb

    rtkb.load()
    vd = rtkb.make_desc((256, 256, 256), (1.0, 1.0, 1.0))
    x = torch.rand((256, 256, 256), device="cuda", generator=torch.Generator(device="cuda").manual_seed(SEED))
    out = torch.empty_like(x)
    for _ in range(2):
        rtkb.ops.tv_denoising_bpdq(vd, x, 5e-5, 3, out=out)
    torch.cuda.synchronize()
    print(json.dumps({"profile_tv": "256^3, 3 BPDQ iterations x 2"}), flush=True)


def use_profile_case():
    """256^3 at 0.5 mm (the benchmark's voxel size, so the same tile
    footprints and kernel configuration) from 360 of the 1024x768 projections:
    small enough for multi-pass ncu captures (1.2 GB on the device)."""
    global NX, NY, NZ, NP, WORKLOAD
    NX = NY = NZ = 256
    NP = 360
    WORKLOAD = dict(WORKLOAD, workload="profile case: FDK backprojection 256^3 @0.5mm <- 360 x 1024x768 @0.388mm",
                    volume=[NX, NY, NZ], projections=[NU, NV, NP])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra-legs", action="store_true",
                    help="skip the FDK pipeline and CG seconds-to-residual legs")
    ap.add_argument("--bp-schedule", type=int, default=0, choices=[0, 1],
                    help="tile schedule of the timed backprojections (rtkb_bp_set_schedule): 0 every tile from "
                         "projection 0 (default), 1 the projection sweep")
    ap.add_argument("--profile-cg", action="store_true",
                    help="run the CG configuration's kernels once each for ncu captures (256^3, 360 x 512x384): CG "
                         "start + 2 eager iterations, one U-Net forward on the volume, one training step on 4 x 64^3")
    ap.add_argument("--unet-wgrad-kernel", type=int, default=0, choices=[0, 1, 2],
                    help="weight-gradient kernel of the U-Net's training (rtkb_unet_set_wgrad_kernel): 0 mma.sync "
                         "(default), 1 tcgen05 M = 64, 2 tcgen05 M = 128")
    ap.add_argument("--profile-fdk", action="store_true",
                    help="FDK preprocessing (weights + Hann ramp filter) of the 720 x 1024x768 stack, twice, for ncu")
    ap.add_argument("--profile-osem", action="store_true",
                    help="OSEM on the CG configuration's problem (10 projections per subset, beta 0.01): one warm-up "
                         "iteration, then one iteration, for ncu launch lists")
    ap.add_argument("--profile-tv", action="store_true",
                    help="TV denoising (BPDQ) of a uniform random 256^3 volume, 3 iterations, twice, for ncu")
    ap.add_argument("--profile-case", action="store_true",
                    help="small case for ncu captures: 256^3 @1mm from 360 projections, device-timed region only")
    args = ap.parse_args()
    if args.unet_wgrad_kernel:
        import rtk_b200 as rtkb_w
        from rtk_b200 import build as rbuild_w

        rbuild_w.build()
        rtkb_w.ops.check(rtkb_w.load().rtkb_unet_set_wgrad_kernel(args.unet_wgrad_kernel))
    if args.profile_cg:
        return profile_cg()
    if args.profile_fdk:
        return profile_fdk()
    if args.profile_tv:
        return profile_tv()
    if args.profile_osem:
        return profile_osem()
    args.warmup = max(args.warmup, 3)
    if args.profile_case:
        use_profile_case()
    world, rank, local = dist_setup(args.gpus)
    if args.impl == "reference":
        rc = run_reference(args, world, rank)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return rc

    import torch

    import rtk_b200 as rtkb
    from rtk_b200 import build as rbuild

    rbuild.build()
    lib = rtkb.load()
    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    gen = torch.Generator(device="cuda").manual_seed(SEED + rank)

    g = make_geometry()
    vd = rtkb.make_desc((NX, NY, NZ), (VOX,) * 3)
    pd, proj, data_kind = make_projections(torch, g, gen)
    zero = torch.zeros((NZ, NY, NX), device="cuda")
    vol = torch.empty_like(zero)

    def step():
        rtkb.ops.fdk_backproject(g, vd, pd, proj, zero, out=vol, stream=stream)

    tuned = None
    rtkb.ops.backproject_schedule(args.bp_schedule)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if args.profile_case:
        step()
        torch.cuda.synchronize()
        assert rtkb.ops.device_status(stream) == 0
        print(json.dumps({"profile_case": WORKLOAD}), flush=True)
        return 0

    # ---- device-timed region: inputs resident in HBM ----
    sampler = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with sampler:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    t = max_over_ranks(e0.elapsed_time(e1) / 1e3, world)
    clocks = sampler.summary()
    assert rtkb.ops.device_status(stream) == 0
    value = updates_per_step() * args.steps * world / t / 1e9
    ms_per_step = t / args.steps * 1e3

    # ---- end to end through the C ABI: pinned host stack in, pinned host volume out ----
    h_proj = torch.empty((NP, NV, NU), dtype=torch.float32, pin_memory=True)
    h_proj.copy_(proj)
    h_vol = torch.empty((NZ, NY, NX), dtype=torch.float32, pin_memory=True)

    def e2e_step():
        # the stack streams to the device in chunks whose copies overlap the
        # backprojection of the previous chunk; the volume comes back at the end
        rtkb.ops.fdk_backproject_host(g, vd, pd, h_proj, None, out=h_vol, stream=stream)

    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    barrier(world)
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    f1.record(stream)
    torch.cuda.synchronize()
    te = max_over_ranks(f0.elapsed_time(f1) / 1e3, world)
    e2e_value = updates_per_step() * args.steps * world / te / 1e9

    # ---- roofline: L1/shared-memory gather bound ----
    peak_smem = smem_peak_gbs(torch, lib, stream)
    achieved = updates_per_step() * L1_BYTES_PER_UPDATE / (t / args.steps) / 1e9
    pk = peaks()
    hbm_bytes = (NX * NY * NZ * 4 * 2) + (NP * NV * NU * 4)
    roofline = {"bound": "l1", "achieved": achieved, "peak": peak_smem, "unit": "GB/s",
                "frac": achieved / peak_smem if peak_smem else None,
                "traffic": BP_DRAM_BYTES_BY_SCHEDULE[args.bp_schedule] if NX == 512 else None,
                "traffic_source": "recorded constant: ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                                  f"full-size launch of the kernel at commit {BP_TRAFFIC_COMMIT}",
                "peak_source": "measured in this run: shared-memory bilinear-gather probe (rtkb_probe_smem_gather)",
                "per_launch_updates": updates_per_step(), "bytes_per_update": L1_BYTES_PER_UPDATE,
                "hbm": {"algorithmic_bytes_per_launch": hbm_bytes,
                        "achieved_gbs": hbm_bytes / (t / args.steps) / 1e9,
                        "peak_gbs": pk.get("hbm_gbs"), "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"}}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": f"synthetic: {data_kind}", "config": WORKLOAD,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h_proj.numel() * 4,
                    "d2h_bytes_per_step": h_vol.numel() * 4,
                    "path": "rtkb_fdk_backproject_host via ctypes: pinned host stack in, pinned host volume out, "
                            "the stack's copy (subsets growing x1.5 from 15 to 180 projections, the last one the "
                            "remainder) and the volume's copy back (slabs of halving size) overlapped with the backprojection, all "
                            "inside the timed region"},
            "roofline": roofline, "clocks": clocks, "gpu_launches": args.steps,
            "gpu_launches_note": "one rtkb backprojection kernel per step (plus one matrix upload copy)",
            "autotune": tuned}

    legs = {}
    if world == 1 and not args.no_extra_legs:
        # the project's autotuner on this workload (every configuration timed on
        # the real stack, after the timed region): which configuration it picks
        # against the footprint heuristic the timed steps used
        heuristic_cfg, _ = rtkb.ops.backproject_config(-1)
        best, best_ms, times = rtkb.ops.backproject_autotune([(g, vd, pd, proj, zero, vol)], repeats=1, stream=stream)
        line["autotune"] = {"config": best, "heuristic_config": heuristic_cfg,
                            "ms_per_config": [round(t, 2) for t in times]}
        rtkb.ops.fdk_backproject(g, vd, pd, proj, zero, out=vol, stream=stream)

    # the checker on the last timed output (outside every timed region), and
    # the reference's own CUDA back projector on the same stack
    if rank == 0 and world == 1 and not args.no_cpu_baseline and NX == 512:
        try:
            line["oracle_check"] = oracle_slab_error(torch, proj, vol)
        except Exception as ex:  # the check is reported; a failure to run it is reported too
            line["oracle_check"] = {"oracle_rel_l2": None, "error": str(ex)}
        try:
            line["rtk_cuda_reference"] = rtk_cuda_leg(torch, proj, ms_per_step)
        except Exception as ex:
            line["rtk_cuda_reference"] = {"error": str(ex)}

    if world == 1 and not args.no_extra_legs:
        def leg(name, fn, *a, **kw):
            try:
                legs[name] = fn(*a, **kw)
            except Exception as ex:
                legs[name] = {"error": str(ex)}
            if rank == 0:
                emit_leg(name, legs[name])

        leg("bf16_storage", bf16_storage_leg, torch, rtkb, g, vd, pd, proj, vol, stream, peak_smem)
        leg("fdk_pipeline_ms", fdk_pipeline_ms, torch, rtkb, g, vd, pd, proj, stream)
        leg("ramp_filter", ramp_leg, torch, rtkb, g, pd, proj)
        leg("voxel_backprojection", voxel_bp_leg, torch, rtkb, g, vd, pd, proj, stream)
        leg("projection_sweep", sweep_leg, torch, rtkb, g, vd, pd, proj, vol, stream, args.bp_schedule)
        del proj
        leg("joseph_forward", joseph_forward_leg, torch, rtkb, lib, stream)
        leg("joseph_back", joseph_back_leg, torch, rtkb, lib, stream)
        leg("batched", batch_leg, torch, rtkb, stream)
        leg("batched_fdk_cg", c4_leg, torch, rtkb, stream)
        leg("sart", sart_leg, torch, rtkb, stream)
        leg("osem", osem_leg, torch, rtkb, stream)
        leg("regularized_cg", regularized_cg_leg, torch, rtkb, stream)
        leg("preprocess", preprocess_leg, torch, rtkb, stream)
        leg("cg", cg_seconds_to_residual, torch, rtkb, stream)
        line["legs"] = legs_summary(legs)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            threads = os.cpu_count() or 1
            gups_probe, dt = cpu_baseline_gups(oracle_geometry, 2, threads)
            n_s = int(max(2, min(64, 15.0 / max(dt / 2, 1e-3))))
            gups, dt = cpu_baseline_gups(oracle_geometry, n_s, threads)
            line["cpu_baseline"] = {"value": gups, "unit": UNIT, "cores": threads, "kind": "port",
                                    "sample": f"512^3 volume from {n_s} of the 720 projections ({dt:.1f} s)"}
        except Exception as ex:  # the baseline is reported, never the target
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                                    "sample": f"failed: {ex}"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

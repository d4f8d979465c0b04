// backproject.cu -- voxel-driven FDK and voxel-based backprojection on sm_100a.
//
// Replaces CUDA_reconstruct_conebeam (src/rtkCudaFDKBackProjectionImageFilter.cu:95-137)
// and CUDA_back_project (src/rtkCudaBackProjectionImageFilter.cu:125-172) behind
// rtk::FDKBackProjectionImageFilter / rtk::BackProjectionImageFilter, with the
// arithmetic of RTK's CPU filters (include/rtkFDKBackProjectionImageFilter.hxx:152-306,
// include/rtkBackProjectionImageFilter.hxx:352-475): software bilinear
// interpolation with FP64-derived coordinates instead of hardware texture
// filtering, so results match the CPU filters to FP32 rounding.
//
// Design (circular geometries, RTK's optimised-Y path, the common case):
//  * one CTA owns a 16 (x) x NYT (y) x 16 (z) voxel tile and loops over every
//    projection of the stack, accumulating in registers: the volume is read and
//    written once per call;
//  * warp 8 is the producer: per projection it projects the tile's corners in
//    FP64, sizes the detector footprint, writes FP32 tile-relative projection
//    coefficients into a stage header and TMA-loads the footprint box
//    (BW x BH floats, no multicast) into a 4-stage shared-memory ring;
//  * warps 0-7 are consumers: thread (x, z) owns a y-column of NYT voxels.  For
//    the optimised-Y geometry u and w do not depend on y, so the reciprocal, u
//    and its interpolation weight are computed once per column and projection,
//    and each voxel costs one v step, four shared-memory loads and three lerps;
//  * coordinates are relative to the footprint box, so FP32 keeps ~1e-5 pixel
//    accuracy; a tile whose footprint does not fit the box (or whose corners
//    are not all in front of the source) falls back to an FP64 global-memory
//    path for that projection.
#include "rtkb_backproject.h"
#include "rtkb_internal.h"
#include "rtkb_ptx.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <type_traits>

namespace rtkb
{
namespace dev
{
__device__ unsigned int g_device_status = 0;
__device__ unsigned int g_wait_limit = kDefaultWaitLimit;
}
struct BatchProblemHandle; // device-side problem table of a prepared batch
} // namespace rtkb

namespace
{
using namespace rtkb::dev;

constexpr int kTX = 16;
constexpr int kTZ = 16;
constexpr int kConsumerWarps = 8;
constexpr int kThreads = 32 * (kConsumerWarps + 1);
constexpr int kStages = 4;
constexpr int kHeaderBytes = 256;

struct __align__(16) StageHeader
{
  float4 a0;    // u numerator: A0x A0y A0z c0 (box-relative)
  float4 a1;    // v numerator
  float4 a2;    // w
  float4 lim;   // valid u range [x, y), valid v range [z, w) (box-relative)
  int4   fl;    // flags, ub, vb, unused
  double m[12]; // FP64 buffer-index matrix: boundary decisions and the slow path
  float  mf[12]; // FP32 copy: corner projection for the footprint box
};
static_assert(sizeof(StageHeader) <= kHeaderBytes, "stage header overflow");

// Samples whose FP32 coordinate lies within kBand pixels of a detector bound
// are accepted or rejected with FP64 arithmetic, so RTK's hard acceptance
// test (0 <= floor(u) <= N-2) is decided as the FP64 CPU filters decide it.
constexpr float kBand = 1e-3f;

__device__ __forceinline__ float
rcp_approx(float x)
{
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

constexpr float kFloorBias = 12582912.f;     // 1.5 * 2^23
constexpr int   kFloorBiasBits = 0x4B400000; // its bit pattern

// Stored projection element: float32, or bfloat16 (BF16 storage variant;
// interpolation and accumulation stay FP32).
template <typename T>
__device__ __forceinline__ float
tap(const T * p)
{
  return *p;
}
template <>
__device__ __forceinline__ float
tap<__nv_bfloat16>(const __nv_bfloat16 * p)
{
  return __uint_as_float((unsigned)*reinterpret_cast<const unsigned short *>(p) << 16);
}
template <typename T>
__device__ __forceinline__ float
gtap(const T * p)
{
  return __ldg(p);
}
template <>
__device__ __forceinline__ float
gtap<__nv_bfloat16>(const __nv_bfloat16 * p)
{
  return __uint_as_float((unsigned)__ldg(reinterpret_cast<const unsigned short *>(p)) << 16);
}
template <typename T>
__device__ __forceinline__ T
zero_elem()
{
  return T(0);
}
template <>
__device__ __forceinline__ __nv_bfloat16
zero_elem<__nv_bfloat16>()
{
  return __ushort_as_bfloat16((unsigned short)0);
}
// TMA boxes must start at x * sizeof(T) = 0 mod 16
template <typename T>
constexpr int kAlignElems = 16 / (int)sizeof(T);

__device__ __noinline__ bool
accept_fp64(const double * m, int row, int X, int Y, int Z, int n)
{
  const double x = X, y = Y, z = Z;
  const double rw = 1.0 / (m[8] * x + m[9] * y + m[10] * z + m[11]);
  const double c = (m[row * 4 + 0] * x + m[row * 4 + 1] * y + m[row * 4 + 2] * z + m[row * 4 + 3]) * rw;
  return c >= 0.0 && c < n - 1.0;
}

constexpr int kFlagFast = 1;
constexpr int kFlagUInterior = 2;
constexpr int kFlagVInterior = 4;
constexpr int kFlagSkip = 8; // the whole tile projects off the detector

template <int BW, int BH, typename T = float>
struct Layout
{
  static constexpr int kBoxBytes = BW * BH * (int)sizeof(T);
  // TMA writes its boxes to 128-byte aligned shared memory: the ring's stride
  // is the box rounded up to 128 bytes
  static constexpr int kBoxStride = (kBoxBytes + 127) / 128 * 128;
  static constexpr int kBoxStrideElems = kBoxStride / (int)sizeof(T);
  static constexpr int kHeaders = 0;
  static constexpr int kBoxes = kStages * kHeaderBytes;
  static constexpr int kBars = kBoxes + kStages * kBoxStride;
  static_assert(kBoxes % 128 == 0 && kBoxStride % 128 == 0, "TMA box destinations must be 128-byte aligned");
  static constexpr int kTotal = kBars + 2 * kStages * 8;
};

// FP64 slow path for one voxel and projection: RTK's optimised-path
// arithmetic with global-memory bilinear taps.  Out of line: the rare path's
// FP64 registers stay off the hot loop.
template <typename T>
__device__ __noinline__ float
slow_voxel(const double * M, const T * __restrict__ proj, long long pofs, int nu, int nv, int X, int Y, int Z,
           bool fdkw)
{
  const double x = X, y = Y, z = Z;
  const double w = M[8] * x + M[9] * y + M[10] * z + M[11];
  const double rw = 1.0 / w;
  const double u = (M[0] * x + M[1] * y + M[2] * z + M[3]) * rw;
  const double v = (M[4] * x + M[5] * y + M[6] * z + M[7]) * rw;
  if (!(u >= 0.0 && u < nu - 1.0 && v >= 0.0 && v < nv - 1.0))
    return 0.f;
  const int     iu = (int)floor(u), iv = (int)floor(v);
  const double  fu = u - iu, fv = v - iv;
  const T *     q = proj + pofs + (long long)iv * nu + iu;
  const double  a = (1 - fu) * gtap(q) + fu * gtap(q + 1);
  const double  b = (1 - fu) * gtap(q + nu) + fu * gtap(q + nu + 1);
  const double  val = (1 - fv) * a + fv * b;
  return (float)(fdkw ? rw * rw * val : val);
}

constexpr size_t kProgressBytes = 16; // the sweep counter, after a launch's matrices and modes

// Launches of at most this many projections start each tile's accumulators
// from the input volume (bp_consumer's INIT form).
constexpr int kInitFromInputMaxProjections = 256;

// Projection sweep (tile schedule 1, rtkb_bp_set_schedule): the producers of
// one launch count the 2^shift-projection chunks they have issued in one
// device counter, and a tile starts at the projection the resident CTAs have
// reached on average (counter x 2^shift / resident CTAs, modulo the stack)
// and walks the stack from there, wrapping around.  Tiles that start at
// different times then read the same projections at the same time and share
// their detector rows in L2 (DRAM reads of the 512^3 <- 720 x 1024x768 launch:
// 69.4 -> 13.2 GB).  It changes the order in which a voxel's projections are
// summed (FP32 rounding, different from run to run), not the terms.
struct Sweep
{
  unsigned * counter;
  unsigned   ctas, shift;
};

// Producer warp: per projection, project the tile's corners, size the
// footprint box, publish the tile-relative coefficients and start the TMA
// load of the box.
// gbase: projections this CTA's ring has already carried (persistent
// kernels continue the stage index and barrier parity across tiles).
// Returns false when a bounded wait gave up.
// SWEEP: start at the sweep's projection (sw) instead of projection 0; the
// stage header then carries each stage's projection index for the consumers.
template <int BW, int BH, int NYT, typename T, bool SWEEP = false>
__device__ __forceinline__ bool
bp_producer(const CUtensorMap * tmap, const T * __restrict__ proj, const double * __restrict__ mats, int nproj,
            int nu, int nv, int x0, int y0, int z0, StageHeader * hdr, T * boxes, uint64_t * full,
            uint64_t * empty, int use_tma, unsigned gbase = 0, Sweep sw = Sweep{ nullptr, 1u, 0u })
{
  using L = Layout<BW, BH, T>;
  const int lane = threadIdx.x & 31;
  if (use_tma && lane == 0)
    prefetch_tensor_map(tmap);
  // Footprint of the whole tile, including voxels beyond a ragged volume
  // edge: consumers compute (but never store) those y's, so their shared-
  // memory taps must stay inside the box too.
  const int   x1 = x0 + kTX - 1, y1 = y0 + NYT - 1, z1 = z0 + kTZ - 1;
  const int   c = lane & 7;
  const float X = (float)((c & 1) ? x1 : x0), Y = (float)((c & 2) ? y1 : y0), Z = (float)((c & 4) ? z1 : z0);
  // Lanes 0-11 each carry one matrix entry, loaded one projection ahead; the
  // matrix goes through the stage header (FP64 and an FP32 copy) so the warp
  // reads it from shared memory instead of holding it in registers.
  int p0 = 0; // the tile's first projection
  if constexpr (SWEEP)
  {
    if (lane == 0 && nproj > 0)
    {
      const unsigned long long c = *static_cast<volatile unsigned *>(sw.counter);
      p0 = (int)(((c << sw.shift) / sw.ctas) % (unsigned long long)nproj);
    }
    p0 = __shfl_sync(0xffffffffu, p0, 0);
  }
  double mnext = (lane < 12 && nproj > 0) ? __ldg(mats + 12 * (long long)p0 + lane) : 0.0;
  for (int j = 0; j < nproj; j++)
  {
    const int      p = SWEEP ? ((p0 + j < nproj) ? p0 + j : p0 + j - nproj) : j;
    const unsigned gp = gbase + (unsigned)j;
    const int      s = (int)(gp % kStages);
    const unsigned k = gp / kStages;
    if (gp >= (unsigned)kStages && !mbar_wait(&empty[s], (k - 1) & 1))
      return false;
    StageHeader * h = hdr + s;
    if (lane < 12)
    {
      h->m[lane] = mnext;
      h->mf[lane] = (float)mnext;
    }
    if (lane < 12 && j + 1 < nproj)
      mnext = __ldg(mats + 12 * (long long)(SWEEP ? ((p + 1 < nproj) ? p + 1 : 0) : p + 1) + lane);
    if constexpr (SWEEP)
    {
      if (lane == 0 && ((j + 1) & ((1 << sw.shift) - 1)) == 0)
        atomicAdd(sw.counter, 1u);
    }
    __syncwarp();
    // The box needs the corners to ~1e-4 pixel only: FP32 is enough.
    const float * mf = h->mf;
    const float   tw = mf[8] * X, ty = mf[9] * Y, tz = mf[10] * Z;
    const float   w = tw + ty + tz + mf[11];
    const float   wtol = 1e-4f * (fabsf(tw) + fabsf(ty) + fabsf(tz) + fabsf(mf[11]));
    const float   rw = 1.0f / w;
    float         umin = fmaf(mf[0], X, fmaf(mf[1], Y, fmaf(mf[2], Z, mf[3]))) * rw, umax = umin;
    float         vmin = fmaf(mf[4], X, fmaf(mf[5], Y, fmaf(mf[6], Z, mf[7]))) * rw, vmax = vmin;
    int           wsign = (w > wtol) ? 1 : ((w < -wtol) ? 2 : 3); // bits: 1 positive, 2 negative
#pragma unroll
    for (int o = 1; o < 8; o <<= 1)
    {
      umin = fminf(umin, __shfl_xor_sync(0xffffffffu, umin, o));
      umax = fmaxf(umax, __shfl_xor_sync(0xffffffffu, umax, o));
      vmin = fminf(vmin, __shfl_xor_sync(0xffffffffu, vmin, o));
      vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
      wsign |= __shfl_xor_sync(0xffffffffu, wsign, o);
    }
    // The tile's image is the hull of its projected corners only when w has
    // one sign over the tile (no voxel at the source plane).  Matrices are
    // finite (checked on the host), so a NaN or infinite u/v needs w near 0 at
    // a corner, which fails the sign test.
    const float margin = 0.05f;
    bool        fast = (wsign == 1 || wsign == 2) && isfinite(umin) && isfinite(umax) && isfinite(vmin) &&
               isfinite(vmax) && fabsf(umin) < 1e7f && fabsf(umax) < 1e7f && fabsf(vmin) < 1e7f && fabsf(vmax) < 1e7f;
    int ub = 0, vb = 0;
    if (fast)
    {
      ub = ((int)floorf(umin - margin)) & ~(kAlignElems<T> - 1);
      vb = (int)floorf(vmin - margin);
      fast = (umax + margin < (float)(ub + BW - 1)) && (vmax + margin < (float)(vb + BH - 1));
    }
    // Every voxel of the tile fails RTK's acceptance test (0 <= u < nu-1,
    // 0 <= v < nv-1) when its footprint lies beyond a detector edge.
    const bool skip = fast && ((umax + margin < 0.f) || (umin - margin >= (float)(nu - 1)) ||
                               (vmax + margin < 0.f) || (vmin - margin >= (float)(nv - 1)));
    if (skip)
      fast = false;
    const double * m = h->m;
    T *      box = boxes + s * L::kBoxStrideElems;
    if (lane == 0)
    {
      int flags = 0;
      if (fast)
      {
        const double wo = m[8] * x0 + m[9] * y0 + m[10] * z0 + m[11];
        const double uo = m[0] * x0 + m[1] * y0 + m[2] * z0 + m[3];
        const double vo = m[4] * x0 + m[5] * y0 + m[6] * z0 + m[7];
        h->a0 = make_float4((float)(m[0] - ub * m[8]), (float)(m[1] - ub * m[9]), (float)(m[2] - ub * m[10]),
                            (float)(uo - ub * wo));
        h->a1 = make_float4((float)(m[4] - vb * m[8]), (float)(m[5] - vb * m[9]), (float)(m[6] - vb * m[10]),
                            (float)(vo - vb * wo));
        h->a2 = make_float4((float)m[8], (float)m[9], (float)m[10], (float)wo);
        h->lim = make_float4((float)(-ub), (float)(nu - 1 - ub), (float)(-vb), (float)(nv - 1 - vb));
        flags = kFlagFast;
        if (umin - margin >= 0.0 && umax + margin < nu - 1.0)
          flags |= kFlagUInterior;
        if (vmin - margin >= 0.0 && vmax + margin < nv - 1.0)
          flags |= kFlagVInterior;
      }
      h->fl = make_int4(skip ? kFlagSkip : flags, ub, vb, SWEEP ? p : 0);
    }
    if (fast && use_tma)
    {
      if (lane == 0)
      {
        mbar_arrive_expect_tx(&full[s], (uint32_t)L::kBoxBytes);
        tma_load_3d(box, tmap, ub, vb, p, &full[s]);
      }
    }
    else
    {
      if (fast)
      {
        // plain-load fallback when the stack cannot be described to TMA
        const long long pofs = (long long)p * nu * nv;
        for (int e = lane; e < BW * BH; e += 32)
        {
          const int gu = ub + e % BW, gv = vb + e / BW;
          box[e] = (gu >= 0 && gu < nu && gv >= 0 && gv < nv) ? proj[pofs + (long long)gv * nu + gu] : zero_elem<T>();
        }
      }
      __syncwarp();
      if (lane == 0)
        mbar_arrive(&full[s]);
    }
  }
  // drain: wait for the last copies to land before the CTA may exit
  for (int p = max(0, nproj - kStages); p < nproj; p++)
  {
    const unsigned gp = gbase + (unsigned)p;
    if (!mbar_wait(&full[gp % kStages], (gp / kStages) & 1))
      return false;
  }
  return true;
}

// Consumer warps: thread (x, z) of the tile accumulates its y-column over the
// stack and adds it to the volume.  Returns false when a bounded wait gave up.
template <int BW, int BH, int NYT, bool FDKW, typename T, bool SWEEP = false, bool INIT = false>
__device__ __forceinline__ bool
bp_consumer(const T * __restrict__ proj, int nproj, int nu, int nv, int nx, int ny, int nz, int x0, int y0, int z0,
            const StageHeader * hdr, const T * boxes, uint64_t * full, uint64_t * empty, const float * vol_in,
            float * vol_out, unsigned gbase = 0)
{
  const int lane = threadIdx.x & 31;
  // --------------------------------------------------------------- consumers
  const int   t = threadIdx.x;
  // warp w covers x in [8 (w % 2), +8) and z in [4 (w / 2), +4): 8 x 4
  // voxels whose taps span few detector columns (see the box widths below)
  const int   dx = (lane & 7) + 8 * ((t >> 5) & 1), dz = (lane >> 3) + 4 * (t >> 6);
  const int   X = x0 + dx, Z = z0 + dz;
  const bool  active = (X < nx) && (Z < nz);
  const float fdx = (float)dx, fdz = (float)dz;
  static_assert(NYT % 2 == 0, "voxel columns are processed in pairs");
  // Accumulators of voxels 2k and 2k+1 share a register pair, so the
  // interior loop runs on sm_100's packed FP32 instructions (FFMA2).
  float2      acc2[NYT / 2];
#define BP_ACC(j) (((j) & 1) ? acc2[(j) >> 1].y : acc2[(j) >> 1].x)
  if constexpr (INIT)
  {
    // short launches: the accumulators start from the input volume, as RTK's
    // filters add every projection into the output image, and its loads are
    // in flight while the first box arrives instead of after the last one
#pragma unroll
    for (int j = 0; j < NYT; j++)
      BP_ACC(j) = (active && y0 + j < ny) ? vol_in[((long long)Z * ny + y0 + j) * nx + X] : 0.f;
  }
  else
  {
#pragma unroll
    for (int k = 0; k < NYT / 2; k++)
      acc2[k] = make_float2(0.f, 0.f);
    // the input volume is read after the last projection: start pulling it
    // into L2 now, so that tiles do not wait on DRAM at their end
    if (active)
    {
#pragma unroll
      for (int j = 0; j < NYT; j++)
        if (y0 + j < ny)
          asm volatile("prefetch.global.L2 [%0];" ::"l"(vol_in + ((long long)Z * ny + y0 + j) * nx + X));
    }
  }

  for (int p = 0; p < nproj; p++)
  {
    const unsigned gp = gbase + (unsigned)p;
    const int      s = (int)(gp % kStages);
    if (!mbar_wait(&full[s], (gp / kStages) & 1))
      return false;
    const StageHeader * h = hdr + s;
    const T *           box = boxes + s * Layout<BW, BH, T>::kBoxStrideElems;
    const int4          fl = h->fl;
    if (active)
    {
      if (fl.x & kFlagFast)
      {
        const float4 a0 = h->a0, a1 = h->a1, a2 = h->a2;
        const float  nw = fmaf(a2.x, fdx, fmaf(a2.z, fdz, a2.w));
        const float  rw = rcp_approx(nw); // <= 1 ulp: ~1e-5 pixel at |u| <= 64
        const float  u = fmaf(a0.x, fdx, fmaf(a0.z, fdz, a0.w)) * rw;
        const float  v0 = fmaf(a1.x, fdx, fmaf(a1.z, fdz, a1.w)) * rw;
        const float  dv = a1.y * rw;
        const float  wt = FDKW ? rw * rw : 1.f;
        bool         uok = true;
        if (!(fl.x & kFlagUInterior))
        {
          const float4 lim = h->lim;
          uok = (u >= lim.x && u < lim.y);
          if (fabsf(u - lim.x) < kBand || fabsf(u - lim.y) < kBand)
            uok = accept_fp64(h->m, 0, X, y0, Z, nu); // u does not depend on y on this path
        }
        if (uok)
        {
          const float   flu = floorf(u);
          const float   fu = u - flu;
          const T *     col = box + (int)flu;
          if (fl.x & kFlagVInterior)
          {
            // Voxels j and j+1 per step on packed FP32 instructions: the
            // same operations and roundings as one voxel at a time, with
            // b - a written as fma(-1, a, b), so the sums are bit-identical.
            const float2 fu2 = make_float2(fu, fu), wt2 = make_float2(wt, wt);
            const float2 m1 = make_float2(-1.f, -1.f);
#pragma unroll
            for (int j = 0; j < NYT; j += 2)
            {
              const float2 v = make_float2(fmaf((float)j, dv, v0), fmaf((float)(j + 1), dv, v0));
              float2 fv;
              const T * qa;
              const T * qb;
              if constexpr (sizeof(T) == 4)
              {
                // floor(v) and its integer without the conversion unit: for
                // |v| < 2^22, v + 1.5 * 2^23 lies in [2^23, 2^24), where floats
                // are spaced 1, so rounding the sum toward zero gives floor(v)
                // + 1.5 * 2^23 exactly, and its low mantissa bits floor(v) +
                // 2^22.  Bit-identical to floorf and (int)floorf; v stays
                // inside the box here.  (Slower with BF16 taps, whose
                // widening already keeps the integer pipes busy.)
                const float2 tb = __fadd2_rz(v, make_float2(kFloorBias, kFloorBias));
                fv = __ffma2_rn(m1, __fadd2_rn(tb, make_float2(-kFloorBias, -kFloorBias)), v);
                qa = col + (__float_as_int(tb.x) - kFloorBiasBits) * BW;
                qb = col + (__float_as_int(tb.y) - kFloorBiasBits) * BW;
              }
              else
              {
                const float2 fl = make_float2(floorf(v.x), floorf(v.y));
                fv = __ffma2_rn(m1, fl, v);
                qa = col + (int)fl.x * BW;
                qb = col + (int)fl.y * BW;
              }
              const float2 p00 = make_float2(tap(qa), tap(qb)), p01 = make_float2(tap(qa + 1), tap(qb + 1));
              const float2 p10 = make_float2(tap(qa + BW), tap(qb + BW));
              const float2 p11 = make_float2(tap(qa + BW + 1), tap(qb + BW + 1));
              const float2 r0 = __ffma2_rn(fu2, __ffma2_rn(m1, p00, p01), p00);
              const float2 r1 = __ffma2_rn(fu2, __ffma2_rn(m1, p10, p11), p10);
              acc2[j >> 1] = __ffma2_rn(wt2, __ffma2_rn(fv, __ffma2_rn(m1, r0, r1), r0), acc2[j >> 1]);
            }
          }
          else
          {
            // Acceptance mask in FP32; voxels within kBand of a bound are
            // re-decided in FP64 outside the unrolled loop.
            const float4 lim = h->lim;
            unsigned     ok = 0, near = 0;
#pragma unroll
            for (int j = 0; j < NYT; j++)
            {
              const float v = fmaf((float)j, dv, v0);
              ok |= (v >= lim.z && v < lim.w) ? (1u << j) : 0u;
              near |= (fabsf(v - lim.z) < kBand || fabsf(v - lim.w) < kBand) ? (1u << j) : 0u;
            }
            while (near)
            {
              const int j = __ffs(near) - 1;
              near &= near - 1;
              ok = accept_fp64(h->m, 1, X, y0 + j, Z, nv) ? (ok | (1u << j)) : (ok & ~(1u << j));
            }
#pragma unroll
            for (int j = 0; j < NYT; j++)
            {
              if (ok & (1u << j))
              {
                const float   v = fmaf((float)j, dv, v0);
                const float   flv = floorf(v);
                const float   fv = v - flv;
                const T *     q = col + (int)flv * BW;
                const float   p00 = tap(q), p01 = tap(q + 1), p10 = tap(q + BW), p11 = tap(q + BW + 1);
                const float   r0 = fmaf(fu, p01 - p00, p00);
                const float   r1 = fmaf(fu, p11 - p10, p10);
                BP_ACC(j) = fmaf(wt, fmaf(fv, r1 - r0, r0), BP_ACC(j));
              }
            }
          }
        }
      }
      else if (!(fl.x & kFlagSkip))
      {
        const long long pofs = (long long)(SWEEP ? fl.w : p) * nu * nv; // the stage's projection
#pragma unroll
        for (int j = 0; j < NYT; j++)
          BP_ACC(j) += slow_voxel(h->m, proj, pofs, nu, nv, X, y0 + j, Z, FDKW);
      }
    }
    __syncwarp();
    if (lane == 0)
      mbar_arrive(&empty[s]);
  }

  if (active)
  {
#pragma unroll
    for (int j = 0; j < NYT; j++)
    {
      const int Y = y0 + j;
      if (Y < ny)
      {
        const long long o = ((long long)Z * ny + Y) * nx + X;
        vol_out[o] = INIT ? BP_ACC(j) : vol_in[o] + BP_ACC(j);
      }
    }
  }
  return true;
}
#undef BP_ACC

template <int BW, int BH, int NYT, int MINB, bool FDKW, typename T = float, bool SWEEP = false, bool INIT = false>
__global__ void __launch_bounds__(kThreads, MINB)
bp_tiled_kernel(const __grid_constant__ CUtensorMap tmap, const T * __restrict__ proj,
                const double * __restrict__ mats, int nproj, int nu, int nv, int nx, int ny, int nz, int ntx,
                int ntz, const float * vol_in, float * vol_out, int use_tma, Sweep sw)
{
  using L = Layout<BW, BH, T>;
  extern __shared__ __align__(1024) unsigned char smem[];
  StageHeader * hdr = reinterpret_cast<StageHeader *>(smem + L::kHeaders);
  T *           boxes = reinterpret_cast<T *>(smem + L::kBoxes);
  uint64_t *    full = reinterpret_cast<uint64_t *>(smem + L::kBars);
  uint64_t *    empty = full + kStages;

  const int warp = threadIdx.x >> 5;
  const int b = blockIdx.x;
  const int tx = b % ntx, tz = (b / ntx) % ntz, ty = b / (ntx * ntz);
  const int x0 = tx * kTX, y0 = ty * NYT, z0 = tz * kTZ;

  if (threadIdx.x == 0)
  {
    for (int s = 0; s < kStages; s++)
    {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kConsumerWarps);
    }
    fence_barrier_init();
  }
  __syncthreads();

  if (warp == kConsumerWarps)
  {
    bp_producer<BW, BH, NYT, T, SWEEP>(&tmap, proj, mats, nproj, nu, nv, x0, y0, z0, hdr, boxes, full, empty, use_tma,
                                       0u, sw);
    return;
  }

  bp_consumer<BW, BH, NYT, FDKW, T, SWEEP, INIT>(proj, nproj, nu, nv, nx, ny, nz, x0, y0, z0, hdr, boxes, full, empty, vol_in,
                                           vol_out);
}

constexpr int kBatchSmemExtra = 1024 + 16; // base alignment slack + work item + abort flag

// One problem of a persistent batched launch: its own TMA descriptor (in
// global memory), matrices, sizes and volumes; tile_begin = index of its
// first work item in the batch's queue.
struct __align__(64) BatchProblem
{
  CUtensorMap    tmap;
  const float *  proj;
  const double * mats;
  const float *  vin;
  float *        vout;
  long long      tile_begin;
  int            nproj, nu, nv, nx, ny, nz, ntx, ntz, use_tma, pad;
};

// Persistent batched backprojection: every CTA takes (problem, tile) work
// items from a global counter until the queue is empty, so many problems of
// uneven sizes share one launch without tail effects per problem.  The
// stage ring continues across items (gbase), so no barrier is re-armed; a
// bounded wait that gives up raises a CTA-wide abort at the next item.
template <int BW, int BH, int NYT, int MINB, bool FDKW>
__global__ void __launch_bounds__(kThreads, MINB)
bp_batch_kernel(const BatchProblem * __restrict__ probs, int nprob, long long nitems,
                unsigned long long * __restrict__ counter)
{
  using L = Layout<BW, BH, float>;
  // No static shared variables here: they would shift the dynamic region and
  // break the 128-byte alignment TMA needs for its destination boxes.  The
  // base is aligned explicitly (the launch adds kBatchSmemExtra bytes).
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char * smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  StageHeader *   hdr = reinterpret_cast<StageHeader *>(smem + L::kHeaders);
  float *         boxes = reinterpret_cast<float *>(smem + L::kBoxes);
  uint64_t *      full = reinterpret_cast<uint64_t *>(smem + L::kBars);
  uint64_t *      empty = full + kStages;
  long long &     item_sh = *reinterpret_cast<long long *>(smem + L::kTotal);
  int &           abort_sh = *reinterpret_cast<int *>(smem + L::kTotal + 8);
  const int       warp = threadIdx.x >> 5;
  if (threadIdx.x == 0)
  {
    for (int s = 0; s < kStages; s++)
    {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kConsumerWarps);
    }
    fence_barrier_init();
    abort_sh = 0;
  }
  unsigned gbase = 0;
  for (;;)
  {
    __syncthreads();
    if (threadIdx.x == 0)
      item_sh = (long long)atomicAdd(counter, 1ULL);
    __syncthreads();
    const long long item = item_sh;
    if (item >= nitems || abort_sh)
      break;
    int lo = 0, hi = nprob - 1;
    while (lo < hi)
    {
      const int mid = (lo + hi + 1) >> 1;
      if (probs[mid].tile_begin <= item)
        lo = mid;
      else
        hi = mid - 1;
    }
    const BatchProblem & P = probs[lo];
    const long long      local = item - P.tile_begin;
    const int            tx = (int)(local % P.ntx), tz = (int)((local / P.ntx) % P.ntz),
               ty = (int)(local / ((long long)P.ntx * P.ntz));
    const int x0 = tx * kTX, y0 = ty * NYT, z0 = tz * kTZ;
    bool      ok;
    if (warp == kConsumerWarps)
      ok = bp_producer<BW, BH, NYT, float>(&P.tmap, P.proj, P.mats, P.nproj, P.nu, P.nv, x0, y0, z0, hdr, boxes, full,
                                           empty, P.use_tma, gbase);
    else
      ok = bp_consumer<BW, BH, NYT, FDKW, float>(P.proj, P.nproj, P.nu, P.nv, P.nx, P.ny, P.nz, x0, y0, z0, hdr, boxes,
                                                 full, empty, P.vin, P.vout, gbase);
    if (!ok)
      abort_sh = 1;
    gbase += (unsigned)P.nproj;
  }
}

// Generic path (any geometry): one thread per voxel, FP64 arithmetic, RTK's
// optimised-path bounds for modes 1/2 and itk::LinearInterpolateImageFunction
// semantics (clamp-to-edge, accepted range [-0.5, N-0.5)) for mode 0.
template <bool FDKW, typename T = float>
__global__ void __launch_bounds__(256)
bp_generic_kernel(const T * __restrict__ proj, const double * __restrict__ mats, const int * __restrict__ modes,
                  int nproj, int nu, int nv, int nx, int ny, int nz, const float * vol_in, float * vol_out)
{
  const long long n = (long long)nx * ny * nz;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x)
  {
    const int    X = (int)(idx % nx), Y = (int)((idx / nx) % ny), Z = (int)(idx / ((long long)nx * ny));
    const double x = X, y = Y, z = Z;
    double       acc = 0.;
    for (int p = 0; p < nproj; p++)
    {
      const double * M = mats + 12 * (long long)p;
      const double   w = __ldg(M + 8) * x + __ldg(M + 9) * y + __ldg(M + 10) * z + __ldg(M + 11);
      const double   rw = 1.0 / w;
      const double   u = (__ldg(M + 0) * x + __ldg(M + 1) * y + __ldg(M + 2) * z + __ldg(M + 3)) * rw;
      const double   v = (__ldg(M + 4) * x + __ldg(M + 5) * y + __ldg(M + 6) * z + __ldg(M + 7)) * rw;
      const T *      P = proj + (long long)p * nu * nv;
      const double   wt = FDKW ? rw * rw : 1.0;
      if (__ldg(modes + p))
      {
        if (u >= 0.0 && u < nu - 1.0 && v >= 0.0 && v < nv - 1.0)
        {
          const int     iu = (int)floor(u), iv = (int)floor(v);
          const double  fu = u - iu, fv = v - iv;
          const T *     q = P + (long long)iv * nu + iu;
          acc += wt * ((1 - fv) * ((1 - fu) * gtap(q) + fu * gtap(q + 1)) +
                       fv * ((1 - fu) * gtap(q + nu) + fu * gtap(q + nu + 1)));
        }
      }
      else if (u >= -0.5 && u < nu - 0.5 && v >= -0.5 && v < nv - 0.5)
      {
        const double uc = fmin(fmax(u, 0.0), nu - 1.0), vc = fmin(fmax(v, 0.0), nv - 1.0);
        const int    iu = (int)floor(uc), iv = (int)floor(vc);
        const int    iu1 = min(iu + 1, nu - 1), iv1 = min(iv + 1, nv - 1);
        const double fu = uc - iu, fv = vc - iv;
        const double a = (1 - fu) * gtap(P + (long long)iv * nu + iu) + fu * gtap(P + (long long)iv * nu + iu1);
        const double b = (1 - fu) * gtap(P + (long long)iv1 * nu + iu) + fu * gtap(P + (long long)iv1 * nu + iu1);
        acc += wt * ((1 - fv) * a + fv * b);
      }
    }
    vol_out[idx] = vol_in[idx] + (float)acc;
  }
}

struct BpConfig
{
  int bw, bh, nyt, minb;
};

// Candidate (box width, box height, voxels per thread column, CTAs per SM the
// register budget targets), in order of preference; the first whose box
// holds the probed footprints is used unless the autotuner forces one.
constexpr int           kNumBpConfigs = 6;
// Box rows are 16 (mod 32) words long: a warp covers 8 x 4 voxels, whose taps
// span at most ~16 columns, so when its lanes straddle two detector rows the
// second row's taps fall in the other half of the banks (rows 4 banks apart
// cost 25 % extra shared-memory wavefronts in conflicts).  16-voxel columns at
// 3 CTAs per SM with a 48-row box come first (fastest on 512^3 x 720); 24-voxel
// columns at 2 CTAs per SM amortise each column's set-up over more voxels;
// the rest hold taller and wider footprints.
static const BpConfig   kBpConfigs[kNumBpConfigs] = { { 80, 48, 16, 3 }, { 80, 72, 24, 2 }, { 80, 72, 16, 2 },
                                                      { 80, 32, 8, 3 }, { 112, 48, 8, 2 }, { 144, 64, 8, 1 } };
// BF16 boxes: widths are multiples of 8 elements (16-byte TMA rows); 96 and
// 160 elements are 48 and 80 words, again 16 (mod 32); same order as the FP32
// table.
static const BpConfig   kBpConfigsBf16[kNumBpConfigs] = { { 96, 48, 16, 3 }, { 96, 72, 24, 2 }, { 96, 72, 16, 2 },
                                                          { 96, 32, 8, 3 }, { 160, 48, 8, 2 }, { 160, 64, 8, 1 } };
static thread_local int g_bp_forced_config = -1;
static thread_local int g_bp_last_config = -1;

// Largest detector footprint of a 16 x NYT x 16 tile, probed on the tiles at
// the volume's corners (where magnification peaks) and its centre.
static void
estimate_footprint(const std::vector<double> & mats, int nproj, int nx, int ny, int nz, int nyt, double & fw,
                   double & fh)
{
  fw = 0.;
  fh = 0.;
  const int tiles_x[3] = { 0, std::max(0, (nx - 1) / kTX * kTX), std::max(0, (nx / 2) / kTX * kTX) };
  const int tiles_y[3] = { 0, std::max(0, (ny - 1) / nyt * nyt), std::max(0, (ny / 2) / nyt * nyt) };
  const int tiles_z[3] = { 0, std::max(0, (nz - 1) / kTZ * kTZ), std::max(0, (nz / 2) / kTZ * kTZ) };
  // footprints vary smoothly with the projection: probe about 64 of them
  // (the estimate only picks the box size; tiles that do not fit take the
  // FP64 path, so it never affects results)
  const int step = std::max(1, nproj / 64);
  for (int p = 0; p < nproj; p += step)
  {
    const double * m = mats.data() + 12 * p;
    for (int a = 0; a < 3; a++)
      for (int bq = 0; bq < 3; bq++)
        for (int cq = 0; cq < 3; cq++)
        {
          const int x0 = tiles_x[a], y0 = tiles_y[bq], z0 = tiles_z[cq];
          double    umin = 1e300, umax = -1e300, vmin = 1e300, vmax = -1e300;
          bool      ok = true;
          int       sign = 0;
          for (int c = 0; c < 8; c++)
          {
            const double X = (c & 1) ? x0 + kTX - 1 : x0;
            const double Y = (c & 2) ? y0 + nyt - 1 : y0;
            const double Z = (c & 4) ? z0 + kTZ - 1 : z0;
            const double w = m[8] * X + m[9] * Y + m[10] * Z + m[11];
            const int    sw = (w > 0.) ? 1 : ((w < 0.) ? -1 : 0);
            if (sw == 0 || (sign != 0 && sw != sign))
            {
              ok = false;
              break;
            }
            sign = sw;
            const double u = (m[0] * X + m[1] * Y + m[2] * Z + m[3]) / w;
            const double v = (m[4] * X + m[5] * Y + m[6] * Z + m[7]) / w;
            umin = std::min(umin, u);
            umax = std::max(umax, u);
            vmin = std::min(vmin, v);
            vmax = std::max(vmax, v);
          }
          if (ok)
          {
            fw = std::max(fw, umax - umin);
            fh = std::max(fh, vmax - vmin);
          }
        }
  }
}

// Tile schedule of the tiled kernel (rtkb_bp_set_schedule): 0 every tile
// walks the stack from projection 0 (deterministic sums); 1 the projection
// sweep, chunks of 2^g_bp_sweep_shift projections.
static int g_bp_schedule = 0;
static int g_bp_sweep_shift = 4;

template <int BW, int BH, int NYT, int MINB, bool FDKW, typename T>
static int
launch_tiled(const CUtensorMap & tmap, bool use_tma, const T * d_proj, const double * d_mats, int nproj, int nu,
             int nv, int nx, int ny, int nz, const float * vin, float * vout, unsigned * d_progress, cudaStream_t st)
{
  using L = Layout<BW, BH, T>;
  const int       ntx = (nx + kTX - 1) / kTX, nty = (ny + NYT - 1) / NYT, ntz = (nz + kTZ - 1) / kTZ;
  const long long nblocks = (long long)ntx * nty * ntz;
  if (nblocks > 0x7fffffffLL)
    return rtkb::fail(RTKB_ERR_UNSUPPORTED, "volume too large for one launch");
  if (g_bp_schedule == 1 && d_progress)
  {
    auto kern = bp_tiled_kernel<BW, BH, NYT, MINB, FDKW, T, true>;
    RTKB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L::kTotal));
    int dev = 0, sms = 0, per_sm = 0;
    RTKB_CUDA_TRY(cudaGetDevice(&dev));
    RTKB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    RTKB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, L::kTotal));
    const Sweep sw{ d_progress, (unsigned)std::max(1, sms * std::max(per_sm, 1)), (unsigned)g_bp_sweep_shift };
    RTKB_CUDA_TRY(cudaMemsetAsync(d_progress, 0, sizeof(unsigned), st));
    kern<<<(unsigned)nblocks, kThreads, L::kTotal, st>>>(tmap, d_proj, d_mats, nproj, nu, nv, nx, ny, nz, ntx, ntz,
                                                         vin, vout, use_tma ? 1 : 0, sw);
    RTKB_CUDA_TRY(cudaGetLastError());
    return RTKB_OK;
  }
  // launches of few projections per tile (the host-buffer path's subsets and
  // slabs) start their accumulators from the input volume; long ones keep the
  // read at the end (measured: starting from the input slowed a 720-projection
  // launch by 1.2 %)
  auto kern = nproj <= kInitFromInputMaxProjections ? bp_tiled_kernel<BW, BH, NYT, MINB, FDKW, T, false, true>
                                                    : bp_tiled_kernel<BW, BH, NYT, MINB, FDKW, T, false, false>;
  RTKB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L::kTotal));
  kern<<<(unsigned)nblocks, kThreads, L::kTotal, st>>>(tmap, d_proj, d_mats, nproj, nu, nv, nx, ny, nz, ntx, ntz, vin,
                                                       vout, use_tma ? 1 : 0, Sweep{ nullptr, 1u, 0u });
  RTKB_CUDA_TRY(cudaGetLastError());
  return RTKB_OK;
}

template <bool FDKW>
static int
dispatch_tiled(int cfg, const CUtensorMap & tmap, bool use_tma, const float * d_proj, const double * d_mats,
               int nproj, int nu, int nv, int nx, int ny, int nz, const float * vin, float * vout, unsigned * d_progress,
               cudaStream_t st)
{
#define RTKB_BP_LAUNCH(BW, BH, NYT, MINB)                                                                              \
  return launch_tiled<BW, BH, NYT, MINB, FDKW, float>(tmap, use_tma, d_proj, d_mats, nproj, nu, nv, nx, ny, nz, vin,   \
                                                      vout, d_progress, st)
  switch (cfg)
  {
    case 0:
      RTKB_BP_LAUNCH(80, 48, 16, 3);
    case 1:
      RTKB_BP_LAUNCH(80, 72, 24, 2);
    case 2:
      RTKB_BP_LAUNCH(80, 72, 16, 2);
    case 3:
      RTKB_BP_LAUNCH(80, 32, 8, 3);
    case 4:
      RTKB_BP_LAUNCH(112, 48, 8, 2);
    default:
      RTKB_BP_LAUNCH(144, 64, 8, 1);
  }
#undef RTKB_BP_LAUNCH
}

template <bool FDKW>
static int
dispatch_tiled(int cfg, const CUtensorMap & tmap, bool use_tma, const __nv_bfloat16 * d_proj, const double * d_mats,
               int nproj, int nu, int nv, int nx, int ny, int nz, const float * vin, float * vout, unsigned * d_progress,
               cudaStream_t st)
{
#define RTKB_BP_LAUNCH(BW, BH, NYT, MINB)                                                                              \
  return launch_tiled<BW, BH, NYT, MINB, FDKW, __nv_bfloat16>(tmap, use_tma, d_proj, d_mats, nproj, nu, nv, nx, ny, nz, \
                                                              vin, vout, d_progress, st)
  switch (cfg)
  {
    case 0:
      RTKB_BP_LAUNCH(96, 48, 16, 3);
    case 1:
      RTKB_BP_LAUNCH(96, 72, 24, 2);
    case 2:
      RTKB_BP_LAUNCH(96, 72, 16, 2);
    case 3:
      RTKB_BP_LAUNCH(96, 32, 8, 3);
    case 4:
      RTKB_BP_LAUNCH(160, 48, 8, 2);
    default:
      RTKB_BP_LAUNCH(160, 64, 8, 1);
  }
#undef RTKB_BP_LAUNCH
}

template <int BW, int BH, int NYT, int MINB, bool FDKW>
static int
launch_batch(const BatchProblem * d_probs, int nprob, long long nitems, unsigned long long * d_counter, cudaStream_t st)
{
  using L = Layout<BW, BH, float>;
  auto      kern = bp_batch_kernel<BW, BH, NYT, MINB, FDKW>;
  const int smem = L::kTotal + kBatchSmemExtra;
  RTKB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  int dev = 0, sms = 0, per_sm = 0;
  RTKB_CUDA_TRY(cudaGetDevice(&dev));
  RTKB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  RTKB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem));
  const long long grid = std::max<long long>(1, std::min<long long>(nitems, (long long)sms * std::max(per_sm, 1)));
  kern<<<(unsigned)grid, kThreads, smem, st>>>(d_probs, nprob, nitems, d_counter);
  RTKB_CUDA_TRY(cudaGetLastError());
  return RTKB_OK;
}

template <bool FDKW>
static int
dispatch_batch(int cfg, const BatchProblem * d_probs, int nprob, long long nitems, unsigned long long * d_counter,
               cudaStream_t st)
{
  switch (cfg)
  {
    case 0:
      return launch_batch<80, 48, 16, 3, FDKW>(d_probs, nprob, nitems, d_counter, st);
    case 1:
      return launch_batch<80, 72, 24, 2, FDKW>(d_probs, nprob, nitems, d_counter, st);
    case 2:
      return launch_batch<80, 72, 16, 2, FDKW>(d_probs, nprob, nitems, d_counter, st);
    case 3:
      return launch_batch<80, 32, 8, 3, FDKW>(d_probs, nprob, nitems, d_counter, st);
    case 4:
      return launch_batch<112, 48, 8, 2, FDKW>(d_probs, nprob, nitems, d_counter, st);
    default:
      return launch_batch<144, 64, 8, 1, FDKW>(d_probs, nprob, nitems, d_counter, st);
  }
}

// FP32 -> BF16 (round to nearest even), two elements per thread
__global__ void __launch_bounds__(256)
to_bf16_kernel(const float * __restrict__ in, __nv_bfloat16 * __restrict__ out, long long n)
{
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16_rn(in[i]);
}

} // namespace

namespace rtkb
{

// Converts RTK index-to-index matrices (absolute indices) to buffer
// coordinates and applies the optimised-path simplifications.
void
to_buffer_matrix(const rtkb_image_desc & vol, const rtkb_image_desc & proj, int mode, const double * in, double * out)
{
  double m[12];
  std::memcpy(m, in, sizeof(m));
  // volume buffer index -> absolute index: column 3 += M[:, 0..2] . index
  for (int r = 0; r < 3; r++)
    m[r * 4 + 3] += m[r * 4 + 0] * vol.index[0] + m[r * 4 + 1] * vol.index[1] + m[r * 4 + 2] * vol.index[2];
  // projection absolute index -> buffer index: u -= index0, v -= index1 (after the division)
  for (int c = 0; c < 4; c++)
  {
    m[0 * 4 + c] -= proj.index[0] * m[8 + c];
    m[1 * 4 + c] -= proj.index[1] * m[8 + c];
  }
  // RTK's optimised paths ignore the (< 1e-10) coefficients that select them
  if (mode == 1)
  {
    m[0] = 0.;
    m[8] = 0.;
  }
  else if (mode == 2)
  {
    m[1] = 0.;
    m[9] = 0.;
  }
  std::memcpy(out, m, sizeof(m));
}

// Host half of a backprojection: argument checks, RTK's path per projection
// (the tiled kernel needs optimised-Y everywhere), the tile configuration from
// footprints probed on the host, and the TMA descriptor of the stack.  No
// device work: the launch half (bp_launch) can run later, and inside a stream
// capture, as long as d_proj keeps its address.
template <typename T>
int
bp_prepare(const int vol_size[3], const int proj_size[3], int nproj, const double * mats, const int * modes, bool fdk,
           const T * d_proj, BpPrepared & out)
{
  constexpr bool    kBf16 = sizeof(T) == 2;
  const BpConfig *  configs = kBf16 ? kBpConfigsBf16 : kBpConfigs;
  constexpr double  kSlack = kAlignElems<T> - 1 + 0.2; // box origin rounding + margins
  const int nx = vol_size[0], ny = vol_size[1], nz = vol_size[2];
  const int nu = proj_size[0], nv = proj_size[1];
  if (nx <= 0 || ny <= 0 || nz <= 0 || nu <= 0 || nv <= 0 || nproj < 0 || proj_size[2] < nproj)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "invalid sizes");
  if (nproj > 0 && (!d_proj || !mats || !modes))
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null buffer");
  out = BpPrepared{};
  out.nproj = nproj;
  out.nu = nu;
  out.nv = nv;
  out.np_total = proj_size[2];
  out.nx = nx;
  out.ny = ny;
  out.nz = nz;
  out.fdk = fdk;
  bool all_opt_y = true;
  for (int p = 0; p < nproj; p++)
  {
    for (int q = 0; q < 12; q++)
      if (!std::isfinite(mats[12 * p + q]))
        return fail(RTKB_ERR_INVALID_ARGUMENT, "non-finite projection matrix");
    if (modes[p] != 2)
      all_opt_y = false;
  }
  if (nproj == 0)
    return RTKB_OK;
  if (!all_opt_y)
  {
    out.generic = true;
    return RTKB_OK;
  }
  // first configuration whose box holds the footprints probed on the host
  std::vector<double> mv(mats, mats + 12 * (size_t)nproj);
  double              fw[3], fh[3]; // columns of 8, 16, 24 voxels
  for (int q = 0; q < 3; q++)
    estimate_footprint(mv, nproj, nx, ny, nz, 8 * (q + 1), fw[q], fh[q]);
  int cfg = kNumBpConfigs - 1;
  for (int c = 0; c < kNumBpConfigs; c++)
  {
    const int q = configs[c].nyt / 8 - 1;
    if (fw[q] + kSlack < configs[c].bw - 1 && fh[q] + 0.2 < configs[c].bh - 1)
    {
      cfg = c;
      break;
    }
  }
  if (g_bp_forced_config >= 0)
    cfg = g_bp_forced_config; // a box too small for some tiles only sends them to the FP64 path
  g_bp_last_config = cfg;
  out.cfg = cfg;
  // TMA needs 16-byte aligned rows and base address
  std::memset(&out.tmap, 0, sizeof(out.tmap));
  EncodeTiledFn            enc = tensor_map_encoder();
  const long long          np_total = proj_size[2];
  const unsigned long long esz = sizeof(T);
  if (enc && ((unsigned long long)nu * esz) % 16 == 0 && (reinterpret_cast<uintptr_t>(d_proj) % 16) == 0 &&
      np_total <= 0x7fffffffLL)
  {
    const unsigned long long dims[3] = { (unsigned long long)nu, (unsigned long long)nv, (unsigned long long)np_total };
    const unsigned long long strides[2] = { (unsigned long long)nu * esz, (unsigned long long)nu * nv * esz };
    const unsigned           box[3] = { (unsigned)configs[cfg].bw, (unsigned)configs[cfg].bh, 1u };
    const unsigned           estr[3] = { 1u, 1u, 1u };
    const int r = enc(&out.tmap, kBf16 ? (int)CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : (int)CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                      3u, const_cast<T *>(d_proj), dims, strides, box, estr, (int)CU_TENSOR_MAP_INTERLEAVE_NONE,
                      (int)CU_TENSOR_MAP_SWIZZLE_NONE, (int)CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                      (int)CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    out.use_tma = (r == 0);
  }
  return RTKB_OK;
}

// Device half: d_vout = d_vin + BP(d_proj) with the matrices and modes already
// in device memory (d_vin may equal d_vout).  Stream-ordered launches only.
template <typename T>
int
bp_launch(const BpPrepared & b, const T * d_proj, const double * d_mats, const int * d_modes, const float * d_vin,
          float * d_vout, cudaStream_t st, unsigned * d_progress = nullptr)
{
  const long long nvox = (long long)b.nx * b.ny * b.nz;
  if (b.nproj == 0)
  {
    if (d_vout != d_vin)
      RTKB_CUDA_TRY(cudaMemcpyAsync(d_vout, d_vin, nvox * sizeof(float), cudaMemcpyDeviceToDevice, st));
    return RTKB_OK;
  }
  if (b.generic)
  {
    const long long blocks = std::min<long long>((nvox + 255) / 256, 148LL * 64);
    if (b.fdk)
      bp_generic_kernel<true, T><<<(unsigned)blocks, 256, 0, st>>>(d_proj, d_mats, d_modes, b.nproj, b.nu, b.nv, b.nx,
                                                                   b.ny, b.nz, d_vin, d_vout);
    else
      bp_generic_kernel<false, T><<<(unsigned)blocks, 256, 0, st>>>(d_proj, d_mats, d_modes, b.nproj, b.nu, b.nv, b.nx,
                                                                    b.ny, b.nz, d_vin, d_vout);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? RTKB_OK : cuda_fail(e, "bp_generic_kernel launch");
  }
  return b.fdk ? dispatch_tiled<true>(b.cfg, b.tmap, b.use_tma, d_proj, d_mats, b.nproj, b.nu, b.nv, b.nx, b.ny, b.nz,
                                      d_vin, d_vout, d_progress, st)
               : dispatch_tiled<false>(b.cfg, b.tmap, b.use_tma, d_proj, d_mats, b.nproj, b.nu, b.nv, b.nx, b.ny, b.nz,
                                       d_vin, d_vout, d_progress, st);
}

template <typename T>
int
backproject_buffer(const int vol_size[3], const int proj_size[3], int nproj, const double * mats, const int * modes,
                   bool fdk, const T * d_proj, const float * d_vin, float * d_vout, cudaStream_t st,
                   void * fixed_scratch = nullptr)
{
  if (!d_vin || !d_vout)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null buffer");
  BpPrepared b;
  int        rc = bp_prepare(vol_size, proj_size, nproj, mats, modes, fdk, d_proj, b);
  if (rc != RTKB_OK || nproj == 0)
    return rc != RTKB_OK ? rc : bp_launch<T>(b, d_proj, nullptr, nullptr, d_vin, d_vout, st);
  // matrices, modes and the sweep counter in one scratch block: the caller's
  // when given, else a stream-ordered allocation
  const size_t mbytes = sizeof(double) * 12 * (size_t)nproj;
  void *       scratch = fixed_scratch;
  if (!scratch)
    RTKB_CUDA_TRY(rtkb::scratch_malloc(&scratch, mbytes + sizeof(int) * nproj + kProgressBytes, st));
  double *    d_mats = static_cast<double *>(scratch);
  int *       d_modes = reinterpret_cast<int *>(static_cast<char *>(scratch) + mbytes);
  unsigned *  d_progress = reinterpret_cast<unsigned *>(d_modes + nproj);
  cudaError_t e = cudaMemcpyAsync(d_mats, mats, mbytes, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_modes, modes, sizeof(int) * nproj, cudaMemcpyHostToDevice, st);
  rc = e == cudaSuccess ? bp_launch<T>(b, d_proj, d_mats, d_modes, d_vin, d_vout, st, d_progress)
                        : cuda_fail(e, "cudaMemcpyAsync");
  if (!fixed_scratch)
  {
    cudaError_t fe = rtkb::scratch_free(scratch, st);
    if (rc == RTKB_OK && fe != cudaSuccess)
      rc = cuda_fail(fe, "cudaFreeAsync");
  }
  return rc;
}

// The voxel-based back projector as a reusable object (the CG plan's
// BP_VOXELBASED choice): matrices and modes uploaded once at creation into
// device memory the caller owns, launches replayable inside a CUDA graph.
size_t
voxel_backprojector_bytes(int nproj)
{
  return ((sizeof(double) * 12 + sizeof(int)) * (size_t)std::max(nproj, 1) + kProgressBytes + 255) & ~size_t(255);
}

int
voxel_backprojector_create(const rtkb_geometry * g, const rtkb_image_desc & vol, const rtkb_image_desc & proj,
                           const float * d_proj, void * d_mem, VoxelBackprojector & out)
{
  if (g->g.radius_cylindrical != 0.)
    return fail(RTKB_ERR_UNSUPPORTED, "the reusable voxel-based back projector models flat panels only");
  const int           nproj = proj.size[2];
  std::vector<double> mats(12 * (size_t)std::max(nproj, 1));
  std::vector<int>    modes(std::max(nproj, 1));
  for (int s = 0; s < nproj; s++)
  {
    double m[12];
    modes[s] = bp_matrix(g->g, vol, proj, proj.index[2] + s, false, m);
    to_buffer_matrix(vol, proj, modes[s], m, mats.data() + 12 * s);
  }
  int rc = bp_prepare<float>(vol.size, proj.size, nproj, mats.data(), modes.data(), false, d_proj, out.prep);
  if (rc != RTKB_OK)
    return rc;
  out.d_proj = d_proj;
  out.d_mats = static_cast<double *>(d_mem);
  out.d_modes = reinterpret_cast<int *>(static_cast<char *>(d_mem) + sizeof(double) * 12 * (size_t)std::max(nproj, 1));
  out.d_progress = reinterpret_cast<unsigned *>(out.d_modes + std::max(nproj, 1));
  RTKB_CUDA_TRY(cudaMemcpy(out.d_mats, mats.data(), sizeof(double) * mats.size(), cudaMemcpyHostToDevice));
  RTKB_CUDA_TRY(cudaMemcpy(out.d_modes, modes.data(), sizeof(int) * modes.size(), cudaMemcpyHostToDevice));
  return RTKB_OK;
}

int
voxel_backprojector_launch(const VoxelBackprojector & b, const float * d_vin, float * d_vout, cudaStream_t st)
{
  return bp_launch<float>(b.prep, b.d_proj, b.d_mats, b.d_modes, d_vin, d_vout, st, b.d_progress);
}

template <typename T>
static int
backproject_geometry(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                     const T * d_proj, const float * d_vin, float * d_vout, void * stream, bool fdk,
                     void * fixed_scratch = nullptr)
{
  std::string why;
  if (!g)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "Geometry has not been set.");
  if (!desc_valid(vol, why) || !desc_valid(proj, why))
    return fail(RTKB_ERR_INVALID_ARGUMENT, why);
  const int nproj = proj->size[2];
  if (proj->index[2] < 0 || (long long)proj->index[2] + nproj > (long long)g->g.p.size())
    return fail(RTKB_ERR_INVALID_ARGUMENT, "Mismatch between the number of projections and the geometry entries.");
  if (g->g.radius_cylindrical != 0.)
  {
    // RTK's FDK back projector refuses cylindrical detectors; its voxel-based
    // one handles a cylinder centred on the source (float stacks here)
    if (fdk || fixed_scratch)
      return fail(RTKB_ERR_UNSUPPORTED,
                  "Voxel-based FDK back projector can currently not handle cylindrical detectors");
    if constexpr (!std::is_same<T, float>::value)
      return fail(RTKB_ERR_UNSUPPORTED, "cylindrical detectors need a float32 projection stack");
    else
      return cylindrical_backproject(g, *vol, *proj, d_proj, d_vin, d_vout, static_cast<cudaStream_t>(stream));
  }
  std::vector<double> mats(12 * (size_t)nproj);
  std::vector<int>    modes(nproj);
  for (int s = 0; s < nproj; s++)
  {
    double m[12];
    modes[s] = bp_matrix(g->g, *vol, *proj, proj->index[2] + s, fdk, m);
    to_buffer_matrix(*vol, *proj, modes[s], m, mats.data() + 12 * s);
  }
  return backproject_buffer(vol->size, proj->size, nproj, mats.data(), modes.data(), fdk, d_proj, d_vin, d_vout,
                            static_cast<cudaStream_t>(stream), fixed_scratch);
}

} // namespace rtkb

// A prepared batch: device tables (problem descriptors with their TMA maps,
// matrices, work counter) built once on the host; executing it is one
// counter reset and one persistent launch (plus separate launches for the
// problems on RTK's generic path).
struct rtkb_bp_batch
{
  bool                       fdk = true;
  int                        cfg = 0;
  int                        nbatch = 0;
  long long                  items = 0;
  void *                     mem = nullptr;
  rtkb::BatchProblemHandle * probs = nullptr; // device array (opaque on the host side)
  unsigned long long *       counter = nullptr;
  struct Generic
  {
    rtkb_bp_problem     p;
    std::vector<double> mats;
    std::vector<int>    modes;
  };
  std::vector<Generic> generic;
};

namespace rtkb
{

static void
release_batch(rtkb_bp_batch * b)
{
  if (!b)
    return;
  if (b->mem)
    cudaFree(b->mem);
  delete b;
}

static int
create_batch(const rtkb_bp_problem * probs, int n, bool fdk, int cfg, rtkb_bp_batch ** out)
{
  if (!out)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null batch pointer");
  *out = nullptr;
  if (n < 0 || (n > 0 && !probs))
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null problem list");
  if (cfg >= kNumBpConfigs)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "configuration out of range");
  rtkb_bp_batch * B = new rtkb_bp_batch();
  B->fdk = fdk;
  struct Host
  {
    int                 idx;
    std::vector<double> mats;
  };
  std::vector<Host> batch;
  double            fw[3] = { 0., 0., 0. }, fh[3] = { 0., 0., 0. }; // columns of 8, 16, 24 voxels
  for (int i = 0; i < n; i++)
  {
    const rtkb_bp_problem & P = probs[i];
    std::string             why;
    int                     rc = RTKB_OK;
    if (!P.geometry)
      rc = fail(RTKB_ERR_INVALID_ARGUMENT, "Geometry has not been set.");
    else if (!desc_valid(&P.vol, why) || !desc_valid(&P.proj, why))
      rc = fail(RTKB_ERR_INVALID_ARGUMENT, why);
    else if (P.geometry->g.radius_cylindrical != 0.)
      rc = fail(RTKB_ERR_UNSUPPORTED, "Voxel-based FDK back projector can currently not handle cylindrical detectors");
    else if (P.proj.index[2] < 0 || (long long)P.proj.index[2] + P.proj.size[2] > (long long)P.geometry->g.p.size())
      rc = fail(RTKB_ERR_INVALID_ARGUMENT, "Mismatch between the number of projections and the geometry entries.");
    else if (!P.d_vol_in || !P.d_vol_out || (P.proj.size[2] > 0 && !P.d_proj))
      rc = fail(RTKB_ERR_INVALID_ARGUMENT, "null buffer");
    if (rc != RTKB_OK)
    {
      release_batch(B);
      return rc;
    }
    const int           np = P.proj.size[2];
    std::vector<double> mats(12 * (size_t)np);
    std::vector<int>    modes(np);
    bool                opt_y = true;
    for (int sidx = 0; sidx < np; sidx++)
    {
      double m[12];
      modes[sidx] = bp_matrix(P.geometry->g, P.vol, P.proj, P.proj.index[2] + sidx, fdk, m);
      to_buffer_matrix(P.vol, P.proj, modes[sidx], m, mats.data() + 12 * sidx);
      for (int q = 0; q < 12; q++)
        if (!std::isfinite(mats[12 * sidx + q]))
        {
          release_batch(B);
          return fail(RTKB_ERR_INVALID_ARGUMENT, "non-finite projection matrix");
        }
      opt_y = opt_y && modes[sidx] == 2;
    }
    if (!opt_y || np == 0)
    {
      B->generic.push_back(rtkb_bp_batch::Generic{ P, std::move(mats), std::move(modes) });
      continue;
    }
    for (int q = 0; q < 3; q++)
    {
      double a, b;
      estimate_footprint(mats, np, P.vol.size[0], P.vol.size[1], P.vol.size[2], 8 * (q + 1), a, b);
      fw[q] = std::max(fw[q], a);
      fh[q] = std::max(fh[q], b);
    }
    batch.push_back(Host{ i, std::move(mats) });
  }
  if (cfg < 0)
  {
    cfg = kNumBpConfigs - 1;
    for (int c = 0; c < kNumBpConfigs; c++)
    {
      const int q = kBpConfigs[c].nyt / 8 - 1;
      if (fw[q] + 3.2 < kBpConfigs[c].bw - 1 && fh[q] + 0.2 < kBpConfigs[c].bh - 1)
      {
        cfg = c;
        break;
      }
    }
  }
  B->cfg = cfg;
  B->nbatch = (int)batch.size();
  if (batch.empty())
  {
    *out = B;
    return RTKB_OK;
  }
  const BpConfig            C = kBpConfigs[cfg];
  std::vector<BatchProblem> hp(batch.size());
  size_t                    nmats = 0;
  for (const Host & h : batch)
    nmats += h.mats.size();
  const size_t pbytes = (hp.size() * sizeof(BatchProblem) + 255) & ~size_t(255);
  const size_t mbytes = (nmats * sizeof(double) + 255) & ~size_t(255);
  cudaError_t  e = cudaMalloc(&B->mem, pbytes + mbytes + 256);
  if (e != cudaSuccess)
  {
    release_batch(B);
    return cuda_fail(e, "cudaMalloc (batch tables)");
  }
  BatchProblem * d_probs = static_cast<BatchProblem *>(B->mem);
  double *       d_mats = reinterpret_cast<double *>(static_cast<char *>(B->mem) + pbytes);
  B->probs = reinterpret_cast<BatchProblemHandle *>(d_probs);
  B->counter = reinterpret_cast<unsigned long long *>(static_cast<char *>(B->mem) + pbytes + mbytes);
  std::vector<double> allm;
  allm.reserve(nmats);
  long long     items = 0;
  EncodeTiledFn enc = tensor_map_encoder();
  for (size_t k = 0; k < batch.size(); k++)
  {
    const rtkb_bp_problem & P = probs[batch[k].idx];
    BatchProblem &          Q = hp[k];
    std::memset(&Q, 0, sizeof(Q));
    Q.proj = P.d_proj;
    Q.mats = d_mats + allm.size();
    allm.insert(allm.end(), batch[k].mats.begin(), batch[k].mats.end());
    Q.vin = P.d_vol_in;
    Q.vout = P.d_vol_out;
    Q.nproj = P.proj.size[2];
    Q.nu = P.proj.size[0];
    Q.nv = P.proj.size[1];
    Q.nx = P.vol.size[0];
    Q.ny = P.vol.size[1];
    Q.nz = P.vol.size[2];
    Q.ntx = (Q.nx + kTX - 1) / kTX;
    Q.ntz = (Q.nz + kTZ - 1) / kTZ;
    const int nty = (Q.ny + C.nyt - 1) / C.nyt;
    Q.tile_begin = items;
    items += (long long)Q.ntx * nty * Q.ntz;
    Q.use_tma = 0;
    if (enc && (Q.nu % 4) == 0 && (reinterpret_cast<uintptr_t>(P.d_proj) % 16) == 0)
    {
      const unsigned long long dims[3] = { (unsigned long long)Q.nu, (unsigned long long)Q.nv,
                                           (unsigned long long)Q.nproj };
      const unsigned long long strides[2] = { (unsigned long long)Q.nu * 4ULL, (unsigned long long)Q.nu * Q.nv * 4ULL };
      const unsigned           box[3] = { (unsigned)C.bw, (unsigned)C.bh, 1u };
      const unsigned           estr[3] = { 1u, 1u, 1u };
      const int r = enc(&Q.tmap, (int)CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3u, const_cast<float *>(P.d_proj), dims, strides,
                        box, estr, (int)CU_TENSOR_MAP_INTERLEAVE_NONE, (int)CU_TENSOR_MAP_SWIZZLE_NONE,
                        (int)CU_TENSOR_MAP_L2_PROMOTION_L2_128B, (int)CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      Q.use_tma = (r == 0) ? 1 : 0;
    }
  }
  B->items = items;
  e = cudaMemcpy(d_probs, hp.data(), hp.size() * sizeof(BatchProblem), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(d_mats, allm.data(), allm.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess)
  {
    release_batch(B);
    return cuda_fail(e, "batch upload");
  }
  *out = B;
  return RTKB_OK;
}

static int
execute_batch(rtkb_bp_batch * B, cudaStream_t st)
{
  if (!B)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null batch");
  for (rtkb_bp_batch::Generic & G : B->generic)
  {
    const int rc = backproject_buffer(G.p.vol.size, G.p.proj.size, G.p.proj.size[2], G.mats.data(), G.modes.data(),
                                      B->fdk, G.p.d_proj, G.p.d_vol_in, G.p.d_vol_out, st);
    if (rc != RTKB_OK)
      return rc;
  }
  if (B->nbatch == 0)
    return RTKB_OK;
  RTKB_CUDA_TRY(cudaMemsetAsync(B->counter, 0, sizeof(unsigned long long), st));
  const BatchProblem * d_probs = reinterpret_cast<const BatchProblem *>(B->probs);
  return B->fdk ? dispatch_batch<true>(B->cfg, d_probs, B->nbatch, B->items, B->counter, st)
                : dispatch_batch<false>(B->cfg, d_probs, B->nbatch, B->items, B->counter, st);
}

static int
backproject_batch(const rtkb_bp_problem * probs, int n, bool fdk, int cfg, int * used_config, cudaStream_t st)
{
  rtkb_bp_batch * B = nullptr;
  int             rc = create_batch(probs, n, fdk, cfg, &B);
  if (rc != RTKB_OK)
    return rc;
  if (used_config)
    *used_config = B->cfg;
  rc = execute_batch(B, st);
  // the tables are freed only once the launch that reads them has finished
  const cudaError_t e = cudaStreamSynchronize(st);
  if (rc == RTKB_OK && e != cudaSuccess)
    rc = cuda_fail(e, "batch backprojection");
  release_batch(B);
  return rc;
}

} // namespace rtkb

extern "C" int
rtkb_fdk_backproject(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                     const float * d_proj, const float * d_vol_in, float * d_vol_out, void * stream)
{
  RTKB_TRACE();
  try
  {
    return rtkb::backproject_geometry(g, vol, proj, d_proj, d_vol_in, d_vol_out, stream, true);
  }
  catch (...)
  {
    return rtkb::fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

// Host-buffer FDK backprojection: the stack streams through two device
// staging buffers in chunks (RTK's projection subsets,
// include/rtkFDKConeBeamReconstructionFilter.hxx:116-157), each copied on an
// internal stream while the previous chunk is backprojected in place into a
// device copy of the volume on the caller's stream; the last chunk runs slab
// by slab in z, each slab copied back while the next is backprojected.
namespace rtkb
{
static int
fdk_backproject_host(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                     const float * h_proj, const float * h_vol_in, float * h_vol_out, int chunk, cudaStream_t st)
{
  std::string why;
  if (!g)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "Geometry has not been set.");
  if (!desc_valid(vol, why) || !desc_valid(proj, why))
    return fail(RTKB_ERR_INVALID_ARGUMENT, why);
  const int       nproj = proj->size[2];
  const long long per = (long long)proj->size[0] * proj->size[1];
  const long long slice = (long long)vol->size[0] * vol->size[1];
  const int       nz = vol->size[2];
  const long long nvox = slice * nz;
  if (!h_vol_out || (nproj > 0 && !h_proj))
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null buffer");
  if (proj->index[2] < 0 || (long long)proj->index[2] + nproj > (long long)g->g.p.size())
    return fail(RTKB_ERR_INVALID_ARGUMENT, "Mismatch between the number of projections and the geometry entries.");
  if (chunk <= 0)
    chunk = std::max(1, (nproj + 3) / 4);
  chunk = std::max(1, std::min(chunk, std::max(nproj, 1)));
  // Subsets: the first one's copy is the only one nothing overlaps, so it is
  // short (chunk / 12); each next one is 1.5x the previous (a copy at ~50 GB/s
  // takes ~0.7x the time of backprojecting the same projections, so it hides
  // behind the previous subset) up to `chunk`; the last takes the remainder, up
  // to 1.5 chunk, long enough for its slabs' backprojections to hide the
  // volume's copy back.  bounds[k] .. bounds[k + 1] is subset k.
  std::vector<int> bounds{ 0 };
  for (int s = std::max(1, chunk / 12); nproj > 0;)
  {
    const int done = bounds.back(), rem = nproj - done;
    if ((long long)rem * 2 <= 3LL * chunk)
    {
      bounds.push_back(nproj);
      break;
    }
    bounds.push_back(done + std::min(s, chunk));
    s = std::min(chunk, (int)std::ceil(std::min(s, chunk) * 1.5));
  }
  const int nchunks = (int)bounds.size() - 1;
  auto      start = [&](int k) { return bounds[std::min(k, nchunks)]; };
  int       maxchunk = 0;
  for (int k = 0; k < nchunks; k++)
    maxchunk = std::max(maxchunk, start(k + 1) - start(k));
  // The last subset runs as z-slabs of whole 16-slice tile layers, each slab
  // copied back while the next ones are backprojected.  Slab sizes halve (16,
  // 8, 4, 2, 1, 1 layers of 32): a slab's copy (~0.3 ms per 512^2 x 16 layer)
  // hides behind the next slab's backprojection (~0.7 ms per layer for ~230
  // projections), most tiles run in large launches whose last wave is nearly
  // full, and only the last, one-layer slab's copy is exposed.
  constexpr int kSlabs = 16;
  int           zb[kSlabs + 1];
  int           nslab = 0;
  zb[0] = 0;
  {
    const int layers = (nz + 15) / 16;
    int       done = 0;
    while (done < layers && nslab < kSlabs)
    {
      const int rem = layers - done;
      int       take = rem <= 2 ? 1 : rem / 2; // the last two layers as two one-layer slabs
      if (nslab == kSlabs - 1)
        take = rem; // the last slot takes the rest
      done += take;
      zb[++nslab] = std::min(nz, 16 * done);
    }
  }
  if (nchunks == 0)
    nslab = 1, zb[1] = nz;
  const size_t vbytes = ((size_t)nvox * sizeof(float) + 255) / 256 * 256;
  const size_t sbytes = ((size_t)maxchunk * per * sizeof(float) + 255) / 256 * 256;
  const int    nstage = std::min(nchunks, 2);
  constexpr int kEvents = 6 + kSlabs; // allocation, chunk copied (2), stage free (2), copies done, slab done
  cudaStream_t  cs = nullptr;
  cudaEvent_t   ev[kEvents] = {};
  void *        mem = nullptr;
  int           rc = RTKB_OK;
  RTKB_CUDA_TRY(rtkb::scratch_malloc(&mem, vbytes + nstage * sbytes, st));
  do
  {
    cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    for (int i = 0; i < kEvents && e == cudaSuccess; i++)
      e = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming);
    if (e != cudaSuccess)
    {
      rc = cuda_fail(e, "stream/event creation");
      break;
    }
    float * d_vol = static_cast<float *>(mem);
    float * stage[2] = { reinterpret_cast<float *>(static_cast<char *>(mem) + vbytes),
                         reinterpret_cast<float *>(static_cast<char *>(mem) + vbytes + sbytes) };
    // the copy stream may touch the allocation once the caller's stream has
    // made it (stream-ordered allocation)
    e = cudaEventRecord(ev[0], st);
    if (e == cudaSuccess)
      e = cudaStreamWaitEvent(cs, ev[0], 0);
    if (e == cudaSuccess)
      e = h_vol_in ? cudaMemcpyAsync(d_vol, h_vol_in, (size_t)nvox * sizeof(float), cudaMemcpyHostToDevice, st)
                   : cudaMemsetAsync(d_vol, 0, (size_t)nvox * sizeof(float), st);
    if (e != cudaSuccess)
    {
      rc = cuda_fail(e, "volume initialisation");
      break;
    }
    for (int k = 0; k < nchunks && rc == RTKB_OK; k++)
    {
      const int b = k & 1;
      const int first = start(k), nk = start(k + 1) - first;
      if (k >= 2)
        e = cudaStreamWaitEvent(cs, ev[3 + b], 0); // the backprojection of chunk k-2 is done with stage b
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(stage[b], h_proj + (size_t)first * per, (size_t)nk * per * sizeof(float),
                            cudaMemcpyHostToDevice, cs);
      if (e == cudaSuccess)
        e = cudaEventRecord(ev[1 + b], cs);
      if (e == cudaSuccess)
        e = cudaStreamWaitEvent(st, ev[1 + b], 0);
      if (e != cudaSuccess)
      {
        rc = cuda_fail(e, "chunk copy");
        break;
      }
      rtkb_image_desc sub = *proj;
      sub.size[2] = nk;
      sub.index[2] = proj->index[2] + first;
      if (k < nchunks - 1)
      {
        rc = backproject_geometry(g, vol, &sub, static_cast<const float *>(stage[b]), d_vol, d_vol, st, true);
        if (rc == RTKB_OK && (e = cudaEventRecord(ev[3 + b], st)) != cudaSuccess)
          rc = cuda_fail(e, "cudaEventRecord");
        continue;
      }
      for (int q = 0; q < nslab && rc == RTKB_OK; q++)
      {
        // slab q of the volume: a region with its z index offset, as RTK
        // backprojects a requested region
        rtkb_image_desc vs = *vol;
        vs.size[2] = zb[q + 1] - zb[q];
        vs.index[2] = vol->index[2] + zb[q];
        float * d_slab = d_vol + (size_t)zb[q] * slice;
        rc = backproject_geometry(g, &vs, &sub, static_cast<const float *>(stage[b]), d_slab, d_slab, st, true);
        if (rc != RTKB_OK)
          break;
        e = cudaEventRecord(ev[6 + q], st);
        if (e == cudaSuccess)
          e = cudaStreamWaitEvent(cs, ev[6 + q], 0);
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(h_vol_out + (size_t)zb[q] * slice, d_slab, (size_t)vs.size[2] * slice * sizeof(float),
                              cudaMemcpyDeviceToHost, cs);
        if (e != cudaSuccess)
          rc = cuda_fail(e, "slab copy");
      }
    }
    if (rc != RTKB_OK)
      break;
    if (nchunks == 0)
      e = cudaMemcpyAsync(h_vol_out, d_vol, (size_t)nvox * sizeof(float), cudaMemcpyDeviceToHost, st);
    else
    {
      // the caller's stream completes after the last slab's copy
      e = cudaEventRecord(ev[5], cs);
      if (e == cudaSuccess)
        e = cudaStreamWaitEvent(st, ev[5], 0);
    }
    if (e != cudaSuccess)
      rc = cuda_fail(e, "volume copy");
  } while (0);
  if (rc != RTKB_OK && cs)
  {
    // join whatever the copy stream has enqueued before the buffers are freed
    if (cudaEventRecord(ev[5], cs) == cudaSuccess)
      cudaStreamWaitEvent(st, ev[5], 0);
  }
  // events and the copy stream are released once their work completes
  for (int i = 0; i < kEvents; i++)
    if (ev[i])
      cudaEventDestroy(ev[i]);
  if (cs)
    cudaStreamDestroy(cs);
  cudaError_t fe = rtkb::scratch_free(mem, st);
  if (rc == RTKB_OK && fe != cudaSuccess)
    rc = cuda_fail(fe, "cudaFreeAsync");
  return rc;
}
} // namespace rtkb

extern "C" int
rtkb_fdk_backproject_host(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                          const float * h_proj, const float * h_vol_in, float * h_vol_out, int chunk, void * stream)
{
  RTKB_TRACE();
  try
  {
    return rtkb::fdk_backproject_host(g, vol, proj, h_proj, h_vol_in, h_vol_out, chunk,
                                      static_cast<cudaStream_t>(stream));
  }
  catch (...)
  {
    return rtkb::fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

extern "C" int
rtkb_voxel_backproject(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                       const float * d_proj, const float * d_vol_in, float * d_vol_out, void * stream)
{
  RTKB_TRACE();
  try
  {
    return rtkb::backproject_geometry(g, vol, proj, d_proj, d_vol_in, d_vol_out, stream, false);
  }
  catch (...)
  {
    return rtkb::fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

extern "C" int
rtkb_fdk_backproject_bf16(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                          const void * d_proj_bf16, const float * d_vol_in, float * d_vol_out, void * stream)
{
  RTKB_TRACE();
  try
  {
    return rtkb::backproject_geometry(g, vol, proj, static_cast<const __nv_bfloat16 *>(d_proj_bf16), d_vol_in,
                                      d_vol_out, stream, true);
  }
  catch (...)
  {
    return rtkb::fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

extern "C" int
rtkb_voxel_backproject_bf16(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                            const void * d_proj_bf16, const float * d_vol_in, float * d_vol_out, void * stream)
{
  RTKB_TRACE();
  try
  {
    return rtkb::backproject_geometry(g, vol, proj, static_cast<const __nv_bfloat16 *>(d_proj_bf16), d_vol_in,
                                      d_vol_out, stream, false);
  }
  catch (...)
  {
    return rtkb::fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

extern "C" int
rtkb_fdk_backproject_batch(const rtkb_bp_problem * problems, int n, int config, int * used_config, void * stream)
{
  RTKB_TRACE();
  try
  {
    return rtkb::backproject_batch(problems, n, true, config, used_config, static_cast<cudaStream_t>(stream));
  }
  catch (...)
  {
    return rtkb::fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

extern "C" int
rtkb_voxel_backproject_batch(const rtkb_bp_problem * problems, int n, int config, int * used_config, void * stream)
{
  RTKB_TRACE();
  try
  {
    return rtkb::backproject_batch(problems, n, false, config, used_config, static_cast<cudaStream_t>(stream));
  }
  catch (...)
  {
    return rtkb::fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

extern "C" int
rtkb_bp_batch_create(const rtkb_bp_problem * problems, int n, int fdk, int config, rtkb_bp_batch ** batch)
{
  RTKB_TRACE();
  try
  {
    return rtkb::create_batch(problems, n, fdk != 0, config, batch);
  }
  catch (...)
  {
    return rtkb::fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

extern "C" int
rtkb_bp_batch_execute(rtkb_bp_batch * batch, void * stream)
{
  RTKB_TRACE();
  return rtkb::execute_batch(batch, static_cast<cudaStream_t>(stream));
}

extern "C" int
rtkb_bp_batch_config(const rtkb_bp_batch * batch)
{
  return batch ? batch->cfg : -1;
}

extern "C" void
rtkb_bp_batch_destroy(rtkb_bp_batch * batch)
{
  rtkb::release_batch(batch);
}

extern "C" int
rtkb_backproject_autotune(const rtkb_bp_problem * problems, int n, int fdk, int repeats, int * best_config,
                          double * best_ms, double * config_ms, void * stream)
{
  RTKB_TRACE();
  using namespace rtkb;
  if (!problems || n <= 0 || !best_config)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  for (int i = 0; i < n; i++)
    if (problems[i].d_vol_in == problems[i].d_vol_out)
      return fail(RTKB_ERR_INVALID_ARGUMENT, "autotuning runs the batch repeatedly: d_vol_out must not alias d_vol_in");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaEvent_t  e0 = nullptr, e1 = nullptr;
  RTKB_CUDA_TRY(cudaEventCreate(&e0));
  RTKB_CUDA_TRY(cudaEventCreate(&e1));
  int    best = -1, rc = RTKB_OK;
  double best_t = 1e300;
  const int saved_force = g_bp_forced_config;
  for (int c = 0; c < kNumBpConfigs && rc == RTKB_OK; c++)
  {
    // one problem: time the single-problem kernel its own calls run (with the
    // configuration forced); several: a prepared persistent batch
    rtkb_bp_batch * B = nullptr;
    if (n > 1)
    {
      rc = create_batch(problems, n, fdk != 0, c, &B);
      if (rc != RTKB_OK)
        break;
    }
    g_bp_forced_config = c;
    const rtkb_bp_problem & P0 = problems[0];
    auto run = [&]() {
      return n > 1 ? execute_batch(B, st)
                   : backproject_geometry(P0.geometry, &P0.vol, &P0.proj, P0.d_proj, P0.d_vol_in, P0.d_vol_out, stream,
                                          fdk != 0);
    };
    rc = run(); // warm-up
    cudaError_t e = cudaEventRecord(e0, st);
    for (int r = 0; r < std::max(repeats, 1) && rc == RTKB_OK && e == cudaSuccess; r++)
      rc = run();
    if (e == cudaSuccess)
      e = cudaEventRecord(e1, st);
    if (e == cudaSuccess)
      e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess)
      e = cudaEventElapsedTime(&ms, e0, e1);
    if (e != cudaSuccess && rc == RTKB_OK)
      rc = cuda_fail(e, "autotune timing");
    release_batch(B);
    g_bp_forced_config = saved_force;
    const double t = ms / std::max(repeats, 1);
    if (config_ms)
      config_ms[c] = t;
    if (rc == RTKB_OK && t < best_t)
    {
      best_t = t;
      best = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != RTKB_OK)
    return rc;
  *best_config = best;
  if (best_ms)
    *best_ms = best_t;
  return RTKB_OK;
}

extern "C" int
rtkb_convert_to_bf16(const float * d_in, void * d_out, long long n, void * stream)
{
  RTKB_TRACE();
  if ((!d_in || !d_out) && n > 0)
    return rtkb::fail(RTKB_ERR_INVALID_ARGUMENT, "null buffer");
  if (n <= 0)
    return RTKB_OK;
  const long long blocks = std::min<long long>((n + 255) / 256, 148LL * 32);
  to_bf16_kernel<<<(unsigned)blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
    d_in, static_cast<__nv_bfloat16 *>(d_out), n);
  RTKB_CUDA_TRY(cudaGetLastError());
  return RTKB_OK;
}

extern "C" int
rtkb_backproject_matrices(const int vol_size[3], const int proj_size[3], int n_proj, const double * matrices,
                          const int * modes, int weighting, const float * d_proj, const float * d_vol_in,
                          float * d_vol_out, void * stream)
{
  RTKB_TRACE();
  if (!vol_size || !proj_size)
    return rtkb::fail(RTKB_ERR_INVALID_ARGUMENT, "null size");
  try
  {
    return rtkb::backproject_buffer(vol_size, proj_size, n_proj, matrices, modes, weighting != 0, d_proj, d_vol_in,
                                    d_vol_out, static_cast<cudaStream_t>(stream));
  }
  catch (...)
  {
    return rtkb::fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

extern "C" int
rtkb_device_status(void * stream, int * status)
{
  if (!status)
    return rtkb::fail(RTKB_ERR_INVALID_ARGUMENT, "null status");
  unsigned int v = 0, zero = 0;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  RTKB_CUDA_TRY(cudaMemcpyFromSymbolAsync(&v, rtkb::dev::g_device_status, sizeof(v), 0, cudaMemcpyDeviceToHost, st));
  RTKB_CUDA_TRY(cudaStreamSynchronize(st));
  RTKB_CUDA_TRY(cudaMemcpyToSymbolAsync(rtkb::dev::g_device_status, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice,
                                        st));
  RTKB_CUDA_TRY(cudaStreamSynchronize(st));
  // a wait that gave up, else another failed device-side check (a tile whose
  // footprint left its staged box)
  *status = v == 0 ? RTKB_OK : (v & RTKB_STATUS_TIMEOUT) ? RTKB_ERR_TIMEOUT : RTKB_ERR_CUDA;
  return RTKB_OK;
}

// ---- failure detection without a GPU fault --------------------------------------
namespace
{
// One CTA waits, with the library's bounded wait, on an mbarrier that expects
// one arrival nobody makes; the wait gives up after g_wait_limit polls,
// records the timeout and the kernel returns.
__global__ void
wait_self_test_kernel()
{
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0)
  {
    rtkb::dev::mbar_init(&bar, 1);
    rtkb::dev::fence_barrier_init();
  }
  __syncthreads();
  if (threadIdx.x == 0)
    rtkb::dev::mbar_wait(&bar, 0);
  __syncthreads();
}
} // namespace

extern "C" int
rtkb_set_wait_limit(unsigned int polls, unsigned int * previous)
{
  if (polls == 0)
    return rtkb::fail(RTKB_ERR_INVALID_ARGUMENT, "the wait limit must be at least one poll");
  unsigned int old = 0;
  RTKB_CUDA_TRY(cudaMemcpyFromSymbol(&old, rtkb::dev::g_wait_limit, sizeof(old)));
  RTKB_CUDA_TRY(cudaMemcpyToSymbol(rtkb::dev::g_wait_limit, &polls, sizeof(polls)));
  if (previous)
    *previous = old;
  return RTKB_OK;
}

extern "C" int
rtkb_wait_self_test(void * stream)
{
  RTKB_TRACE();
  wait_self_test_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>();
  RTKB_CUDA_TRY(cudaGetLastError());
  return RTKB_OK;
}

extern "C" int
rtkb_backproject_config(int force, int * last_used, int * count)
{
  if (force < -1 || force >= kNumBpConfigs)
    return rtkb::fail(RTKB_ERR_INVALID_ARGUMENT, "backprojection configuration index out of range");
  if (last_used)
    *last_used = g_bp_last_config;
  if (count)
    *count = kNumBpConfigs;
  g_bp_forced_config = force;
  return RTKB_OK;
}

extern "C" int
rtkb_bp_set_schedule(int schedule, int sweep_shift)
{
  if (schedule < 0 || schedule > 1 || sweep_shift < 0 || sweep_shift > 10)
    return rtkb::fail(RTKB_ERR_INVALID_ARGUMENT, "backprojection schedule out of range");
  g_bp_schedule = schedule;
  g_bp_sweep_shift = sweep_shift;
  return RTKB_OK;
}

// ---- FDK backprojection without device allocations ----------------------------
//
// Some callers cannot allocate device memory while they reconstruct: an
// application whose device memory is entirely reserved by its own allocator
// (an image pipeline's GPU buffer pool, a framework's caching allocator at its
// limit), or an on-line reconstruction loop that must not take cudaMalloc's
// implicit device synchronisation.  rtkb_fdk_backproject_static_scratch serves
// them: its only scratch (the FP64 projection matrices and path modes of the
// stack) lives in the file-scope device array below, which every GPU that loads
// this library holds from module load until the process exits.
namespace
{
constexpr int kStaticMaxProjections = 2048;
constexpr int kStaticBytesPerProjection = 12 * sizeof(double) + sizeof(int);
static __device__ __align__(256) unsigned char
  g_bp_static_scratch[kStaticMaxProjections * kStaticBytesPerProjection + kProgressBytes];

std::mutex g_static_mutex;
void *     g_static_address[256] = {}; // per device ordinal
void *     g_static_context[256] = {}; // the context each address belongs to

// The driver's cuCtxGetCurrent, reached through the runtime (the library does
// not link libcuda).  Null if the driver does not export it.
using CtxGetCurrentFn = int (*)(void **);
CtxGetCurrentFn
ctx_get_current()
{
  static std::once_flag  once;
  static CtxGetCurrentFn fn = nullptr;
  std::call_once(once, [] {
    void *                          ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<CtxGetCurrentFn>(ptr);
    else
      cudaGetLastError();
  });
  return fn;
}

// Device address of g_bp_static_scratch on the current device, looked up with
// that device current the first time the entry point runs there, and again
// whenever the device's context has changed since (after cudaDeviceReset the
// module, and so the array, is loaded anew at another address).  In host code
// the array's name is only a stand-in for the symbol, never a device address.
int
static_scratch_address(void ** out)
{
  int dev = 0;
  RTKB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 256)
    return rtkb::fail(RTKB_ERR_UNSUPPORTED, "device ordinal out of range");
  void *          ctx = nullptr;
  CtxGetCurrentFn get = ctx_get_current();
  if (get && get(&ctx) != 0)
    ctx = nullptr;
  std::lock_guard<std::mutex> lock(g_static_mutex);
  if (!g_static_address[dev] || !ctx || g_static_context[dev] != ctx)
  {
    void *      p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_bp_static_scratch); // makes the primary context current
    if (e != cudaSuccess)
      return rtkb::cuda_fail(e, "cudaGetSymbolAddress(g_bp_static_scratch)");
    if (get && get(&ctx) != 0)
      ctx = nullptr;
    g_static_address[dev] = p;
    g_static_context[dev] = ctx;
  }
  *out = g_static_address[dev];
  return RTKB_OK;
}
} // namespace

extern "C" int
rtkb_fdk_backproject_static_scratch(const rtkb_geometry * g, const rtkb_image_desc * vol,
                                    const rtkb_image_desc * proj, const float * d_proj, const float * d_vol_in,
                                    float * d_vol_out, void * stream)
{
  RTKB_TRACE();
  if (proj && proj->size[2] > kStaticMaxProjections)
    return rtkb::fail(RTKB_ERR_INVALID_ARGUMENT,
                      "rtkb_fdk_backproject_static_scratch: the stack has more than 2048 projections, the size of "
                      "its static scratch; split the stack or use rtkb_fdk_backproject");
  try
  {
    void * scratch = nullptr;
    int    rc = static_scratch_address(&scratch);
    if (rc != RTKB_OK)
      return rc;
    return rtkb::backproject_geometry(g, vol, proj, d_proj, d_vol_in, d_vol_out, stream, true, scratch);
  }
  catch (...)
  {
    return rtkb::fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

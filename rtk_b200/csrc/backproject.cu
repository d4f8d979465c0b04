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
#include "rtkb_internal.h"
#include "rtkb_ptx.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>
#include <mutex>

namespace rtkb
{
namespace dev
{
__device__ unsigned int g_device_status = 0;
}
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
  static constexpr int kHeaders = 0;
  static constexpr int kBoxes = kStages * kHeaderBytes;
  static constexpr int kBars = kBoxes + kStages * kBoxBytes;
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

// Producer warp: per projection, project the tile's corners, size the
// footprint box, publish the tile-relative coefficients and start the TMA
// load of the box.
template <int BW, int BH, int NYT, typename T>
__device__ __forceinline__ void
bp_producer(const CUtensorMap * tmap, const T * __restrict__ proj, const double * __restrict__ mats, int nproj,
            int nu, int nv, int x0, int y0, int z0, StageHeader * hdr, T * boxes, uint64_t * full,
            uint64_t * empty, int use_tma)
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
  double mnext = (lane < 12 && nproj > 0) ? __ldg(mats + lane) : 0.0;
  for (int p = 0; p < nproj; p++)
  {
    const int s = p % kStages, k = p / kStages;
    if (p >= kStages && !mbar_wait(&empty[s], (k - 1) & 1))
      return;
    StageHeader * h = hdr + s;
    if (lane < 12)
    {
      h->m[lane] = mnext;
      h->mf[lane] = (float)mnext;
    }
    if (lane < 12 && p + 1 < nproj)
      mnext = __ldg(mats + 12 * (long long)(p + 1) + lane);
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
    T *      box = boxes + s * (BW * BH);
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
      h->fl = make_int4(skip ? kFlagSkip : flags, ub, vb, 0);
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
    if (!mbar_wait(&full[p % kStages], (p / kStages) & 1))
      return;
}

template <int BW, int BH, int NYT, int MINB, bool FDKW, typename T = float>
__global__ void __launch_bounds__(kThreads, MINB)
bp_tiled_kernel(const __grid_constant__ CUtensorMap tmap, const T * __restrict__ proj,
                const double * __restrict__ mats, int nproj, int nu, int nv, int nx, int ny, int nz, int ntx,
                int ntz, const float * vol_in, float * vol_out, int use_tma)
{
  using L = Layout<BW, BH, T>;
  extern __shared__ __align__(1024) unsigned char smem[];
  StageHeader * hdr = reinterpret_cast<StageHeader *>(smem + L::kHeaders);
  T *           boxes = reinterpret_cast<T *>(smem + L::kBoxes);
  uint64_t *    full = reinterpret_cast<uint64_t *>(smem + L::kBars);
  uint64_t *    empty = full + kStages;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
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
    bp_producer<BW, BH, NYT, T>(&tmap, proj, mats, nproj, nu, nv, x0, y0, z0, hdr, boxes, full, empty, use_tma);
    return;
  }

  // --------------------------------------------------------------- consumers
  const int   t = threadIdx.x;
  const int   dx = t % kTX, dz = t / kTX;
  const int   X = x0 + dx, Z = z0 + dz;
  const bool  active = (X < nx) && (Z < nz);
  const float fdx = (float)dx, fdz = (float)dz;
  float       acc[NYT];
#pragma unroll
  for (int j = 0; j < NYT; j++)
    acc[j] = 0.f;

  for (int p = 0; p < nproj; p++)
  {
    const int s = p % kStages, k = p / kStages;
    if (!mbar_wait(&full[s], k & 1))
      return;
    const StageHeader * h = hdr + s;
    const T *           box = boxes + s * (BW * BH);
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
#pragma unroll
            for (int j = 0; j < NYT; j++)
            {
              const float   v = fmaf((float)j, dv, v0);
              const float   flv = floorf(v);
              const float   fv = v - flv;
              const T *     q = col + (int)flv * BW;
              const float   p00 = tap(q), p01 = tap(q + 1), p10 = tap(q + BW), p11 = tap(q + BW + 1);
              const float   r0 = fmaf(fu, p01 - p00, p00);
              const float   r1 = fmaf(fu, p11 - p10, p10);
              acc[j] = fmaf(wt, fmaf(fv, r1 - r0, r0), acc[j]);
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
                acc[j] = fmaf(wt, fmaf(fv, r1 - r0, r0), acc[j]);
              }
            }
          }
        }
      }
      else if (!(fl.x & kFlagSkip))
      {
        const long long pofs = (long long)p * nu * nv;
#pragma unroll
        for (int j = 0; j < NYT; j++)
          acc[j] += slow_voxel(h->m, proj, pofs, nu, nv, X, y0 + j, Z, FDKW);
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
        vol_out[o] = vol_in[o] + acc[j];
      }
    }
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
// Box widths of 68 and 132 floats put consecutive rows 4 banks apart, so taps
// in the same column but different rows do not collide.
static const BpConfig   kBpConfigs[kNumBpConfigs] = { { 68, 64, 16, 3 }, { 68, 64, 16, 2 }, { 68, 32, 8, 3 },
                                                      { 68, 32, 8, 2 },  { 132, 64, 16, 1 }, { 132, 64, 8, 1 } };
// BF16 boxes: widths are multiples of 8 elements (16-byte TMA rows); 72 and
// 136 elements are 36 and 68 words, again 4 banks per row.
static const BpConfig   kBpConfigsBf16[kNumBpConfigs] = { { 72, 64, 16, 3 }, { 72, 64, 16, 2 }, { 72, 32, 8, 3 },
                                                          { 72, 32, 8, 2 },  { 136, 64, 16, 1 }, { 136, 64, 8, 1 } };
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
  for (int p = 0; p < nproj; p++)
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

template <int BW, int BH, int NYT, int MINB, bool FDKW, typename T>
static int
launch_tiled(const CUtensorMap & tmap, bool use_tma, const T * d_proj, const double * d_mats, int nproj, int nu,
             int nv, int nx, int ny, int nz, const float * vin, float * vout, cudaStream_t st)
{
  using L = Layout<BW, BH, T>;
  auto kern = bp_tiled_kernel<BW, BH, NYT, MINB, FDKW, T>;
  RTKB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L::kTotal));
  const int       ntx = (nx + kTX - 1) / kTX, nty = (ny + NYT - 1) / NYT, ntz = (nz + kTZ - 1) / kTZ;
  const long long nblocks = (long long)ntx * nty * ntz;
  if (nblocks > 0x7fffffffLL)
    return rtkb::fail(RTKB_ERR_UNSUPPORTED, "volume too large for one launch");
  kern<<<(unsigned)nblocks, kThreads, L::kTotal, st>>>(tmap, d_proj, d_mats, nproj, nu, nv, nx, ny, nz, ntx, ntz, vin,
                                                       vout, use_tma ? 1 : 0);
  RTKB_CUDA_TRY(cudaGetLastError());
  return RTKB_OK;
}

template <bool FDKW>
static int
dispatch_tiled(int cfg, const CUtensorMap & tmap, bool use_tma, const float * d_proj, const double * d_mats,
               int nproj, int nu, int nv, int nx, int ny, int nz, const float * vin, float * vout, cudaStream_t st)
{
#define RTKB_BP_LAUNCH(BW, BH, NYT, MINB)                                                                              \
  return launch_tiled<BW, BH, NYT, MINB, FDKW, float>(tmap, use_tma, d_proj, d_mats, nproj, nu, nv, nx, ny, nz, vin,   \
                                                      vout, st)
  switch (cfg)
  {
    case 0:
      RTKB_BP_LAUNCH(68, 64, 16, 3);
    case 1:
      RTKB_BP_LAUNCH(68, 64, 16, 2);
    case 2:
      RTKB_BP_LAUNCH(68, 32, 8, 3);
    case 3:
      RTKB_BP_LAUNCH(68, 32, 8, 2);
    case 4:
      RTKB_BP_LAUNCH(132, 64, 16, 1);
    default:
      RTKB_BP_LAUNCH(132, 64, 8, 1);
  }
#undef RTKB_BP_LAUNCH
}

template <bool FDKW>
static int
dispatch_tiled(int cfg, const CUtensorMap & tmap, bool use_tma, const __nv_bfloat16 * d_proj, const double * d_mats,
               int nproj, int nu, int nv, int nx, int ny, int nz, const float * vin, float * vout, cudaStream_t st)
{
#define RTKB_BP_LAUNCH(BW, BH, NYT, MINB)                                                                              \
  return launch_tiled<BW, BH, NYT, MINB, FDKW, __nv_bfloat16>(tmap, use_tma, d_proj, d_mats, nproj, nu, nv, nx, ny, nz, \
                                                              vin, vout, st)
  switch (cfg)
  {
    case 0:
      RTKB_BP_LAUNCH(72, 64, 16, 3);
    case 1:
      RTKB_BP_LAUNCH(72, 64, 16, 2);
    case 2:
      RTKB_BP_LAUNCH(72, 32, 8, 3);
    case 3:
      RTKB_BP_LAUNCH(72, 32, 8, 2);
    case 4:
      RTKB_BP_LAUNCH(136, 64, 16, 1);
    default:
      RTKB_BP_LAUNCH(136, 64, 8, 1);
  }
#undef RTKB_BP_LAUNCH
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

template <typename T>
int
backproject_buffer(const int vol_size[3], const int proj_size[3], int nproj, const double * mats, const int * modes,
                   bool fdk, const T * d_proj, const float * d_vin, float * d_vout, cudaStream_t st,
                   void * fixed_scratch = nullptr)
{
  constexpr bool    kBf16 = sizeof(T) == 2;
  const BpConfig *  configs = kBf16 ? kBpConfigsBf16 : kBpConfigs;
  constexpr double  kSlack = kAlignElems<T> - 1 + 0.2; // box origin rounding + margins
  const int nx = vol_size[0], ny = vol_size[1], nz = vol_size[2];
  const int nu = proj_size[0], nv = proj_size[1];
  if (nx <= 0 || ny <= 0 || nz <= 0 || nu <= 0 || nv <= 0 || nproj < 0 || proj_size[2] < nproj)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "invalid sizes");
  if (!d_vin || !d_vout || (nproj > 0 && !d_proj) || (nproj > 0 && (!mats || !modes)))
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null buffer");
  const long long nvox = (long long)nx * ny * nz;
  if (nproj == 0)
  {
    if (d_vout != d_vin)
      RTKB_CUDA_TRY(cudaMemcpyAsync(d_vout, d_vin, nvox * sizeof(float), cudaMemcpyDeviceToDevice, st));
    return RTKB_OK;
  }
  bool all_opt_y = true;
  for (int p = 0; p < nproj; p++)
  {
    for (int q = 0; q < 12; q++)
      if (!std::isfinite(mats[12 * p + q]))
        return fail(RTKB_ERR_INVALID_ARGUMENT, "non-finite projection matrix");
    if (modes[p] != 2)
      all_opt_y = false;
  }
  // matrices and modes in one scratch block: the caller's when given, else a
  // stream-ordered allocation
  const size_t mbytes = sizeof(double) * 12 * (size_t)nproj;
  void *       scratch = fixed_scratch;
  if (!scratch)
    RTKB_CUDA_TRY(cudaMallocAsync(&scratch, mbytes + sizeof(int) * nproj, st));
  double * d_mats = static_cast<double *>(scratch);
  int *    d_modes = reinterpret_cast<int *>(static_cast<char *>(scratch) + mbytes);
  int      rc = RTKB_OK;
  do
  {
    cudaError_t e = cudaMemcpyAsync(d_mats, mats, mbytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_modes, modes, sizeof(int) * nproj, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess)
    {
      rc = cuda_fail(e, "cudaMemcpyAsync");
      break;
    }
    if (!all_opt_y)
    {
      const long long blocks = std::min<long long>((nvox + 255) / 256, 148LL * 64);
      if (fdk)
        bp_generic_kernel<true, T><<<(unsigned)blocks, 256, 0, st>>>(d_proj, d_mats, d_modes, nproj, nu, nv, nx, ny,
                                                                     nz, d_vin, d_vout);
      else
        bp_generic_kernel<false, T><<<(unsigned)blocks, 256, 0, st>>>(d_proj, d_mats, d_modes, nproj, nu, nv, nx, ny,
                                                                      nz, d_vin, d_vout);
      e = cudaGetLastError();
      if (e != cudaSuccess)
        rc = cuda_fail(e, "bp_generic_kernel launch");
      break;
    }
    // first configuration whose box holds the footprints probed on the host
    std::vector<double> mv(mats, mats + 12 * (size_t)nproj);
    double              fw8, fh8, fw16, fh16;
    estimate_footprint(mv, nproj, nx, ny, nz, 8, fw8, fh8);
    estimate_footprint(mv, nproj, nx, ny, nz, 16, fw16, fh16);
    int cfg = kNumBpConfigs - 1;
    for (int c = 0; c < kNumBpConfigs; c++)
    {
      const double fw = configs[c].nyt == 16 ? fw16 : fw8, fh = configs[c].nyt == 16 ? fh16 : fh8;
      if (fw + kSlack < configs[c].bw - 1 && fh + 0.2 < configs[c].bh - 1)
      {
        cfg = c;
        break;
      }
    }
    if (g_bp_forced_config >= 0)
      cfg = g_bp_forced_config; // a box too small for some tiles only sends them to the FP64 path
    g_bp_last_config = cfg;
    // TMA needs 16-byte aligned rows and base address
    CUtensorMap tmap;
    std::memset(&tmap, 0, sizeof(tmap));
    bool              use_tma = false;
    EncodeTiledFn     enc = tensor_map_encoder();
    const long long   np_total = proj_size[2];
    const unsigned long long esz = sizeof(T);
    if (enc && ((unsigned long long)nu * esz) % 16 == 0 && (reinterpret_cast<uintptr_t>(d_proj) % 16) == 0 &&
        np_total <= 0x7fffffffLL)
    {
      const unsigned long long dims[3] = { (unsigned long long)nu, (unsigned long long)nv,
                                           (unsigned long long)np_total };
      const unsigned long long strides[2] = { (unsigned long long)nu * esz, (unsigned long long)nu * nv * esz };
      const unsigned           box[3] = { (unsigned)configs[cfg].bw, (unsigned)configs[cfg].bh, 1u };
      const unsigned           estr[3] = { 1u, 1u, 1u };
      const int r = enc(&tmap, kBf16 ? (int)CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : (int)CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                        3u, const_cast<T *>(d_proj), dims, strides,
                        box, estr, (int)CU_TENSOR_MAP_INTERLEAVE_NONE, (int)CU_TENSOR_MAP_SWIZZLE_NONE,
                        (int)CU_TENSOR_MAP_L2_PROMOTION_L2_128B, (int)CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      use_tma = (r == 0);
    }
    rc = fdk ? dispatch_tiled<true>(cfg, tmap, use_tma, d_proj, d_mats, nproj, nu, nv, nx, ny, nz, d_vin, d_vout, st)
             : dispatch_tiled<false>(cfg, tmap, use_tma, d_proj, d_mats, nproj, nu, nv, nx, ny, nz, d_vin, d_vout,
                                     st);
  } while (0);
  if (!fixed_scratch)
  {
    cudaError_t fe = cudaFreeAsync(scratch, st);
    if (rc == RTKB_OK && fe != cudaSuccess)
      rc = cuda_fail(fe, "cudaFreeAsync");
  }
  return rc;
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
  if (g->g.radius_cylindrical != 0.)
    return fail(RTKB_ERR_UNSUPPORTED,
                "Voxel-based FDK back projector can currently not handle cylindrical detectors");
  const int nproj = proj->size[2];
  if (proj->index[2] < 0 || (long long)proj->index[2] + nproj > (long long)g->g.p.size())
    return fail(RTKB_ERR_INVALID_ARGUMENT, "Mismatch between the number of projections and the geometry entries.");
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

extern "C" int
rtkb_fdk_backproject(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                     const float * d_proj, const float * d_vol_in, float * d_vol_out, void * stream)
{
  try
  {
    return rtkb::backproject_geometry(g, vol, proj, d_proj, d_vol_in, d_vol_out, stream, true);
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
rtkb_convert_to_bf16(const float * d_in, void * d_out, long long n, void * stream)
{
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
  *status = (int)v;
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
static __device__ __align__(256) unsigned char g_bp_static_scratch[kStaticMaxProjections * kStaticBytesPerProjection];

std::mutex g_static_mutex;
void *     g_static_address[256] = {}; // per device ordinal

// Device address of g_bp_static_scratch on the current device, looked up once
// per device with that device current.  In host code the array's name is only
// a stand-in for the symbol, never a device address.
int
static_scratch_address(void ** out)
{
  int dev = 0;
  RTKB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 256)
    return rtkb::fail(RTKB_ERR_UNSUPPORTED, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_static_mutex);
  if (!g_static_address[dev])
  {
    void *      p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_bp_static_scratch);
    if (e != cudaSuccess)
      return rtkb::cuda_fail(e, "cudaGetSymbolAddress(g_bp_static_scratch)");
    g_static_address[dev] = p;
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

// unet.cu -- the learned preconditioner: a 3-level 3D U-Net (16/32/64
// channels) with hand-written BF16 tensor-core convolutions (forward, data
// gradient, weight gradient), FP32 accumulation and an Adam trainer.
//
// No RTK counterpart: RTK's conjugate gradient is unpreconditioned
// (include/rtkConjugateGradientImageFilter.hxx:108-258).  The network maps a
// normal-equation residual r to an approximation of (A^T A)^-1 r; it is
// trained on pairs (A e, e) produced by the projector pair itself and used
// inside flexible PCG (cg.cu).
//
// Architecture (no biases, ReLU after every 3x3x3 convolution; with the input
// divided by s = rms(r) and the output multiplied by s the map is positively
// homogeneous):
//   L1  conv 1->16 (CUDA cores, FP32 weights)        level 0
//   L2  conv 16->16                                  level 0   -> skip e1
//   avg-pool 2x2x2
//   L3  conv 16->32, L4 conv 32->32                  level 1   -> skip e2
//   avg-pool 2x2x2
//   L5  conv 32->64, L6 conv 64->64                  level 2
//   L7  conv [nearest-up(L6), e2] 96->32, L8 32->32  level 1
//   L9  conv [nearest-up(L8), e1] 48->16, L10 16->16 level 0
//   L11 1x1x1 conv 16->1, no activation (FP32 weights)
// Activations are channels-last BF16 tensors [batch][z][y][x][C].  Weights are
// kept as FP32 masters [tap][c_in][c_out] (tap = (kz*3+ky)*3+kx, cross-
// correlation as torch.nn.functional.conv3d with padding 1) and repacked to
// BF16 after every update.
//
// The forward and data-gradient convolutions run on tcgen05 (implicit GEMM:
// M = voxels of an 8x16x4 output tile as four M = 128 accumulators in tensor
// memory, N = output channels, K = 27 taps x 16-channel input chunks, operands
// from shared-memory descriptors); the weight gradient uses mma.sync m16n8k16
// with ldmatrix gathers by default, or a tcgen05 kernel with MN-major operands
// (rtkb_unet_set_wgrad_kernel; slower for these layer widths).  Up-sampling and concatenation of the decoder inputs
// are folded into the halo loaders, the ReLU-derivative mask into the
// data-gradient epilogue.
#include "rtkb_internal.h"
#include "rtkb_ptx.cuh"

#include <cuda_bf16.h>

#include <cstring>
#include <random>

namespace
{

typedef __nv_bfloat16 bf16;

constexpr int kTX = 16, kTY = 4, kTZ = 4;                         // output tile
constexpr int kHX = kTX + 2, kHY = kTY + 2, kHZ = kTZ + 2;         // halo tile
constexpr int kHalo = kHX * kHY * kHZ;                            // 648 voxels
constexpr int kHaloBytes = kHalo * 32;                            // 16 BF16 channels per voxel
constexpr int kTileVox = kTX * kTY * kTZ;                         // 256
constexpr int kThreads = 256;

// ---- small helpers ------------------------------------------------------------------------------
__device__ __forceinline__ unsigned
smem_u32(const void * p)
{
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void
ldsm_x4_t(unsigned addr, unsigned & r0, unsigned & r1, unsigned & r2, unsigned & r3)
{
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(addr));
}

__device__ __forceinline__ void
mma_bf16(float * c, unsigned a0, unsigned a1, unsigned a2, unsigned a3, unsigned b0, unsigned b1)
{
  asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
               "{%0,%1,%2,%3};"
               : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
               : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ unsigned
pack_bf16x2(float lo, float hi)
{
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const unsigned *>(&v);
}

__device__ __forceinline__ float2
unpack_bf16x2(unsigned u)
{
  __nv_bfloat162 v;
  *reinterpret_cast<unsigned *>(&v) = u;
  return __bfloat1622float2(v);
}

// Conv input: channels [0, ca) come from tensor a (at half resolution when
// a_half, read by nearest up-sampling), channels [ca, ca+cb) from tensor b.
struct ConvIn
{
  const bf16 * a;
  const bf16 * b;
  int          ca, cb, a_half;
};

struct Dims
{
  int nx, ny, nz, batch;
  int tx, ty, tz; // tile counts
  __host__ __device__ long long vox() const { return (long long)nx * ny * nz; }
};

Dims
make_dims(int nx, int ny, int nz, int batch)
{
  Dims d{ nx, ny, nz, batch, (nx + kTX - 1) / kTX, (ny + kTY - 1) / kTY, (nz + kTZ - 1) / kTZ };
  return d;
}

__device__ __forceinline__ void
tile_origin(const Dims & d, long long tile, int & n, int & x0, int & y0, int & z0)
{
  const int tx = (int)(tile % d.tx);
  long long r = tile / d.tx;
  const int ty = (int)(r % d.ty);
  r /= d.ty;
  const int tz = (int)(r % d.tz);
  n = (int)(r / d.tz);
  x0 = tx * kTX;
  y0 = ty * kTY;
  z0 = tz * kTZ;
}

// Halo chunk -> shared memory: 16 channels of chunk c for the (18 x 6 x 6)
// neighbourhood of the tile; each voxel is 32 bytes whose two 16-byte halves
// are swapped when bit 2 of the voxel index is set (conflict-free ldmatrix
// rows).  Zero outside the volume.
__device__ __forceinline__ void
load_halo(char * halo, const ConvIn & in, const Dims & d, int n, int x0, int y0, int z0, int chunk)
{
  const bool from_a = chunk * 16 < in.ca;
  const int  cs = from_a ? in.ca : in.cb;
  const int  c0 = from_a ? chunk * 16 : chunk * 16 - in.ca;
  const bf16 * src = from_a ? in.a : in.b;
  const bool half = from_a && in.a_half;
  const int  snx = half ? d.nx >> 1 : d.nx, sny = half ? d.ny >> 1 : d.ny, snz = half ? d.nz >> 1 : d.nz;
  for (int i = threadIdx.x; i < kHalo * 2; i += kThreads)
  {
    const int hv = i >> 1, h = i & 1;
    const int hx = hv % kHX, hy = (hv / kHX) % kHY, hz = hv / (kHX * kHY);
    const int gx = x0 - 1 + hx, gy = y0 - 1 + hy, gz = z0 - 1 + hz;
    uint4     v = make_uint4(0u, 0u, 0u, 0u);
    if (gx >= 0 && gx < d.nx && gy >= 0 && gy < d.ny && gz >= 0 && gz < d.nz)
    {
      const int sx = half ? gx >> 1 : gx, sy = half ? gy >> 1 : gy, sz = half ? gz >> 1 : gz;
      const long long off = ((((long long)n * snz + sz) * sny + sy) * snx + sx) * cs + c0 + h * 8;
      v = *reinterpret_cast<const uint4 *>(src + off);
    }
    *reinterpret_cast<uint4 *>(halo + hv * 32 + ((h ^ ((hv >> 2) & 1)) << 4)) = v;
  }
}

// ---- forward / data-gradient convolution on the 5th-generation tensor cores ------------------------
// tcgen05.mma (kind::f16: BF16 x BF16 -> FP32 in tensor memory), operands in
// shared memory described by matrix descriptors (K-major, no swizzle).  A CTA
// (one warpgroup) owns an 8 (x) x 16 (y) x 4 (z) output tile: four M = 128
// accumulators (one per z-slice, 8 x-voxels x 16 y-rows), N = output channels.
// Per 16-channel input chunk the 10 x 18 x 6 halo is stored as
// [k-half][voxel][8 channels], so the A operand of tap (dz, dy, dx) and slice
// z is a descriptor starting at that tap's first halo voxel with 8-row groups
// one halo row (10 voxels = 160 bytes) apart; weights are packed as
// [tap][k-half][c_out][8 c_in].  One thread issues the 27 x 4 MMAs of a chunk
// and commits them to an mbarrier; the epilogue reads the accumulators with
// tcgen05.ld, applies ReLU or the gradient mask and stores BF16.
constexpr int kCX = 8, kCY = 16, kCZ = 4;                   // output tile
constexpr int kCHX = kCX + 2, kCHY = kCY + 2, kCHZ = kCZ + 2; // halo
constexpr int kCHalo = kCHX * kCHY * kCHZ;                   // 1080 voxels
constexpr int kCHaloBytes = kCHalo * 32;

struct TcDims
{
  int nx, ny, nz, batch, tx, ty, tz;
};

TcDims
make_tc_dims(int nx, int ny, int nz, int batch)
{
  TcDims d{ nx, ny, nz, batch, (nx + kCX - 1) / kCX, (ny + kCY - 1) / kCY, (nz + kCZ - 1) / kCZ };
  return d;
}

__device__ __forceinline__ uint64_t
umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
  // start address, leading and stride byte offsets (all >> 4), version 1 (sm_100), no swizzle
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

template <int N>
__device__ __forceinline__ constexpr uint32_t
umma_idesc_bf16()
{
  // FP32 accumulator, BF16 A and B, both K-major, N >> 3, M = 128 >> 4
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void
umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate)
{
  asm volatile("{\n\t.reg .pred p;\n\t"
               "setp.ne.b32 p, %4, 0;\n\t"
               "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
               :
               : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void
umma_commit(uint64_t * bar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               ::"r"(rtkb::dev::smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void
tmem_ld16(uint32_t taddr, uint32_t (&r)[16])
{
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                 "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                 "=r"(r[15])
               : "r"(taddr));
}

template <int N>
__global__ void __launch_bounds__(128, 1)
conv_fwd_tc_kernel(ConvIn in, const bf16 * __restrict__ wpack, TcDims d, bf16 * __restrict__ out,
                   const bf16 * __restrict__ mask, int relu)
{
  constexpr int      kCols = (kCZ * N <= 32) ? 32 : (kCZ * N <= 64) ? 64 : (kCZ * N <= 128) ? 128 : (kCZ * N <= 256) ? 256 : 512;
  constexpr uint32_t kIdesc = umma_idesc_bf16<N>();
  extern __shared__ __align__(128) char smem[];
  char *             halo = smem;                              // [2][kCHalo][16 B]
  char *             wsm = smem + kCHaloBytes;                 // [27][2][N][16 B]
  uint64_t *         bar = reinterpret_cast<uint64_t *>(wsm + 27 * 2 * N * 16);
  uint32_t *         tmem_slot = reinterpret_cast<uint32_t *>(bar + 1);
  const int          warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  long long          tile = blockIdx.x;
  const int          tx = (int)(tile % d.tx);
  tile /= d.tx;
  const int ty = (int)(tile % d.ty);
  tile /= d.ty;
  const int tz = (int)(tile % d.tz);
  const int n = (int)(tile / d.tz);
  const int x0 = tx * kCX, y0 = ty * kCY, z0 = tz * kCZ;

  if (warp == 0)
  {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(rtkb::dev::smem_u32(tmem_slot)),
                 "r"((uint32_t)kCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0)
  {
    rtkb::dev::mbar_init(bar, 1);
    rtkb::dev::fence_barrier_init();
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;
  const int      nchunks = (in.ca + in.cb) / 16;
  const uint32_t halo_s = rtkb::dev::smem_u32(halo), w_s = rtkb::dev::smem_u32(wsm);
  bool           ok = true;

  for (int chunk = 0; chunk < nchunks && ok; chunk++)
  {
    // halo chunk: 16 channels of the 10 x 18 x 6 neighbourhood, [k-half][voxel][16 B], zero outside
    {
      const bool   from_a = chunk * 16 < in.ca;
      const int    cs = from_a ? in.ca : in.cb;
      const int    c0 = from_a ? chunk * 16 : chunk * 16 - in.ca;
      const bf16 * src = from_a ? in.a : in.b;
      const bool   half = from_a && in.a_half;
      const int    snx = half ? d.nx >> 1 : d.nx, sny = half ? d.ny >> 1 : d.ny, snz = half ? d.nz >> 1 : d.nz;
      for (int i = threadIdx.x; i < kCHalo * 2; i += 128)
      {
        const int hv = i >> 1, h = i & 1;
        const int hx = hv % kCHX, hy = (hv / kCHX) % kCHY, hz = hv / (kCHX * kCHY);
        const int gx = x0 - 1 + hx, gy = y0 - 1 + hy, gz = z0 - 1 + hz;
        uint4     v = make_uint4(0u, 0u, 0u, 0u);
        if (gx >= 0 && gx < d.nx && gy >= 0 && gy < d.ny && gz >= 0 && gz < d.nz)
        {
          const int sx = half ? gx >> 1 : gx, sy = half ? gy >> 1 : gy, sz = half ? gz >> 1 : gz;
          v = *reinterpret_cast<const uint4 *>(src + ((((long long)n * snz + sz) * sny + sy) * snx + sx) * cs + c0 + h * 8);
        }
        *reinterpret_cast<uint4 *>(halo + (h * kCHalo + hv) * 16) = v;
      }
      const uint4 * wsrc = reinterpret_cast<const uint4 *>(wpack + (size_t)chunk * 27 * 2 * N * 8);
      uint4 *       wdst = reinterpret_cast<uint4 *>(wsm);
      for (int i = threadIdx.x; i < 27 * 2 * N; i += 128)
        wdst[i] = wsrc[i];
    }
    // make the generic-proxy stores visible to the tensor cores, then issue
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0)
    {
      asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll 1
      for (int t = 0; t < 27; t++)
      {
        const int      dz = t / 9, dy = (t / 3) % 3, dx = t % 3;
        const uint64_t db = umma_desc(w_s + (uint32_t)(t * 2 * N * 16), (uint32_t)(N * 16), 128u);
#pragma unroll
        for (int zl = 0; zl < kCZ; zl++)
        {
          const int      hv0 = ((zl + dz) * kCHY + dy) * kCHX + dx;
          const uint64_t da = umma_desc(halo_s + (uint32_t)(hv0 * 16), (uint32_t)(kCHalo * 16), (uint32_t)(kCHX * 16));
          umma_bf16(tmem + (uint32_t)(zl * N), da, db, kIdesc, (chunk > 0 || t > 0) ? 1u : 0u);
        }
      }
      umma_commit(bar);
    }
    // the MMAs read shared memory asynchronously: wait before it is overwritten
    // (a wait that gave up stops every thread: the loop stays CTA-uniform)
    ok = __syncthreads_and(rtkb::dev::mbar_wait(bar, (uint32_t)(chunk & 1)) ? 1 : 0) != 0;
  }
  asm volatile("tcgen05.fence::after_thread_sync;");

  // epilogue: warp w reads TMEM lanes 32w..32w+31 = output rows m (x = m % 8, y = m / 8)
  if (ok)
  {
    const int m = warp * 32 + lane;
    const int x = x0 + (m & 7), y = y0 + (m >> 3);
#pragma unroll 1
    for (int zl = 0; zl < kCZ; zl++)
    {
      const int  z = z0 + zl;
      const bool inside = x < d.nx && y < d.ny && z < d.nz;
      const long long vbase = ((((long long)n * d.nz + z) * d.ny + y) * d.nx + x) * N;
#pragma unroll
      for (int cb = 0; cb < N; cb += 16)
      {
        uint32_t r[16];
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(zl * N + cb), r);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (!inside)
          continue;
        unsigned o[8];
#pragma unroll
        for (int q = 0; q < 8; q++)
        {
          float v0 = __uint_as_float(r[2 * q]), v1 = __uint_as_float(r[2 * q + 1]);
          if (relu)
          {
            v0 = fmaxf(v0, 0.f);
            v1 = fmaxf(v1, 0.f);
          }
          if (mask)
          {
            const float2 mk = unpack_bf16x2(*reinterpret_cast<const unsigned *>(mask + vbase + cb + 2 * q));
            v0 = mk.x > 0.f ? v0 : 0.f;
            v1 = mk.y > 0.f ? v1 : 0.f;
          }
          o[q] = pack_bf16x2(v0, v1);
        }
        uint4 * dst = reinterpret_cast<uint4 *>(out + vbase + cb);
        dst[0] = make_uint4(o[0], o[1], o[2], o[3]);
        dst[1] = make_uint4(o[4], o[5], o[6], o[7]);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)kCols));
}

// ---- the same convolution, pipelined: TMA halo loads overlapped with the MMAs ----------------------
// Two stages of [halo | weights].  While the MMAs of chunk c read stage c & 1,
// stage (c + 1) & 1 is filled with chunk c + 1 once the MMAs of chunk c - 1
// (its previous reader) have completed.  A full-resolution source is loaded
// by TMA: two boxes of 8 channels x 10 x 18 x 6 voxels (5-D tensor map over
// [batch][z][y][x][channel]), which land exactly in the [k-half][voxel][16 B]
// layout the A descriptors read, zero-filled outside the volume; the chunk's
// weights [27][2][N][8] come by one bulk copy.  A half-resolution source
// (nearest up-sampling, decoder inputs) is gathered by the threads into the
// same layout, still overlapped with the previous chunk's MMAs.  Every wait is
// bounded; a wait that gives up ends the chunk loop on every thread.
__device__ __forceinline__ void
tma_load_5d(void * dst, const CUtensorMap * map, int c0, int c1, int c2, int c3, int c4, uint64_t * bar)
{
  asm volatile("cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
               " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(rtkb::dev::smem_u32(dst)),
               "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4),
               "r"(rtkb::dev::smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void
bulk_load(void * dst, const void * src, uint32_t bytes, uint64_t * bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                 rtkb::dev::smem_u32(dst)),
               "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(rtkb::dev::smem_u32(bar))
               : "memory");
}

template <int N, int NS>
struct PipeLayout
{
  static constexpr int kW = 27 * 2 * N * 16;            // weight bytes per chunk
  static constexpr int kStage = kCHaloBytes + kW;        // one stage (multiple of 128 bytes)
  static constexpr int kBars = NS * kStage;              // full[2], done[2], TMEM slot
  static constexpr int kTotal = kBars + 64 + 128;        // + alignment slack of the dynamic base
  static_assert(kCHaloBytes % 128 == 0 && kW % 128 == 0, "TMA destinations need 128-byte alignment");
};

template <int N, int NS>
__global__ void __launch_bounds__(128, 1)
conv_fwd_pipe_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b, int tma_a,
                     int tma_b, ConvIn in, const bf16 * __restrict__ wpack, TcDims d, bf16 * __restrict__ out,
                     const bf16 * __restrict__ mask, int relu)
{
  using L = PipeLayout<N, NS>;
  constexpr int      kCols = (kCZ * N <= 32) ? 32 : (kCZ * N <= 64) ? 64 : (kCZ * N <= 128) ? 128 : (kCZ * N <= 256) ? 256 : 512;
  constexpr uint32_t kIdesc = umma_idesc_bf16<N>();
  extern __shared__ __align__(128) char smem_raw[];
  char * smem = reinterpret_cast<char *>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  uint64_t *         full = reinterpret_cast<uint64_t *>(smem + L::kBars);
  uint64_t *         done = full + 2;
  uint32_t *         tmem_slot = reinterpret_cast<uint32_t *>(done + 2);
  __shared__ int     s_ok;
  const int          warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  long long          tile = blockIdx.x;
  const int          tx = (int)(tile % d.tx);
  tile /= d.tx;
  const int ty = (int)(tile % d.ty);
  tile /= d.ty;
  const int tz = (int)(tile % d.tz);
  const int n = (int)(tile / d.tz);
  const int x0 = tx * kCX, y0 = ty * kCY, z0 = tz * kCZ;

  if (warp == 0)
  {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(rtkb::dev::smem_u32(tmem_slot)),
                 "r"((uint32_t)kCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0)
  {
    for (int q = 0; q < 2; q++)
    {
      rtkb::dev::mbar_init(&full[q], 1);
      rtkb::dev::mbar_init(&done[q], 1);
    }
    rtkb::dev::fence_barrier_init();
    s_ok = 1;
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;
  const int      nchunks = (in.ca + in.cb) / 16;

  // fill stage st with chunk c (block-uniform branch)
  auto load_chunk = [&](int c, int st) {
    char *       halo = smem + st * L::kStage;
    char *       wsm = halo + kCHaloBytes;
    const bool   from_a = c * 16 < in.ca;
    const int    c0 = from_a ? c * 16 : c * 16 - in.ca;
    const bool   tma = from_a ? tma_a != 0 : tma_b != 0;
    const bf16 * wsrc = wpack + (size_t)c * 27 * 2 * N * 8;
    if (tma)
    {
      if (threadIdx.x == 0)
      {
        const CUtensorMap * map = from_a ? &map_a : &map_b;
        rtkb::dev::mbar_arrive_expect_tx(&full[st], (uint32_t)(kCHaloBytes + L::kW));
        tma_load_5d(halo, map, c0, x0 - 1, y0 - 1, z0 - 1, n, &full[st]);
        tma_load_5d(halo + kCHalo * 16, map, c0 + 8, x0 - 1, y0 - 1, z0 - 1, n, &full[st]);
        bulk_load(wsm, wsrc, (uint32_t)L::kW, &full[st]);
      }
      return;
    }
    const int    cs = from_a ? in.ca : in.cb;
    const bf16 * src = from_a ? in.a : in.b;
    const bool   half = from_a && in.a_half;
    const int    snx = half ? d.nx >> 1 : d.nx, sny = half ? d.ny >> 1 : d.ny, snz = half ? d.nz >> 1 : d.nz;
    for (int i = threadIdx.x; i < kCHalo * 2; i += 128)
    {
      const int hv = i >> 1, h = i & 1;
      const int hx = hv % kCHX, hy = (hv / kCHX) % kCHY, hz = hv / (kCHX * kCHY);
      const int gx = x0 - 1 + hx, gy = y0 - 1 + hy, gz = z0 - 1 + hz;
      uint4     v = make_uint4(0u, 0u, 0u, 0u);
      if (gx >= 0 && gx < d.nx && gy >= 0 && gy < d.ny && gz >= 0 && gz < d.nz)
      {
        const int sx = half ? gx >> 1 : gx, sy = half ? gy >> 1 : gy, sz = half ? gz >> 1 : gz;
        v = *reinterpret_cast<const uint4 *>(src + ((((long long)n * snz + sz) * sny + sy) * snx + sx) * cs + c0 + h * 8);
      }
      *reinterpret_cast<uint4 *>(halo + (h * kCHalo + hv) * 16) = v;
    }
    const uint4 * w4 = reinterpret_cast<const uint4 *>(wsrc);
    uint4 *       wdst = reinterpret_cast<uint4 *>(wsm);
    for (int i = threadIdx.x; i < 27 * 2 * N; i += 128)
      wdst[i] = w4[i];
    // the tensor cores read this stage through the async proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0)
      rtkb::dev::mbar_arrive(&full[st]);
  };

  // thread 0's count of fills / commits issued and seen complete per stage (to
  // drain in-flight copies and MMAs if a wait gives up)
  int fill_issued[2] = { 0, 0 }, fill_seen[2] = { 0, 0 }, commit_issued[2] = { 0, 0 }, commit_seen[2] = { 0, 0 };
  if (nchunks > 0)
  {
    load_chunk(0, 0);
    fill_issued[0]++;
  }
  bool ok = true;
  for (int c = 0; c < nchunks && ok; c++)
  {
    const int      st = c % NS;
    const uint32_t par = (uint32_t)((c / NS) & 1);
    if (threadIdx.x == 0)
    {
      if (rtkb::dev::mbar_wait(&full[st], par))
      {
        fill_seen[st]++;
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t halo_s = rtkb::dev::smem_u32(smem + st * L::kStage);
        const uint32_t w_s = halo_s + (uint32_t)kCHaloBytes;
#pragma unroll 1
        for (int t = 0; t < 27; t++)
        {
          const int      dz = t / 9, dy = (t / 3) % 3, dx = t % 3;
          const uint64_t db = umma_desc(w_s + (uint32_t)(t * 2 * N * 16), (uint32_t)(N * 16), 128u);
#pragma unroll
          for (int zl = 0; zl < kCZ; zl++)
          {
            const int      hv0 = ((zl + dz) * kCHY + dy) * kCHX + dx;
            const uint64_t da = umma_desc(halo_s + (uint32_t)(hv0 * 16), (uint32_t)(kCHalo * 16), (uint32_t)(kCHX * 16));
            umma_bf16(tmem + (uint32_t)(zl * N), da, db, kIdesc, (c > 0 || t > 0) ? 1u : 0u);
          }
        }
        umma_commit(&done[st]);
        commit_issued[st]++;
      }
      else
        s_ok = 0;
    }
    if (c + 1 < nchunks)
    {
      // chunk c + 1's stage is free once its previous reader, chunk c + 1 - NS,
      // has completed its MMAs
      const int nx_st = (c + 1) % NS, prev = c + 1 - NS;
      bool      free_ok = true;
      if (prev >= 0)
      {
        free_ok = __syncthreads_and(s_ok ? 1 : 0) != 0 && rtkb::dev::mbar_wait(&done[nx_st], (uint32_t)((prev / NS) & 1));
        if (free_ok && threadIdx.x == 0)
          commit_seen[nx_st]++;
      }
      free_ok = __syncthreads_and(free_ok && s_ok ? 1 : 0) != 0;
      if (free_ok)
      {
        load_chunk(c + 1, nx_st);
        fill_issued[nx_st]++;
      }
      ok = free_ok;
    }
    ok = __syncthreads_and(ok && s_ok ? 1 : 0) != 0;
  }
  // the last chunk's MMAs
  if (ok && nchunks > 0)
  {
    const int  sl = (nchunks - 1) % NS;
    const bool got = rtkb::dev::mbar_wait(&done[sl], (uint32_t)(((nchunks - 1) / NS) & 1));
    if (got && threadIdx.x == 0)
      commit_seen[sl]++;
    ok = __syncthreads_and(got ? 1 : 0) != 0;
  }
  if (!ok && threadIdx.x == 0)
  {
    // a wait gave up: let this CTA's own copies and MMAs finish (bounded)
    // before its shared memory and tensor memory are released
    for (int q = 0; q < NS; q++)
    {
      if (fill_issued[q] > fill_seen[q])
        rtkb::dev::mbar_wait(&full[q], (uint32_t)(fill_seen[q] & 1));
      if (commit_issued[q] > commit_seen[q])
        rtkb::dev::mbar_wait(&done[q], (uint32_t)(commit_seen[q] & 1));
    }
  }
  asm volatile("tcgen05.fence::after_thread_sync;");

  if (ok)
  {
    const int m = warp * 32 + lane;
    const int x = x0 + (m & 7), y = y0 + (m >> 3);
#pragma unroll 1
    for (int zl = 0; zl < kCZ; zl++)
    {
      const int       z = z0 + zl;
      const bool      inside = x < d.nx && y < d.ny && z < d.nz;
      const long long vbase = ((((long long)n * d.nz + z) * d.ny + y) * d.nx + x) * N;
#pragma unroll
      for (int cb = 0; cb < N; cb += 16)
      {
        uint32_t r[16];
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(zl * N + cb), r);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (!inside)
          continue;
        unsigned o[8];
#pragma unroll
        for (int q = 0; q < 8; q++)
        {
          float v0 = __uint_as_float(r[2 * q]), v1 = __uint_as_float(r[2 * q + 1]);
          if (relu)
          {
            v0 = fmaxf(v0, 0.f);
            v1 = fmaxf(v1, 0.f);
          }
          if (mask)
          {
            const float2 mk = unpack_bf16x2(*reinterpret_cast<const unsigned *>(mask + vbase + cb + 2 * q));
            v0 = mk.x > 0.f ? v0 : 0.f;
            v1 = mk.y > 0.f ? v1 : 0.f;
          }
          o[q] = pack_bf16x2(v0, v1);
        }
        uint4 * dst = reinterpret_cast<uint4 *>(out + vbase + cb);
        dst[0] = make_uint4(o[0], o[1], o[2], o[3]);
        dst[1] = make_uint4(o[4], o[5], o[6], o[7]);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)kCols));
}

// ---- weight gradient --------------------------------------------------------------------------------
// dW[t][ci][co] += sum_v in[v + t - 1][ci] * g[v][co] for the 16 input channels
// of chunk blockIdx.y; CTAs stride over voxel tiles and flush once with
// atomics.  Warp w owns taps w, w+8, w+16 (and w+24 for w < 3).
template <int NT>
__global__ void __launch_bounds__(kThreads, 1)
conv_wgrad_kernel(ConvIn in, const bf16 * __restrict__ g, Dims d, float * __restrict__ dW, int cin_total)
{
  constexpr int COUT = NT * 8, S = COUT / 8; // 16-byte segments per gradient row
  extern __shared__ __align__(128) char smem[];
  char *        halo = smem;
  char *        gsm = smem + kHaloBytes;
  const int     lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int     chunk = blockIdx.y;
  const long long ntiles = (long long)d.tx * d.ty * d.tz * d.batch;

  float acc[4][NT][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < NT; j++)
#pragma unroll
      for (int k = 0; k < 4; k++)
        acc[i][j][k] = 0.f;

  const int      mi = lane >> 3;
  const int      a_vox = (lane & 7) + (mi >> 1) * 8, a_half = mi & 1;  // A = in^T via .trans
  const int      b_vox = (lane & 7) + (mi & 1) * 8, b_seg = mi >> 1;   // B = g via .trans
  const unsigned halo_s = smem_u32(halo), g_s = smem_u32(gsm);

  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
  {
    int n, x0, y0, z0;
    tile_origin(d, tile, n, x0, y0, z0);
    __syncthreads();
    load_halo(halo, in, d, n, x0, y0, z0, chunk);
    for (int i = threadIdx.x; i < kTileVox * S; i += kThreads)
    {
      const int v = i / S, s = i % S;
      const int x = x0 + (v & 15), y = y0 + ((v >> 4) & 3), z = z0 + (v >> 6);
      uint4     val = make_uint4(0u, 0u, 0u, 0u);
      if (x < d.nx && y < d.ny && z < d.nz)
        val = *reinterpret_cast<const uint4 *>(g + ((((long long)n * d.nz + z) * d.ny + y) * d.nx + x) * COUT + s * 8);
      const int sw = (v / (8 / S)) & (S - 1);
      *reinterpret_cast<uint4 *>(gsm + v * COUT * 2 + ((s ^ sw) << 4)) = val;
    }
    __syncthreads();
#pragma unroll 1
    for (int q = 0; q < 16; q++)
    {
      const int zl = q >> 2, yl = q & 3;
      unsigned  b[NT][2];
#pragma unroll
      for (int jp = 0; jp < NT / 2; jp++)
      {
        const int v = q * 16 + b_vox, s = jp * 2 + b_seg;
        const int sw = (v / (8 / S)) & (S - 1);
        ldsm_x4_t(g_s + v * COUT * 2 + ((s ^ sw) << 4), b[2 * jp][0], b[2 * jp][1], b[2 * jp + 1][0],
                  b[2 * jp + 1][1]);
      }
#pragma unroll
      for (int i = 0; i < 4; i++)
      {
        const int t = warp + 8 * i;
        if (t < 27)
        {
          const int dz = t / 9, dy = (t / 3) % 3, dx = t % 3;
          const int hv = ((zl + dz) * kHY + (yl + dy)) * kHX + dx + a_vox;
          unsigned  a0, a1, a2, a3;
          ldsm_x4_t(halo_s + hv * 32 + ((a_half ^ ((hv >> 2) & 1)) << 4), a0, a1, a2, a3);
#pragma unroll
          for (int j = 0; j < NT; j++)
            mma_bf16(acc[i][j], a0, a1, a2, a3, b[j][0], b[j][1]);
        }
      }
    }
  }
  // flush: c0,c1 at (ci = lane/4, co = 8j + 2(lane%4)), c2,c3 at ci + 8
#pragma unroll
  for (int i = 0; i < 4; i++)
  {
    const int t = warp + 8 * i;
    if (t >= 27)
      continue;
#pragma unroll
    for (int j = 0; j < NT; j++)
#pragma unroll
      for (int k = 0; k < 4; k++)
      {
        const int ci = chunk * 16 + (lane >> 2) + (k >> 1) * 8, co = j * 8 + (lane & 3) * 2 + (k & 1);
        atomicAdd(dW + ((size_t)t * cin_total + ci) * COUT + co, acc[i][j][k]);
      }
  }
}

// ---- weight gradient on the 5th-generation tensor cores -----------------------------------------------
// dW[t][ci][co] += sum_v in[v + t - 1][ci] * g[v][co] as 27 GEMMs per 16-channel input chunk:
// D_t (M rows = output channels, zero-padded to M; N = 16 input channels) += A B_t^T with A = g^T
// (output channels x voxels) and B_t = the chunk's inputs shifted by tap t (input channels x
// voxels), K = the voxels of an 8 x 16 x KZ tile.  Both operands are MN-major in shared memory
// (8 channels contiguous in 16 bytes, voxels 16 bytes apart): the halo in its [k-half][voxel][8
// channels] layout serves every tap -- tap t is a descriptor offset of one halo voxel step in x,
// one halo row in y, one halo plane in z, with the K step of 8 voxels one halo row (160 bytes) --
// and the gradient tile is stored [channel group][voxel][8 channels].  The 27 accumulators (27 x 16
// FP32 columns of tensor memory) stay in tensor memory across the CTA's tiles and are added to dW
// with atomics once, at the end.  A CTA owns an SM (512 tensor-memory columns); one thread issues the
// 27 x (K / 16) MMAs of a tile and commits them to an mbarrier, waited on with a bound before the
// next tile overwrites the operands.
template <int M>
struct WgradTcLayout
{
  static constexpr int kKZ = (M == 64) ? 4 : 2;                // tile depth
  static constexpr int kKV = kCX * kCY * kKZ;                   // voxels per tile (K)
  static constexpr int kHZ = kKZ + 2;
  static constexpr int kHV = kCHX * kCHY * kHZ;                 // halo voxels
  static constexpr int kA = (M / 8) * kKV * 16;                 // A bytes
  static constexpr int kHalo = kHV * 32;                        // two k-halves
  static constexpr int kTotal = kA + kHalo + 16;                // + mbarrier and TMEM slot
};

template <int M>
__device__ __forceinline__ constexpr uint32_t
umma_idesc_bf16_mn16()
{
  // FP32 accumulator, BF16 A and B, both MN-major (bits 15, 16), N = 16, M
  return (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((uint32_t)(16 >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

template <int COUT, int M>
__global__ void __launch_bounds__(128, 1)
conv_wgrad_tc_kernel(ConvIn in, const bf16 * __restrict__ g, Dims d, float * __restrict__ dW, int cin_total)
{
  using L = WgradTcLayout<M>;
  static_assert(COUT <= M && COUT % 8 == 0, "output channels must fit the MMA's M");
  constexpr uint32_t kCols = 512;
  constexpr uint32_t kIdesc = umma_idesc_bf16_mn16<M>();
  extern __shared__ __align__(128) char smem[];
  char *     asm_a = smem;                                   // [M / 8][KV][16 B]
  char *     halo = smem + L::kA;                            // [2][HV][16 B]
  uint64_t * bar = reinterpret_cast<uint64_t *>(halo + L::kHalo);
  uint32_t * tmem_slot = reinterpret_cast<uint32_t *>(bar + 1);
  const int  warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int  chunk = blockIdx.y;
  const int  tx = (d.nx + kCX - 1) / kCX, ty = (d.ny + kCY - 1) / kCY, tz = (d.nz + L::kKZ - 1) / L::kKZ;
  const long long ntiles = (long long)tx * ty * tz * d.batch;

  if (warp == 0)
  {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(rtkb::dev::smem_u32(tmem_slot)),
                 "r"(kCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0)
  {
    rtkb::dev::mbar_init(bar, 1);
    rtkb::dev::fence_barrier_init();
  }
  // the A rows of padding channels (COUT..M-1) stay zero
  for (int i = (COUT / 8) * L::kKV + threadIdx.x; i < (M / 8) * L::kKV; i += 128)
    *reinterpret_cast<uint4 *>(asm_a + i * 16) = make_uint4(0u, 0u, 0u, 0u);
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;
  const uint32_t a_s = rtkb::dev::smem_u32(asm_a), halo_s = rtkb::dev::smem_u32(halo);
  const bool     from_a = chunk * 16 < in.ca;
  const int      cs = from_a ? in.ca : in.cb;
  const int      c0 = from_a ? chunk * 16 : chunk * 16 - in.ca;
  const bf16 *   src = from_a ? in.a : in.b;
  const bool     half = from_a && in.a_half;
  const int      snx = half ? d.nx >> 1 : d.nx, sny = half ? d.ny >> 1 : d.ny, snz = half ? d.nz >> 1 : d.nz;
  // descriptor offsets: A = (K step 128 B, channel groups KV x 16 B), B = (K step one halo row, k-halves)
  const uint32_t a_k = 128u, a_m = (uint32_t)(L::kKV * 16), b_k = (uint32_t)(kCHX * 16), b_n = (uint32_t)(L::kHV * 16);
  bool           ok = true;
  int            it = 0;
  for (long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, it++)
  {
    long long r = tile;
    const int bx = (int)(r % tx);
    r /= tx;
    const int by = (int)(r % ty);
    r /= ty;
    const int bz = (int)(r % tz);
    const int n = (int)(r / tz);
    const int x0 = bx * kCX, y0 = by * kCY, z0 = bz * L::kKZ;
    // the previous tile's MMAs read the operands asynchronously
    if (it > 0)
    {
      ok = __syncthreads_and(rtkb::dev::mbar_wait(bar, (uint32_t)((it - 1) & 1)) ? 1 : 0) != 0;
      if (!ok)
        break;
    }
    for (int i = threadIdx.x; i < L::kHV * 2; i += 128)
    {
      const int hv = i >> 1, h = i & 1;
      const int hx = hv % kCHX, hy = (hv / kCHX) % kCHY, hz = hv / (kCHX * kCHY);
      const int gx = x0 - 1 + hx, gy = y0 - 1 + hy, gz = z0 - 1 + hz;
      uint4     v = make_uint4(0u, 0u, 0u, 0u);
      if (gx >= 0 && gx < d.nx && gy >= 0 && gy < d.ny && gz >= 0 && gz < d.nz)
      {
        const int sx = half ? gx >> 1 : gx, sy = half ? gy >> 1 : gy, sz = half ? gz >> 1 : gz;
        v = *reinterpret_cast<const uint4 *>(src + ((((long long)n * snz + sz) * sny + sy) * snx + sx) * cs + c0 + h * 8);
      }
      *reinterpret_cast<uint4 *>(halo + (h * L::kHV + hv) * 16) = v;
    }
    for (int i = threadIdx.x; i < L::kKV * (COUT / 8); i += 128)
    {
      const int v = i / (COUT / 8), cg = i % (COUT / 8);
      const int x = x0 + (v & 7), y = y0 + ((v >> 3) & 15), z = z0 + (v >> 7);
      uint4     val = make_uint4(0u, 0u, 0u, 0u);
      if (x < d.nx && y < d.ny && z < d.nz)
        val = *reinterpret_cast<const uint4 *>(g + ((((long long)n * d.nz + z) * d.ny + y) * d.nx + x) * COUT + cg * 8);
      *reinterpret_cast<uint4 *>(asm_a + (cg * L::kKV + v) * 16) = val;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0)
    {
      asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll 1
      for (int t = 0; t < 27; t++)
      {
        const int dz = t / 9, dy = (t / 3) % 3, dx = t % 3;
#pragma unroll 1
        for (int zl = 0; zl < L::kKZ; zl++)
#pragma unroll
          for (int yp = 0; yp < kCY / 2; yp++)
          {
            const int      kv0 = (zl * kCY + 2 * yp) * kCX;
            const int      hv0 = ((zl + dz) * kCHY + 2 * yp + dy) * kCHX + dx;
            // MN-major, no swizzle: leading offset = the K step between 8-voxel core matrices,
            // stride offset = the step between 8-channel groups
            const uint64_t da = umma_desc(a_s + (uint32_t)(kv0 * 16), a_k, a_m);
            const uint64_t db = umma_desc(halo_s + (uint32_t)(hv0 * 16), b_k, b_n);
            umma_bf16(tmem + (uint32_t)(t * 16), da, db, kIdesc, (it > 0 || zl > 0 || yp > 0) ? 1u : 0u);
          }
      }
      umma_commit(bar);
    }
  }
  if (ok && it > 0)
    ok = __syncthreads_and(rtkb::dev::mbar_wait(bar, (uint32_t)((it - 1) & 1)) ? 1 : 0) != 0;
  asm volatile("tcgen05.fence::after_thread_sync;");
  // epilogue: row m of D is output channel m; with M = 128 row m sits in TMEM lane m, with M = 64
  // rows 16w..16w+15 sit in lanes 32w..32w+15
  if (ok && it > 0)
  {
    const int co = (M == 128) ? warp * 32 + lane : (lane < 16 ? warp * 16 + lane : COUT);
#pragma unroll 1
    for (int t = 0; t < 27; t++)
    {
      uint32_t r[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(t * 16), r);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (co < COUT)
#pragma unroll
        for (int c = 0; c < 16; c++)
          atomicAdd(dW + ((size_t)t * cin_total + chunk * 16 + c) * COUT + co, __uint_as_float(r[c]));
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols));
}

// ---- first layer (1 -> 16, CUDA cores) ----------------------------------------------------------------
// out[v][co] = relu( sum_t x[v + t - 1] * inv_s * W1[t][co] )
__global__ void __launch_bounds__(256)
first_fwd_kernel(const float * __restrict__ x, const float * __restrict__ scale, const float * __restrict__ W1, Dims d,
                 bf16 * __restrict__ out)
{
  __shared__ float w[27 * 16];
  for (int i = threadIdx.x; i < 27 * 16; i += blockDim.x)
    w[i] = W1[i];
  __syncthreads();
  const long long nv = d.vox() * d.batch;
  const float     inv_s = scale[1];
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nv; v += (long long)gridDim.x * blockDim.x)
  {
    const int       xi = (int)(v % d.nx), yi = (int)((v / d.nx) % d.ny), zi = (int)((v / ((long long)d.nx * d.ny)) % d.nz);
    const long long base = v - ((long long)zi * d.ny + yi) * d.nx - xi; // start of this batch volume
    float           acc[16];
#pragma unroll
    for (int c = 0; c < 16; c++)
      acc[c] = 0.f;
    for (int t = 0; t < 27; t++)
    {
      const int gx = xi + t % 3 - 1, gy = yi + (t / 3) % 3 - 1, gz = zi + t / 9 - 1;
      if (gx < 0 || gx >= d.nx || gy < 0 || gy >= d.ny || gz < 0 || gz >= d.nz)
        continue;
      const float xv = x[base + ((long long)gz * d.ny + gy) * d.nx + gx];
#pragma unroll
      for (int c = 0; c < 16; c++)
        acc[c] = fmaf(xv, w[t * 16 + c], acc[c]);
    }
    unsigned p[8];
#pragma unroll
    for (int c = 0; c < 8; c++)
      p[c] = pack_bf16x2(fmaxf(acc[2 * c] * inv_s, 0.f), fmaxf(acc[2 * c + 1] * inv_s, 0.f));
    uint4 * o = reinterpret_cast<uint4 *>(out + v * 16);
    o[0] = make_uint4(p[0], p[1], p[2], p[3]);
    o[1] = make_uint4(p[4], p[5], p[6], p[7]);
  }
}

// dW1[t][co] += sum_v x[v + t - 1] * inv_s * g[v][co]
__global__ void __launch_bounds__(256)
first_wgrad_kernel(const float * __restrict__ x, const float * __restrict__ scale, const bf16 * __restrict__ g, Dims d,
                   float * __restrict__ dW1)
{
  __shared__ float xh[kHalo];
  __shared__ float gs[kTileVox * 17];
  const long long  ntiles = (long long)d.tx * d.ty * d.tz * d.batch;
  const float      inv_s = scale[1];
  float            part[2] = { 0.f, 0.f };
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
  {
    int n, x0, y0, z0;
    tile_origin(d, tile, n, x0, y0, z0);
    __syncthreads();
    for (int hv = threadIdx.x; hv < kHalo; hv += blockDim.x)
    {
      const int gx = x0 - 1 + hv % kHX, gy = y0 - 1 + (hv / kHX) % kHY, gz = z0 - 1 + hv / (kHX * kHY);
      float     v = 0.f;
      if (gx >= 0 && gx < d.nx && gy >= 0 && gy < d.ny && gz >= 0 && gz < d.nz)
        v = x[(((long long)n * d.nz + gz) * d.ny + gy) * d.nx + gx] * inv_s;
      xh[hv] = v;
    }
    for (int i = threadIdx.x; i < kTileVox * 16; i += blockDim.x)
    {
      const int v = i >> 4, c = i & 15;
      const int xx = x0 + (v & 15), yy = y0 + ((v >> 4) & 3), zz = z0 + (v >> 6);
      float     val = 0.f;
      if (xx < d.nx && yy < d.ny && zz < d.nz)
        val = __bfloat162float(g[((((long long)n * d.nz + zz) * d.ny + yy) * d.nx + xx) * 16 + c]);
      gs[v * 17 + c] = val;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 2; k++)
    {
      const int o = threadIdx.x + k * 256;
      if (o >= 27 * 16)
        continue;
      const int t = o >> 4, c = o & 15;
      const int dz = t / 9, dy = (t / 3) % 3, dx = t % 3;
      float     s = 0.f;
      for (int v = 0; v < kTileVox; v++)
      {
        const int hv = (((v >> 6) + dz) * kHY + ((v >> 4) & 3) + dy) * kHX + (v & 15) + dx;
        s = fmaf(xh[hv], gs[v * 17 + c], s);
      }
      part[k] += s;
    }
  }
#pragma unroll
  for (int k = 0; k < 2; k++)
  {
    const int o = threadIdx.x + k * 256;
    if (o < 27 * 16)
      atomicAdd(dW1 + o, part[k]);
  }
}

// ---- last layer (16 -> 1, 1x1x1) ------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
last_fwd_kernel(const bf16 * __restrict__ y, const float * __restrict__ W, const float * __restrict__ scale,
                float * __restrict__ out, long long nv)
{
  float w[16];
#pragma unroll
  for (int c = 0; c < 16; c++)
    w[c] = W[c];
  const float s = scale[0];
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nv; v += (long long)gridDim.x * blockDim.x)
  {
    const uint4 * p = reinterpret_cast<const uint4 *>(y + v * 16);
    const uint4   q0 = p[0], q1 = p[1];
    const unsigned u[8] = { q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w };
    float          acc = 0.f;
#pragma unroll
    for (int c = 0; c < 8; c++)
    {
      const float2 f = unpack_bf16x2(u[c]);
      acc = fmaf(f.x, w[2 * c], acc);
      acc = fmaf(f.y, w[2 * c + 1], acc);
    }
    out[v] = acc * s;
  }
}

// Loss (mean squared error, scale 1) and the first backward step, over the
// voxels at least `margin` voxels inside every face of each batch volume
// (count of them: cnt): dout = 2 (out - tgt) / cnt; g[v][c] = W[c] dout
// (y > 0); dW[c] += y[v][c] dout.  Voxels in the margin get dout = 0.
__global__ void __launch_bounds__(256)
last_bwd_kernel(const bf16 * __restrict__ y, const float * __restrict__ W, const float * __restrict__ out,
                const float * __restrict__ tgt, Dims d, int margin, double cnt, bf16 * __restrict__ g,
                float * __restrict__ dW, double * __restrict__ loss)
{
  float w[16], dw[16];
#pragma unroll
  for (int c = 0; c < 16; c++)
  {
    w[c] = W[c];
    dw[c] = 0.f;
  }
  double          l = 0.;
  const float     inv_n2 = (float)(2. / cnt);
  const long long nv = d.vox() * d.batch;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nv; v += (long long)gridDim.x * blockDim.x)
  {
    const int  xi = (int)(v % d.nx), yi = (int)((v / d.nx) % d.ny), zi = (int)((v / ((long long)d.nx * d.ny)) % d.nz);
    const bool in = xi >= margin && xi < d.nx - margin && yi >= margin && yi < d.ny - margin && zi >= margin &&
                    zi < d.nz - margin;
    const float    diff = in ? out[v] - tgt[v] : 0.f;
    const float    dout = diff * inv_n2;
    l += (double)diff * diff;
    const uint4 *  p = reinterpret_cast<const uint4 *>(y + v * 16);
    const uint4    q0 = p[0], q1 = p[1];
    const unsigned u[8] = { q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w };
    unsigned       o[8];
#pragma unroll
    for (int c = 0; c < 8; c++)
    {
      const float2 f = unpack_bf16x2(u[c]);
      dw[2 * c] = fmaf(f.x, dout, dw[2 * c]);
      dw[2 * c + 1] = fmaf(f.y, dout, dw[2 * c + 1]);
      o[c] = pack_bf16x2(f.x > 0.f ? w[2 * c] * dout : 0.f, f.y > 0.f ? w[2 * c + 1] * dout : 0.f);
    }
    uint4 * go = reinterpret_cast<uint4 *>(g + v * 16);
    go[0] = make_uint4(o[0], o[1], o[2], o[3]);
    go[1] = make_uint4(o[4], o[5], o[6], o[7]);
  }
  __shared__ float  sw[8][16];
  __shared__ double sl[8];
  const int         lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < 16; c++)
  {
    float s = dw[c];
#pragma unroll
    for (int k = 16; k > 0; k >>= 1)
      s += __shfl_xor_sync(0xffffffffu, s, k);
    if (lane == 0)
      sw[warp][c] = s;
  }
#pragma unroll
  for (int k = 16; k > 0; k >>= 1)
    l += __shfl_xor_sync(0xffffffffu, l, k);
  if (lane == 0)
    sl[warp] = l;
  __syncthreads();
  if (threadIdx.x < 16)
  {
    float s = 0.f;
    for (int k = 0; k < 8; k++)
      s += sw[k][threadIdx.x];
    atomicAdd(dW + threadIdx.x, s);
  }
  if (threadIdx.x == 0)
  {
    double s = 0.;
    for (int k = 0; k < 8; k++)
      s += sl[k];
    atomicAdd(loss, s);
  }
}

// ---- pooling and the gradients of the skip / up-sampling wiring ---------------------------------------------
// out[u][c] = mean of the 8 children of u; one thread per (u, 8 channels)
__global__ void __launch_bounds__(256)
pool_kernel(const bf16 * __restrict__ in, int C, Dims full, bf16 * __restrict__ out)
{
  const int       hx = full.nx >> 1, hy = full.ny >> 1, hz = full.nz >> 1, G = C / 8;
  const long long n = (long long)hx * hy * hz * full.batch * G;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
  {
    const int g = (int)(i % G);
    long long u = i / G;
    const int x = (int)(u % hx), y = (int)((u / hx) % hy), z = (int)((u / ((long long)hx * hy)) % hz);
    const int b = (int)(u / ((long long)hx * hy * hz));
    float     s[8] = { 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f };
#pragma unroll
    for (int k = 0; k < 8; k++)
    {
      const long long v = (((long long)b * full.nz + 2 * z + (k >> 2)) * full.ny + 2 * y + ((k >> 1) & 1)) * full.nx + 2 * x + (k & 1);
      const uint4     q = *reinterpret_cast<const uint4 *>(in + v * C + g * 8);
      const unsigned  w[4] = { q.x, q.y, q.z, q.w };
#pragma unroll
      for (int c = 0; c < 4; c++)
      {
        const float2 f = unpack_bf16x2(w[c]);
        s[2 * c] += f.x;
        s[2 * c + 1] += f.y;
      }
    }
    *reinterpret_cast<uint4 *>(out + u * C + g * 8) =
      make_uint4(pack_bf16x2(s[0] * .125f, s[1] * .125f), pack_bf16x2(s[2] * .125f, s[3] * .125f),
                 pack_bf16x2(s[4] * .125f, s[5] * .125f), pack_bf16x2(s[6] * .125f, s[7] * .125f));
  }
}

// Gradient of the up-sampled half of a concatenated input: out[u][c] = (sum
// over the 8 children of cat[child][c]) * (y[u][c] > 0), c < ca.
__global__ void __launch_bounds__(256)
up_grad_kernel(const bf16 * __restrict__ cat, int ccat, int ca, const bf16 * __restrict__ y, Dims full,
               bf16 * __restrict__ out)
{
  const int       hx = full.nx >> 1, hy = full.ny >> 1, hz = full.nz >> 1, G = ca / 8;
  const long long n = (long long)hx * hy * hz * full.batch * G;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
  {
    const int g = (int)(i % G);
    long long u = i / G;
    const int x = (int)(u % hx), yy = (int)((u / hx) % hy), z = (int)((u / ((long long)hx * hy)) % hz);
    const int b = (int)(u / ((long long)hx * hy * hz));
    float     s[8] = { 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f };
#pragma unroll
    for (int k = 0; k < 8; k++)
    {
      const long long v = (((long long)b * full.nz + 2 * z + (k >> 2)) * full.ny + 2 * yy + ((k >> 1) & 1)) * full.nx + 2 * x + (k & 1);
      const uint4     q = *reinterpret_cast<const uint4 *>(cat + v * ccat + g * 8);
      const unsigned  w[4] = { q.x, q.y, q.z, q.w };
#pragma unroll
      for (int c = 0; c < 4; c++)
      {
        const float2 f = unpack_bf16x2(w[c]);
        s[2 * c] += f.x;
        s[2 * c + 1] += f.y;
      }
    }
    const uint4    m = *reinterpret_cast<const uint4 *>(y + u * ca + g * 8);
    const unsigned mw[4] = { m.x, m.y, m.z, m.w };
    unsigned       o[4];
#pragma unroll
    for (int c = 0; c < 4; c++)
    {
      const float2 f = unpack_bf16x2(mw[c]);
      o[c] = pack_bf16x2(f.x > 0.f ? s[2 * c] : 0.f, f.y > 0.f ? s[2 * c + 1] : 0.f);
    }
    *reinterpret_cast<uint4 *>(out + u * ca + g * 8) = make_uint4(o[0], o[1], o[2], o[3]);
  }
}

// Gradient of a skip tensor (used by the concatenation and by the pooling):
// out[v][c] = (cat[v][ca + c] + pgrad[parent(v)][c] / 8) * (y[v][c] > 0).
__global__ void __launch_bounds__(256)
skip_grad_kernel(const bf16 * __restrict__ cat, int ccat, int ca, const bf16 * __restrict__ pgrad,
                 const bf16 * __restrict__ y, int cb, Dims full, bf16 * __restrict__ out)
{
  const int       G = cb / 8, hx = full.nx >> 1, hy = full.ny >> 1, hz = full.nz >> 1;
  const long long n = full.vox() * full.batch * G;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
  {
    const int       g = (int)(i % G);
    const long long v = i / G;
    const int x = (int)(v % full.nx), yy = (int)((v / full.nx) % full.ny), z = (int)((v / ((long long)full.nx * full.ny)) % full.nz);
    const int b = (int)(v / full.vox());
    const long long u = (((long long)b * hz + (z >> 1)) * hy + (yy >> 1)) * hx + (x >> 1);
    const uint4 qc = *reinterpret_cast<const uint4 *>(cat + v * ccat + ca + g * 8);
    const uint4 qp = *reinterpret_cast<const uint4 *>(pgrad + u * cb + g * 8);
    const uint4 qm = *reinterpret_cast<const uint4 *>(y + v * cb + g * 8);
    const unsigned wc[4] = { qc.x, qc.y, qc.z, qc.w }, wp[4] = { qp.x, qp.y, qp.z, qp.w },
                   wm[4] = { qm.x, qm.y, qm.z, qm.w };
    unsigned o[4];
#pragma unroll
    for (int c = 0; c < 4; c++)
    {
      const float2 fc = unpack_bf16x2(wc[c]), fp = unpack_bf16x2(wp[c]), fm = unpack_bf16x2(wm[c]);
      o[c] = pack_bf16x2(fm.x > 0.f ? fmaf(fp.x, .125f, fc.x) : 0.f, fm.y > 0.f ? fmaf(fp.y, .125f, fc.y) : 0.f);
    }
    *reinterpret_cast<uint4 *>(out + v * cb + g * 8) = make_uint4(o[0], o[1], o[2], o[3]);
  }
}

// ---- weights: packing, Adam ------------------------------------------------------------------------------
// Forward pack for the tensor-core kernel: wf[c][t][h][co][8] = W[t][16c + 8h + j][co]
// (input chunk c, k-half h, j < 8).  Data-gradient pack (input channels = co,
// output channels = ci, taps mirrored): wd[c'][t][h][ci][8] = W[26 - t][ci][16c' + 8h + j].
__global__ void
pack_kernel(const float * __restrict__ W, int cin, int cout, bf16 * __restrict__ wf, bf16 * __restrict__ wd)
{
  const int n = 27 * cin * cout;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
  {
    const int  co = i % cout, ci = (i / cout) % cin, t = i / (cout * cin);
    const bf16 w = __float2bfloat16_rn(W[i]);
    {
      const int c = ci >> 4, h = (ci >> 3) & 1, j = ci & 7;
      wf[((((size_t)c * 27 + t) * 2 + h) * cout + co) * 8 + j] = w;
    }
    {
      const int c = co >> 4, h = (co >> 3) & 1, j = co & 7;
      wd[((((size_t)c * 27 + (26 - t)) * 2 + h) * cin + ci) * 8 + j] = w;
    }
  }
}

__global__ void
adam_kernel(float * __restrict__ w, const float * __restrict__ g, float * __restrict__ m, float * __restrict__ v, int n,
            float lr, float b1, float b2, float c1, float c2, float eps)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
  {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  }
}

// scale[0] = s = rms(x) (1 when x is zero), scale[1] = 1/s; unit = 1 gives s = 1
constexpr int kScaleBlocks = 148 * 2;
__global__ void __launch_bounds__(256)
sumsq_kernel(const float * __restrict__ x, long long n, double * __restrict__ part)
{
  double s = 0.;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    s = fma((double)x[i], (double)x[i], s);
  __shared__ double sh[8];
#pragma unroll
  for (int k = 16; k > 0; k >>= 1)
    s += __shfl_xor_sync(0xffffffffu, s, k);
  if ((threadIdx.x & 31) == 0)
    sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0)
  {
    double t = 0.;
    for (int k = 0; k < 8; k++)
      t += sh[k];
    part[blockIdx.x] = t;
  }
}

__global__ void
scale_kernel(const double * __restrict__ part, long long n, float * __restrict__ scale, int unit)
{
  if (threadIdx.x != 0)
    return;
  if (unit)
  {
    scale[0] = scale[1] = 1.f;
    return;
  }
  double s = 0.;
  for (int k = 0; k < kScaleBlocks; k++)
    s += part[k];
  const double r = s > 0. ? sqrt(s / (double)n) : 1.;
  scale[0] = (float)r;
  scale[1] = (float)(1. / r);
}

unsigned
grid1(long long n)
{
  return (unsigned)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148LL * 8));
}

// ---- layer table -------------------------------------------------------------------------------------------
struct Layer
{
  int cin, cout, level;
};
constexpr Layer kLayers[11] = { { 1, 16, 0 },  { 16, 16, 0 }, { 16, 32, 1 }, { 32, 32, 1 },
                                { 32, 64, 2 }, { 64, 64, 2 }, { 96, 32, 1 }, { 32, 32, 1 },
                                { 48, 16, 0 }, { 16, 16, 0 }, { 16, 1, 0 } };

long long
layer_params(int l)
{
  return l == 10 ? 16 : 27LL * kLayers[l].cin * kLayers[l].cout;
}

// Dynamic shared memory for a tcgen05 kernel that holds `cols` TMEM columns:
// at least `need`, and enough that the CTAs one SM can hold never ask for more
// than the SM's 512 columns (tcgen05.alloc would otherwise wait for another
// CTA to release its columns).
int
tmem_bounded_smem(int need, int cols)
{
  constexpr int kSmemPerSm = 228 * 1024, kReservedPerCta = 1024;
  const int     max_ctas = 512 / cols;
  const int     floor_bytes = kSmemPerSm / (max_ctas + 1) - kReservedPerCta + 16;
  return std::max(need, floor_bytes);
}

// Convolution kernel (rtkb_unet_set_conv_pipeline): 0 = thread-loaded halo,
// one stage; 1 = TMA-loaded halo, one stage (default); 2 = TMA-loaded halo,
// two stages (the widest data-gradient layers, whose two stages do not fit in
// shared memory, use one).
int g_conv_pipeline = 1;

constexpr int
tmem_cols(int n)
{
  return (n <= 32) ? 32 : (n <= 64) ? 64 : (n <= 128) ? 128 : (n <= 256) ? 256 : 512;
}

// 5-D TMA descriptor of an activation [batch][z][y][x][c] at full resolution,
// box 8 channels x the 10 x 18 x 6 halo; false if it cannot be encoded.
bool
encode_activation_map(CUtensorMap & map, const bf16 * base, int c, int nx, int ny, int nz, int batch)
{
  std::memset(&map, 0, sizeof(map));
  rtkb::EncodeTiledFn enc = rtkb::tensor_map_encoder();
  if (!enc || !base || (reinterpret_cast<uintptr_t>(base) % 16) != 0 || (c * 2) % 16 != 0)
    return false;
  const unsigned long long e = 2;
  const unsigned long long dims[5] = { (unsigned long long)c, (unsigned long long)nx, (unsigned long long)ny,
                                       (unsigned long long)nz, (unsigned long long)batch };
  const unsigned long long strides[4] = { c * e, c * e * nx, c * e * nx * ny, c * e * nx * ny * nz };
  const unsigned           box[5] = { 8u, (unsigned)kCHX, (unsigned)kCHY, (unsigned)kCHZ, 1u };
  const unsigned           estr[5] = { 1u, 1u, 1u, 1u, 1u };
  return enc(&map, (int)CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5u, const_cast<bf16 *>(base), dims, strides, box, estr,
             (int)CU_TENSOR_MAP_INTERLEAVE_NONE, (int)CU_TENSOR_MAP_SWIZZLE_NONE, (int)CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             (int)CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == 0;
}

template <int N, int NS>
void
conv_fwd_pipe_launch(const ConvIn & in, const bf16 * wp, const Dims & d0, bf16 * out, const bf16 * mask, int relu,
                     cudaStream_t st)
{
  using L = PipeLayout<N, NS>;
  const int   smem = tmem_bounded_smem(L::kTotal, tmem_cols(kCZ * N));
  static bool configured = false; // attribute set once per process (same value on every device)
  if (!configured)
  {
    cudaFuncSetAttribute(conv_fwd_pipe_kernel<N, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    configured = true;
  }
  CUtensorMap ma, mb;
  const int   ta = (in.ca > 0 && !in.a_half) ? (encode_activation_map(ma, in.a, in.ca, d0.nx, d0.ny, d0.nz, d0.batch) ? 1 : 0) : 0;
  const int   tb = in.cb > 0 ? (encode_activation_map(mb, in.b, in.cb, d0.nx, d0.ny, d0.nz, d0.batch) ? 1 : 0) : 0;
  if (!ta)
    std::memset(&ma, 0, sizeof(ma));
  if (!tb)
    std::memset(&mb, 0, sizeof(mb));
  const TcDims    d = make_tc_dims(d0.nx, d0.ny, d0.nz, d0.batch);
  const long long tiles = (long long)d.tx * d.ty * d.tz * d.batch;
  conv_fwd_pipe_kernel<N, NS><<<(unsigned)tiles, 128, smem, st>>>(ma, mb, ta, tb, in, wp, d, out, mask, relu);
}

template <int N>
void
conv_fwd_tc_launch(const ConvIn & in, const bf16 * wp, const Dims & d0, bf16 * out, const bf16 * mask, int relu,
                   cudaStream_t st)
{
  if (g_conv_pipeline == 1)
  {
    conv_fwd_pipe_launch<N, 1>(in, wp, d0, out, mask, relu, st);
    return;
  }
  if constexpr (PipeLayout<N, 2>::kTotal <= 227 * 1024)
  {
    if (g_conv_pipeline == 2)
    {
      conv_fwd_pipe_launch<N, 2>(in, wp, d0, out, mask, relu, st);
      return;
    }
  }
  const int smem = tmem_bounded_smem(kCHaloBytes + 27 * 2 * N * 16 + 16, tmem_cols(kCZ * N));
  static bool configured = false; // attribute set once per process (same value on every device)
  if (!configured)
  {
    cudaFuncSetAttribute(conv_fwd_tc_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    configured = true;
  }
  const TcDims    d = make_tc_dims(d0.nx, d0.ny, d0.nz, d0.batch);
  const long long tiles = (long long)d.tx * d.ty * d.tz * d.batch;
  conv_fwd_tc_kernel<N><<<(unsigned)tiles, 128, smem, st>>>(in, wp, d, out, mask, relu);
}

template <int NT>
void
conv_wgrad_launch(const ConvIn & in, const bf16 * g, const Dims & d, float * dW, cudaStream_t st)
{
  const int smem = kHaloBytes + kTileVox * NT * 8 * 2;
  static bool configured = false;
  if (!configured)
  {
    cudaFuncSetAttribute(conv_wgrad_kernel<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    configured = true;
  }
  const long long tiles = (long long)d.tx * d.ty * d.tz * d.batch;
  const unsigned  gx = (unsigned)std::min<long long>(tiles, 148LL * 2);
  const dim3      grid(gx, (unsigned)((in.ca + in.cb) / 16));
  conv_wgrad_kernel<NT><<<grid, kThreads, smem, st>>>(in, g, d, dW, in.ca + in.cb);
}

void
conv_fwd(int cout, const ConvIn & in, const bf16 * wp, const Dims & d, bf16 * out, const bf16 * mask, int relu,
         cudaStream_t st)
{
  switch (cout)
  {
  case 16: conv_fwd_tc_launch<16>(in, wp, d, out, mask, relu, st); break;
  case 32: conv_fwd_tc_launch<32>(in, wp, d, out, mask, relu, st); break;
  case 48: conv_fwd_tc_launch<48>(in, wp, d, out, mask, relu, st); break;
  case 64: conv_fwd_tc_launch<64>(in, wp, d, out, mask, relu, st); break;
  default: conv_fwd_tc_launch<96>(in, wp, d, out, mask, relu, st); break;
  }
}

// Weight-gradient kernel (rtkb_unet_set_wgrad_kernel): 0 = warp-level mma.sync; 1 = tcgen05 with
// M = 64 (tiles of 8 x 16 x 4 voxels); 2 = tcgen05 with M = 128 (tiles of 8 x 16 x 2 voxels).
int g_wgrad_kernel = 0;

template <int COUT, int M>
void
conv_wgrad_tc_launch(const ConvIn & in, const bf16 * g, const Dims & d, float * dW, cudaStream_t st)
{
  using L = WgradTcLayout<M>;
  const int   smem = tmem_bounded_smem(L::kTotal, 512);
  static bool configured = false;
  if (!configured)
  {
    cudaFuncSetAttribute(conv_wgrad_tc_kernel<COUT, M>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    configured = true;
  }
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int       nchunks = (in.ca + in.cb) / 16;
  const long long tiles = (long long)((d.nx + kCX - 1) / kCX) * ((d.ny + kCY - 1) / kCY) *
                          ((d.nz + L::kKZ - 1) / L::kKZ) * d.batch;
  const unsigned  gx = (unsigned)std::max<long long>(1, std::min<long long>(tiles, std::max(1, sms / nchunks)));
  conv_wgrad_tc_kernel<COUT, M><<<dim3(gx, (unsigned)nchunks), 128, smem, st>>>(in, g, d, dW, in.ca + in.cb);
}

template <int COUT>
void
conv_wgrad_dispatch(const ConvIn & in, const bf16 * g, const Dims & d, float * dW, cudaStream_t st)
{
  if (g_wgrad_kernel == 1)
    conv_wgrad_tc_launch<COUT, 64>(in, g, d, dW, st);
  else if (g_wgrad_kernel == 2)
    conv_wgrad_tc_launch<COUT, 128>(in, g, d, dW, st);
  else
    conv_wgrad_launch<COUT / 8>(in, g, d, dW, st);
}

void
conv_wgrad(int cout, const ConvIn & in, const bf16 * g, const Dims & d, float * dW, cudaStream_t st)
{
  switch (cout)
  {
  case 16: conv_wgrad_dispatch<16>(in, g, d, dW, st); break;
  case 32: conv_wgrad_dispatch<32>(in, g, d, dW, st); break;
  default: conv_wgrad_dispatch<64>(in, g, d, dW, st); break;
  }
}

ConvIn
plain(const bf16 * a, int c)
{
  return ConvIn{ a, nullptr, c, 0, 0 };
}

ConvIn
upcat(const bf16 * a, int ca, const bf16 * b, int cb)
{
  return ConvIn{ a, b, ca, cb, 1 };
}

} // namespace

struct rtkb_unet
{
  long long nparams = 0;
  long long off[11] = {};
  void *    pmem = nullptr; // params | grads | adam m | adam v | packed BF16 weights
  float *   W = nullptr, *G = nullptr, *M = nullptr, *V = nullptr;
  bf16 *    wf[11] = {}, *wd[11] = {};
  float *   scale = nullptr;
  double *  part = nullptr, *loss = nullptr;
  int       step = 0;
  // activation workspace
  void *    fmem = nullptr;
  size_t    fbytes = 0;
  int       fdims[4] = { 0, 0, 0, 0 };
  bf16 *    e1a = nullptr, *e1 = nullptr, *p1 = nullptr, *e2a = nullptr, *e2 = nullptr, *p2 = nullptr, *b1 = nullptr,
       *b2 = nullptr, *d2a = nullptr, *d2 = nullptr, *d1a = nullptr, *d1 = nullptr;
  float * out = nullptr;
  // gradient workspace (training)
  void * gmem = nullptr;
  size_t gbytes = 0;
  bf16 * G0a = nullptr, *G0b = nullptr, *Gc0 = nullptr, *G1a = nullptr, *G1b = nullptr, *Gc1 = nullptr, *G2a = nullptr,
       *G2b = nullptr, *Gp2 = nullptr, *Gp1 = nullptr;
};

namespace
{

using rtkb::cuda_fail;
using rtkb::fail;

int
check_dims(int batch, int nx, int ny, int nz)
{
  if (batch < 1 || nx < 4 || ny < 4 || nz < 4 || (nx & 3) || (ny & 3) || (nz & 3))
    return fail(RTKB_ERR_INVALID_ARGUMENT, "U-Net volumes need sizes that are multiples of 4 (two 2x2x2 poolings)");
  if ((long long)nx * ny * nz * batch > (1LL << 31) / 2)
    return fail(RTKB_ERR_UNSUPPORTED, "U-Net batch too large for one call");
  return RTKB_OK;
}

int
reserve_forward(rtkb_unet * u, int batch, int nx, int ny, int nz)
{
  if (u->fmem && u->fdims[0] == batch && u->fdims[1] == nx && u->fdims[2] == ny && u->fdims[3] == nz)
    return RTKB_OK;
  const long long v0 = (long long)nx * ny * nz * batch, v1 = v0 / 8, v2 = v1 / 8;
  auto            up = [](size_t b) { return (b + 255) & ~size_t(255); };
  const size_t    sizes[13] = { up(v0 * 32), up(v0 * 32), up(v1 * 32), up(v1 * 64), up(v1 * 64), up(v2 * 64),
                                up(v2 * 128), up(v2 * 128), up(v1 * 64), up(v1 * 64), up(v0 * 32), up(v0 * 32),
                                up(v0 * 4) };
  size_t          total = 0;
  for (size_t s : sizes)
    total += s;
  if (u->fmem)
    cudaFree(u->fmem);
  u->fmem = nullptr;
  u->fdims[0] = 0;
  cudaError_t e = cudaMalloc(&u->fmem, total);
  if (e != cudaSuccess)
    return cuda_fail(e, "cudaMalloc (U-Net activations)");
  u->fbytes = total;
  char * m = static_cast<char *>(u->fmem);
  bf16 ** ptrs[12] = { &u->e1a, &u->e1, &u->p1, &u->e2a, &u->e2, &u->p2, &u->b1, &u->b2, &u->d2a, &u->d2, &u->d1a, &u->d1 };
  for (int i = 0; i < 12; i++)
  {
    *ptrs[i] = reinterpret_cast<bf16 *>(m);
    m += sizes[i];
  }
  u->out = reinterpret_cast<float *>(m);
  u->fdims[0] = batch;
  u->fdims[1] = nx;
  u->fdims[2] = ny;
  u->fdims[3] = nz;
  if (u->gmem)
  {
    cudaFree(u->gmem);
    u->gmem = nullptr;
  }
  return RTKB_OK;
}

int
reserve_backward(rtkb_unet * u)
{
  if (u->gmem)
    return RTKB_OK;
  const long long v0 = (long long)u->fdims[1] * u->fdims[2] * u->fdims[3] * u->fdims[0], v1 = v0 / 8, v2 = v1 / 8;
  auto            up = [](size_t b) { return (b + 255) & ~size_t(255); };
  const size_t    sizes[10] = { up(v0 * 32), up(v0 * 32), up(v0 * 96), up(v1 * 64), up(v1 * 64),
                                up(v1 * 192), up(v2 * 128), up(v2 * 128), up(v2 * 64), up(v1 * 32) };
  size_t          total = 0;
  for (size_t s : sizes)
    total += s;
  cudaError_t e = cudaMalloc(&u->gmem, total);
  if (e != cudaSuccess)
    return cuda_fail(e, "cudaMalloc (U-Net gradients)");
  u->gbytes = total;
  char * m = static_cast<char *>(u->gmem);
  bf16 ** ptrs[10] = { &u->G0a, &u->G0b, &u->Gc0, &u->G1a, &u->G1b, &u->Gc1, &u->G2a, &u->G2b, &u->Gp2, &u->Gp1 };
  for (int i = 0; i < 10; i++)
  {
    *ptrs[i] = reinterpret_cast<bf16 *>(m);
    m += sizes[i];
  }
  return RTKB_OK;
}

cudaError_t
repack(rtkb_unet * u, cudaStream_t st)
{
  for (int l = 1; l < 10; l++)
    pack_kernel<<<grid1(layer_params(l)), 256, 0, st>>>(u->W + u->off[l], kLayers[l].cin, kLayers[l].cout, u->wf[l],
                                                        u->wd[l]);
  return cudaGetLastError();
}

// Forward pass over the reserved workspace; normalize: divide the input by
// its rms and multiply the output by it.
cudaError_t
forward(rtkb_unet * u, const float * in, float * out, int normalize, cudaStream_t st)
{
  const int  B = u->fdims[0], nx = u->fdims[1], ny = u->fdims[2], nz = u->fdims[3];
  const Dims d0 = make_dims(nx, ny, nz, B), d1 = make_dims(nx / 2, ny / 2, nz / 2, B),
             d2 = make_dims(nx / 4, ny / 4, nz / 4, B);
  const long long v0 = d0.vox() * B;
  if (normalize)
    sumsq_kernel<<<kScaleBlocks, 256, 0, st>>>(in, v0, u->part);
  scale_kernel<<<1, 32, 0, st>>>(u->part, v0, u->scale, normalize ? 0 : 1);
  first_fwd_kernel<<<grid1(v0), 256, 0, st>>>(in, u->scale, u->W + u->off[0], d0, u->e1a);
  conv_fwd(16, plain(u->e1a, 16), u->wf[1], d0, u->e1, nullptr, 1, st);
  pool_kernel<<<grid1(v0 / 8 * 2), 256, 0, st>>>(u->e1, 16, d0, u->p1);
  conv_fwd(32, plain(u->p1, 16), u->wf[2], d1, u->e2a, nullptr, 1, st);
  conv_fwd(32, plain(u->e2a, 32), u->wf[3], d1, u->e2, nullptr, 1, st);
  pool_kernel<<<grid1(v0 / 64 * 4), 256, 0, st>>>(u->e2, 32, d1, u->p2);
  conv_fwd(64, plain(u->p2, 32), u->wf[4], d2, u->b1, nullptr, 1, st);
  conv_fwd(64, plain(u->b1, 64), u->wf[5], d2, u->b2, nullptr, 1, st);
  conv_fwd(32, upcat(u->b2, 64, u->e2, 32), u->wf[6], d1, u->d2a, nullptr, 1, st);
  conv_fwd(32, plain(u->d2a, 32), u->wf[7], d1, u->d2, nullptr, 1, st);
  conv_fwd(16, upcat(u->d2, 32, u->e1, 16), u->wf[8], d0, u->d1a, nullptr, 1, st);
  conv_fwd(16, plain(u->d1a, 16), u->wf[9], d0, u->d1, nullptr, 1, st);
  last_fwd_kernel<<<grid1(v0), 256, 0, st>>>(u->d1, u->W + u->off[10], u->scale, out, v0);
  return cudaGetLastError();
}

// Backward pass of the mean squared error between the last forward output
// (u->out) and tgt; accumulates into u->G (zeroed here) and u->loss.
cudaError_t
backward(rtkb_unet * u, const float * x, const float * tgt, int margin, cudaStream_t st)
{
  const int  B = u->fdims[0], nx = u->fdims[1], ny = u->fdims[2], nz = u->fdims[3];
  const Dims d0 = make_dims(nx, ny, nz, B), d1 = make_dims(nx / 2, ny / 2, nz / 2, B),
             d2 = make_dims(nx / 4, ny / 4, nz / 4, B);
  const long long v0 = d0.vox() * B;
  float *         G = u->G;
  const long long * o = u->off;
  cudaError_t     e = cudaMemsetAsync(G, 0, (size_t)u->nparams * 4, st);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(u->loss, 0, sizeof(double), st);
  if (e != cudaSuccess)
    return e;
  const double cnt = (double)(nx - 2 * margin) * (ny - 2 * margin) * (nz - 2 * margin) * B;
  last_bwd_kernel<<<grid1(v0), 256, 0, st>>>(u->d1, u->W + o[10], u->out, tgt, d0, margin, cnt, u->G0a, G + o[10],
                                             u->loss);
  // L10
  conv_wgrad(16, plain(u->d1a, 16), u->G0a, d0, G + o[9], st);
  conv_fwd(16, plain(u->G0a, 16), u->wd[9], d0, u->G0b, u->d1a, 0, st);
  // L9 (input [up(d2), e1])
  conv_wgrad(16, upcat(u->d2, 32, u->e1, 16), u->G0b, d0, G + o[8], st);
  conv_fwd(48, plain(u->G0b, 16), u->wd[8], d0, u->Gc0, nullptr, 0, st);
  up_grad_kernel<<<grid1(v0 / 8 * 4), 256, 0, st>>>(u->Gc0, 48, 32, u->d2, d0, u->G1a);
  // L8
  conv_wgrad(32, plain(u->d2a, 32), u->G1a, d1, G + o[7], st);
  conv_fwd(32, plain(u->G1a, 32), u->wd[7], d1, u->G1b, u->d2a, 0, st);
  // L7 (input [up(b2), e2])
  conv_wgrad(32, upcat(u->b2, 64, u->e2, 32), u->G1b, d1, G + o[6], st);
  conv_fwd(96, plain(u->G1b, 32), u->wd[6], d1, u->Gc1, nullptr, 0, st);
  up_grad_kernel<<<grid1(v0 / 64 * 8), 256, 0, st>>>(u->Gc1, 96, 64, u->b2, d1, u->G2a);
  // L6, L5
  conv_wgrad(64, plain(u->b1, 64), u->G2a, d2, G + o[5], st);
  conv_fwd(64, plain(u->G2a, 64), u->wd[5], d2, u->G2b, u->b1, 0, st);
  conv_wgrad(64, plain(u->p2, 32), u->G2b, d2, G + o[4], st);
  conv_fwd(32, plain(u->G2b, 64), u->wd[4], d2, u->Gp2, nullptr, 0, st);
  // e2: concatenation (L7) + pooling paths
  skip_grad_kernel<<<grid1(v0 / 8 * 4), 256, 0, st>>>(u->Gc1, 96, 64, u->Gp2, u->e2, 32, d1, u->G1a);
  // L4, L3
  conv_wgrad(32, plain(u->e2a, 32), u->G1a, d1, G + o[3], st);
  conv_fwd(32, plain(u->G1a, 32), u->wd[3], d1, u->G1b, u->e2a, 0, st);
  conv_wgrad(32, plain(u->p1, 16), u->G1b, d1, G + o[2], st);
  conv_fwd(16, plain(u->G1b, 32), u->wd[2], d1, u->Gp1, nullptr, 0, st);
  // e1: concatenation (L9) + pooling paths
  skip_grad_kernel<<<grid1(v0 * 2), 256, 0, st>>>(u->Gc0, 48, 32, u->Gp1, u->e1, 16, d0, u->G0a);
  // L2, L1
  conv_wgrad(16, plain(u->e1a, 16), u->G0a, d0, G + o[1], st);
  conv_fwd(16, plain(u->G0a, 16), u->wd[1], d0, u->G0b, u->e1a, 0, st);
  first_wgrad_kernel<<<(unsigned)std::min<long long>((long long)d0.tx * d0.ty * d0.tz * B, 148LL * 4), 256, 0, st>>>(
    x, u->scale, u->G0b, d0, G + o[0]);
  return cudaGetLastError();
}

} // namespace

// ---- C ABI --------------------------------------------------------------------------------------------------
extern "C" int
rtkb_unet_create(unsigned long long seed, rtkb_unet ** out)
{
  RTKB_TRACE();
  using namespace rtkb;
  if (!out)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null network pointer");
  *out = nullptr;
  rtkb_unet * u = nullptr;
  try
  {
    u = new rtkb_unet();
    long long n = 0;
    for (int l = 0; l < 11; l++)
    {
      u->off[l] = n;
      n += layer_params(l);
    }
    u->nparams = n;
    size_t packed = 0;
    for (int l = 1; l < 10; l++)
      packed += 2 * (size_t)layer_params(l) * 2;
    const size_t fp = ((size_t)n * 4 + 255) & ~size_t(255);
    const size_t total = 4 * fp + packed + 512 + (kScaleBlocks + 2) * sizeof(double);
    cudaError_t  e = cudaMalloc(&u->pmem, total);
    if (e != cudaSuccess)
    {
      delete u;
      return cuda_fail(e, "cudaMalloc (U-Net parameters)");
    }
    char * m = static_cast<char *>(u->pmem);
    u->W = reinterpret_cast<float *>(m);
    u->G = reinterpret_cast<float *>(m + fp);
    u->M = reinterpret_cast<float *>(m + 2 * fp);
    u->V = reinterpret_cast<float *>(m + 3 * fp);
    m += 4 * fp;
    for (int l = 1; l < 10; l++)
    {
      u->wf[l] = reinterpret_cast<bf16 *>(m);
      m += layer_params(l) * 2;
      u->wd[l] = reinterpret_cast<bf16 *>(m);
      m += layer_params(l) * 2;
    }
    m = reinterpret_cast<char *>((reinterpret_cast<uintptr_t>(m) + 255) & ~uintptr_t(255));
    u->scale = reinterpret_cast<float *>(m);
    u->part = reinterpret_cast<double *>(m + 16);
    u->loss = u->part + kScaleBlocks;
    // He-normal initialisation (fan-in 27 c_in; 16 for the 1x1x1 output layer)
    std::vector<float> h((size_t)n);
    std::mt19937_64    rng(seed);
    for (int l = 0; l < 11; l++)
    {
      const double fan = l == 10 ? 16. : 27. * kLayers[l].cin;
      std::normal_distribution<double> nd(0., std::sqrt(2. / fan));
      for (long long i = 0; i < layer_params(l); i++)
        h[(size_t)(u->off[l] + i)] = (float)(l == 10 ? nd(rng) * 0.5 : nd(rng));
    }
    e = cudaMemcpy(u->W, h.data(), (size_t)n * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemset(u->M, 0, 2 * fp);
    if (e == cudaSuccess)
      e = repack(u, nullptr);
    if (e == cudaSuccess)
      e = cudaDeviceSynchronize();
    if (e != cudaSuccess)
    {
      rtkb_unet_destroy(u);
      return cuda_fail(e, "U-Net initialisation");
    }
    *out = u;
    return RTKB_OK;
  }
  catch (...)
  {
    if (u)
      rtkb_unet_destroy(u);
    return fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

extern "C" long long
rtkb_unet_num_parameters(const rtkb_unet * u)
{
  return u ? u->nparams : 0;
}

extern "C" int
rtkb_unet_get_parameters(const rtkb_unet * u, float * host, long long n)
{
  RTKB_TRACE();
  using namespace rtkb;
  if (!u || !host || n != u->nparams)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "parameter count mismatch");
  RTKB_CUDA_TRY(cudaDeviceSynchronize());
  RTKB_CUDA_TRY(cudaMemcpy(host, u->W, (size_t)n * 4, cudaMemcpyDeviceToHost));
  return RTKB_OK;
}

extern "C" int
rtkb_unet_set_parameters(rtkb_unet * u, const float * host, long long n)
{
  using namespace rtkb;
  if (!u || !host || n != u->nparams)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "parameter count mismatch");
  RTKB_CUDA_TRY(cudaDeviceSynchronize());
  RTKB_CUDA_TRY(cudaMemcpy(u->W, host, (size_t)n * 4, cudaMemcpyHostToDevice));
  RTKB_CUDA_TRY(cudaMemset(u->M, 0, (size_t)n * 4));
  RTKB_CUDA_TRY(cudaMemset(u->V, 0, (size_t)n * 4));
  u->step = 0;
  RTKB_CUDA_TRY(repack(u, nullptr));
  RTKB_CUDA_TRY(cudaDeviceSynchronize());
  return RTKB_OK;
}

extern "C" int
rtkb_unet_get_gradients(const rtkb_unet * u, float * host, long long n)
{
  RTKB_TRACE();
  using namespace rtkb;
  if (!u || !host || n != u->nparams)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "parameter count mismatch");
  RTKB_CUDA_TRY(cudaDeviceSynchronize());
  RTKB_CUDA_TRY(cudaMemcpy(host, u->G, (size_t)n * 4, cudaMemcpyDeviceToHost));
  return RTKB_OK;
}

extern "C" int
rtkb_unet_reserve(rtkb_unet * u, int batch, int nx, int ny, int nz)
{
  RTKB_TRACE();
  using namespace rtkb;
  if (!u)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null network");
  const int rc = check_dims(batch, nx, ny, nz);
  return rc != RTKB_OK ? rc : reserve_forward(u, batch, nx, ny, nz);
}

extern "C" int
rtkb_unet_set_wgrad_kernel(int kernel)
{
  if (kernel < 0 || kernel > 2)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "weight-gradient kernel: 0, 1 or 2");
  g_wgrad_kernel = kernel;
  return RTKB_OK;
}

extern "C" int
rtkb_unet_set_conv_pipeline(int enable)
{
  if (enable < 0 || enable > 2)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "convolution kernel: 0, 1 or 2");
  g_conv_pipeline = enable;
  return RTKB_OK;
}

extern "C" int
rtkb_unet_forward(rtkb_unet * u, int batch, int nx, int ny, int nz, const float * d_in, float * d_out, int normalize,
                  void * stream)
{
  RTKB_TRACE();
  using namespace rtkb;
  if (!u || !d_in || !d_out)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  int rc = check_dims(batch, nx, ny, nz);
  if (rc == RTKB_OK)
    rc = reserve_forward(u, batch, nx, ny, nz);
  if (rc != RTKB_OK)
    return rc;
  const cudaError_t e = forward(u, d_in, d_out, normalize, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? RTKB_OK : cuda_fail(e, "U-Net forward");
}

extern "C" int
rtkb_unet_train_step(rtkb_unet * u, int batch, int nx, int ny, int nz, const float * d_in, const float * d_target,
                     int loss_margin, double learning_rate, int update, double * loss, void * stream)
{
  RTKB_TRACE();
  using namespace rtkb;
  if (!u || !d_in || !d_target)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  if (loss_margin < 0 || 2 * loss_margin >= std::min(nx, std::min(ny, nz)))
    return fail(RTKB_ERR_INVALID_ARGUMENT, "loss margin leaves no voxel");
  int rc = check_dims(batch, nx, ny, nz);
  if (rc == RTKB_OK)
    rc = reserve_forward(u, batch, nx, ny, nz);
  if (rc == RTKB_OK)
    rc = reserve_backward(u);
  if (rc != RTKB_OK)
    return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t  e = forward(u, d_in, u->out, 0, st);
  if (e == cudaSuccess)
    e = backward(u, d_in, d_target, loss_margin, st);
  if (e == cudaSuccess && update)
  {
    u->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f / (1.f - (float)std::pow(b1, u->step)), c2 = 1.f / (1.f - (float)std::pow(b2, u->step));
    adam_kernel<<<grid1(u->nparams), 256, 0, st>>>(u->W, u->G, u->M, u->V, (int)u->nparams, (float)learning_rate, b1,
                                                   b2, c1, c2, 1e-8f);
    e = cudaGetLastError();
    if (e == cudaSuccess)
      e = repack(u, st);
  }
  if (e != cudaSuccess)
    return cuda_fail(e, "U-Net training step");
  if (loss)
  {
    double l = 0.;
    RTKB_CUDA_TRY(cudaMemcpyAsync(&l, u->loss, sizeof(double), cudaMemcpyDeviceToHost, st));
    RTKB_CUDA_TRY(cudaStreamSynchronize(st));
    *loss = l / ((double)(nx - 2 * loss_margin) * (ny - 2 * loss_margin) * (nz - 2 * loss_margin) * batch);
  }
  return RTKB_OK;
}

extern "C" void
rtkb_unet_destroy(rtkb_unet * u)
{
  if (!u)
    return;
  if (u->gmem)
    cudaFree(u->gmem);
  if (u->fmem)
    cudaFree(u->fmem);
  if (u->pmem)
    cudaFree(u->pmem);
  delete u;
}

// Internal: forward into caller buffers over an already reserved workspace
// (used by the preconditioned CG plan inside its CUDA graph).
namespace rtkb
{
cudaError_t
unet_apply(rtkb_unet * u, const float * in, float * out, cudaStream_t st)
{
  return forward(u, in, out, 1, st);
}
bool
unet_reserved_for(const rtkb_unet * u, int nx, int ny, int nz)
{
  return u && u->fmem && u->fdims[0] == 1 && u->fdims[1] == nx && u->fdims[2] == ny && u->fdims[3] == nz;
}
} // namespace rtkb

// filters.cu -- projection-domain filters of the FDK pipeline on sm_100a.
//
// One pass over the projection stack applies, in RTK's order, the displaced-
// detector weighting and padding (include/rtkDisplacedDetectorImageFilter.hxx),
// the Parker short-scan weights (include/rtkParkerShortScanImageFilter.hxx),
// the FDK cos(gamma) weighting (include/rtkFDKWeightProjectionFilter.hxx) and the
// ramp filter (include/rtkFFTProjectionsConvolutionImageFilter.hxx:121-276 with
// the kernel of include/rtkFFTRampImageFilter.hxx:47-178).
//
// The ramp filter is a hand-written shared-memory FFT, compiled per padded
// length N: two real rows are filtered at once as the real and imaginary
// parts of one complex sequence (the ramp kernel is real and even, so the rows
// do not mix), zero-padded to the power-of-two length RTK uses without FFTW.
// Stockham radix-16 passes (Govindaraju et al., SC08) with a final radix-8/4/2
// pass, twiddle powers from per-pass tables built in FP64 on the host, padded
// shared-memory indices; the inverse transform is a forward transform of the
// conjugate.  CTAs are persistent: the twiddles and the ramp kernel are loaded
// into shared memory once, and the next row pair is prefetched into registers
// while the current one is transformed.  FDK cos(gamma) weights come from
// FP64 per-row terms evaluated per pixel in FP32, Parker and displaced-detector
// weights from FP64 host tables; the stack is read once and written once.
#include "rtkb_filters.h"

#include <algorithm>
#include <cstring>

namespace
{

constexpr int kMaxFFT = 8192;

struct FilterArgs
{
  const float *  in;
  float *        out;
  const double * fdkp;  // kFdkWeightParams per projection, or null
  const float *  colw;  // per (projection, output column) weight, or null
  const float *  K;     // ramp kernel, N/2+1
  const float2 * tw;    // twiddles e^{-2 pi i m/N}
  const float *  mw;    // truncation mirror weights, next+1
  int            nu_in, nu_out, nv, np, shift, N, next;
};

// Per-row part of the weights: FDK cos(gamma) terms for row r of projection s
// (include/rtkFDKWeightProjectionFilter.hxx:67-128; parameters from the FP64
// host table), evaluated per pixel in FP32 (relative error ~1e-7).
struct RowWeight
{
  float f, num1, sina, sddtana, e, xc0, dxc;
  int   mode; // 0: none, 1: constant (parallel), 2: cos(gamma)
};

__device__ __forceinline__ RowWeight
row_weight(const FilterArgs & a, int s, int r)
{
  RowWeight w{ 1.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0 };
  if (!a.fdkp)
    return w;
  const double * q = a.fdkp + (long long)s * rtkb::kFdkWeightParams;
  w.f = (float)q[0];
  if (q[7] != 0.)
  {
    w.mode = 1;
    return w;
  }
  const double y = q[6] + r * q[9];
  w.mode = 2;
  w.num1 = (float)q[1];
  w.sina = (float)q[2];
  w.sddtana = (float)q[3];
  w.e = (float)(q[4] + y * y);
  w.xc0 = (float)q[5];
  w.dxc = (float)q[8];
  return w;
}

__device__ __forceinline__ float
raw_pixel(const FilterArgs & a, int s, int r, int c)
{
  const int ci = c - a.shift;
  return (ci >= 0 && ci < a.nu_in) ? __ldg(a.in + ((long long)s * a.nv + r) * a.nu_in + ci) : 0.f;
}

__device__ __forceinline__ float
apply_weights(const FilterArgs & a, const RowWeight & w, int s, int c, float v)
{
  if (a.colw)
    v *= __ldg(a.colw + (long long)s * a.nu_out + c);
  if (w.mode == 1)
    v *= w.f;
  else if (w.mode == 2)
  {
    const float x = fmaf((float)c, w.dxc, w.xc0), dxs = x - w.sddtana;
    v *= w.f * (w.num1 - x * w.sina) * rsqrtf(fmaf(dxs, dxs, w.e));
  }
  return v;
}

__device__ __forceinline__ float
weighted_pixel(const FilterArgs & a, const RowWeight & w, int s, int r, int c)
{
  return apply_weights(a, w, s, c, raw_pixel(a, s, r, c));
}

// grid: (column blocks, rows, projections)
__global__ void __launch_bounds__(256)
weight_kernel(FilterArgs a)
{
  const int       r = blockIdx.y, s = blockIdx.z;
  const RowWeight w = row_weight(a, s, r);
  float *         o = a.out + ((long long)s * a.nv + r) * a.nu_out;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < a.nu_out; c += gridDim.x * blockDim.x)
    o[c] = weighted_pixel(a, w, s, r, c);
}

// Shared-memory index with one pad element after every 16: the stride-16
// writes of the first radix-16 Stockham pass then spread over all banks.
__host__ __device__ __forceinline__ constexpr int
pidx(int x)
{
  return x + (x >> 4);
}

__device__ __forceinline__ float2
cmul(float2 a, float2 b)
{
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// d * e^{-2 pi i j / L} for the constant twiddles of a size-L (2, 4, 8) DFT
__device__ __forceinline__ float2
rot_const(float2 d, int j, int L)
{
  constexpr float c = 0.70710678118654752440f; // sqrt(1/2)
  if (L == 2 || j == 0)
    return d;
  if (L == 4 || j == 2)
    return make_float2(d.y, -d.x);
  if (j == 1)
    return make_float2(c * (d.x + d.y), c * (d.y - d.x));
  return make_float2(c * (d.y - d.x), -c * (d.x + d.y));
}

// In-register forward DFT of size R (decimation in frequency), natural order out.
template <int R>
__device__ __forceinline__ void
dft_reg(float2 (&v)[R])
{
#pragma unroll
  for (int half = R / 2; half >= 1; half >>= 1)
  {
#pragma unroll
    for (int i = 0; i < R; i += 2 * half)
    {
#pragma unroll
      for (int j = 0; j < half; j++)
      {
        const float2 x = v[i + j], y = v[i + j + half];
        v[i + j] = make_float2(x.x + y.x, x.y + y.y);
        v[i + j + half] = rot_const(make_float2(x.x - y.x, x.y - y.y), j, 2 * half);
      }
    }
  }
  if (R == 4)
  {
    const float2 t = v[1];
    v[1] = v[2];
    v[2] = t;
  }
  else if (R == 8)
  {
    float2 t = v[1];
    v[1] = v[4];
    v[4] = t;
    t = v[3];
    v[3] = v[6];
    v[6] = t;
  }
}

// In-register forward DFT of size 16 (radix-2 decimation in frequency with the
// W16^j = e^{-2 pi i j/16} constants, then the 4-bit reversal).
__device__ __forceinline__ void
dft16(float2 (&v)[16])
{
  constexpr float c[8] = { 1.f, 0.92387953251128675613f, 0.70710678118654752440f, 0.38268343236508977173f,
                           0.f, -0.38268343236508977173f, -0.70710678118654752440f, -0.92387953251128675613f };
  constexpr float sn[8] = { 0.f, 0.38268343236508977173f, 0.70710678118654752440f, 0.92387953251128675613f,
                            1.f, 0.92387953251128675613f, 0.70710678118654752440f, 0.38268343236508977173f };
#pragma unroll
  for (int j = 0; j < 8; j++)
  {
    const float2 x = v[j], y = v[j + 8];
    const float2 d = make_float2(x.x - y.x, x.y - y.y);
    v[j] = make_float2(x.x + y.x, x.y + y.y);
    v[j + 8] = make_float2(d.x * c[j] + d.y * sn[j], d.y * c[j] - d.x * sn[j]); // d * W16^j
  }
#pragma unroll
  for (int half = 4; half >= 1; half >>= 1)
  {
#pragma unroll
    for (int i = 0; i < 16; i += 2 * half)
    {
#pragma unroll
      for (int j = 0; j < half; j++)
      {
        const float2 x = v[i + j], y = v[i + j + half];
        v[i + j] = make_float2(x.x + y.x, x.y + y.y);
        v[i + j + half] = rot_const(make_float2(x.x - y.x, x.y - y.y), j, 2 * half);
      }
    }
  }
  float2 t[16];
#pragma unroll
  for (int k = 0; k < 16; k++)
    t[k] = v[((k & 1) << 3) | ((k & 2) << 1) | ((k & 4) >> 1) | ((k & 8) >> 3)];
#pragma unroll
  for (int k = 0; k < 16; k++)
    v[k] = t[k];
}

template <int R>
__device__ __forceinline__ void
dft_any(float2 (&v)[R])
{
  if constexpr (R == 16)
    dft16(v);
  else
    dft_reg<R>(v);
}

// Twiddle rows of one pass: powers 1, 2, 4, 8 (those below R) of
// w = e^{-2 pi i k / (Ns R)}, each row Ns entries long (k = 0..Ns-1).
template <int R>
__host__ __device__ constexpr int
twiddle_rows()
{
  return R == 16 ? 4 : R == 8 ? 3 : R == 4 ? 2 : 1;
}

// Compile-time version of the pass chain for a fixed N: every stride, radix
// and loop trip is a constant, so index arithmetic folds into immediates.
template <int N, int T, int Ns, int R>
__device__ __forceinline__ void
fft_pass_c(const float2 * __restrict__ src, float2 * __restrict__ dst, const float2 * __restrict__ twp)
{
  constexpr int nb = N / R;
#pragma unroll
  for (int jj = 0; jj < (nb + T - 1) / T; jj++)
  {
    const int j = threadIdx.x + jj * T;
    if (nb % T != 0 && j >= nb)
      break;
    const int k = j & (Ns - 1);
    float2    v[R];
#pragma unroll
    for (int r = 0; r < R; r++)
      v[r] = src[pidx(j + r * nb)];
    if constexpr (Ns > 1)
    {
      float2 t[R];
      t[1] = twp[k];
      if constexpr (R > 2)
      {
        t[2] = twp[Ns + k];
        t[3] = cmul(t[2], t[1]);
      }
      if constexpr (R > 4)
      {
        t[4] = twp[2 * Ns + k];
        t[5] = cmul(t[4], t[1]);
        t[6] = cmul(t[4], t[2]);
        t[7] = cmul(t[4], t[3]);
      }
      if constexpr (R > 8)
      {
        t[8] = twp[3 * Ns + k];
#pragma unroll
        for (int q = 1; q < 8; q++)
          t[8 + q] = cmul(t[8], t[q]);
      }
#pragma unroll
      for (int r = 1; r < R; r++)
        v[r] = cmul(v[r], t[r]);
    }
    dft_any<R>(v);
    const int d = (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; r++)
      dst[pidx(d + r * Ns)] = v[r];
  }
}

template <int N, int T, int Ns>
__device__ __forceinline__ float2 *
fft_chain(float2 * src, float2 * dst, const float2 * tw)
{
  if constexpr (Ns >= N)
    return src;
  else
  {
    constexpr int R = (N / Ns >= 16) ? 16 : N / Ns;
    fft_pass_c<N, T, Ns, R>(src, dst, tw);
    __syncthreads();
    return fft_chain<N, T, Ns * R>(dst, src, tw + (Ns > 1 ? twiddle_rows<R>() * Ns : 0));
  }
}

// Threads of the ramp kernels: 16 columns per thread cover a row of N.
template <int N>
constexpr int kRampThreads = N / 16 > 64 ? N / 16 : 64;

// Ramp filter of the row pairs first, first + stride, ... < pairs of one stack
// (two real rows as one complex sequence); the pass twiddles and the stack's
// ramp kernel are in shared memory already.  The next pair's raw pixels are
// prefetched into registers while the current pair is transformed.
template <int N>
__device__ __forceinline__ void
ramp_pairs(const FilterArgs & a, long long first, long long pairs, long long stride, float2 * b0, float2 * b1,
           const float2 * tws, const float * Ks)
{
  constexpr int   T = kRampThreads<N>;
  const int       nu = a.nu_out;
  const long long rows = (long long)a.nv * a.np;
  const float     inv = 1.f / (float)N;
  // columns threadIdx.x + i * blockDim.x; blockDim.x >= N / 16, so 16 columns
  // per thread cover the row
  float pa[16], pb[16];
  auto  prefetch = [&](long long pr) {
    const long long ra = 2 * pr, rb = ra + 1;
    const int       sa = (int)(ra / a.nv), rra = (int)(ra % a.nv);
    const bool      hb = rb < rows;
    const int       sb = hb ? (int)(rb / a.nv) : sa, rrb = hb ? (int)(rb % a.nv) : rra;
#pragma unroll
    for (int i = 0; i < 16; i++)
    {
      const int c = threadIdx.x + i * T;
      pa[i] = (c < nu) ? raw_pixel(a, sa, rra, c) : 0.f;
      pb[i] = (c < nu && hb) ? raw_pixel(a, sb, rrb, c) : 0.f;
    }
  };
  if (first < pairs)
    prefetch(first);
  for (long long pr = first; pr < pairs; pr += stride)
  {
    const long long ra = 2 * pr, rb = ra + 1;
    const bool      hb = rb < rows;
    const int       sa = (int)(ra / a.nv), rra = (int)(ra % a.nv);
    const int       sb = hb ? (int)(rb / a.nv) : sa, rrb = hb ? (int)(rb % a.nv) : rra;
    const RowWeight wa = row_weight(a, sa, rra);
    const RowWeight wb = row_weight(a, sb, rrb);
    __syncthreads(); // the previous pair's results have been stored
#pragma unroll
    for (int i = 0; i < 16; i++)
    {
      const int c = threadIdx.x + i * T;
      if (c < N)
      {
        const float x = (c < nu) ? apply_weights(a, wa, sa, c, pa[i]) : 0.f;
        const float y = (c < nu && hb) ? apply_weights(a, wb, sb, c, pb[i]) : 0.f;
        b0[pidx(c)] = make_float2(x, y);
      }
    }
    if (pr + stride < pairs)
      prefetch(pr + stride);
    __syncthreads();
    if (a.next > 0)
    {
      // Ohnesorge mirror extrapolation (PadInputImageRegion :218-258): left
      // values wrap to the end of the circular buffer.
      const float2 SA = b0[pidx(1)], SE = b0[pidx(nu - 1)];
      for (int bq = 1 + threadIdx.x; bq <= a.next; bq += blockDim.x)
      {
        const float  w = __ldg(a.mw + bq);
        const float2 l = b0[pidx(bq)], r = b0[pidx(nu - 1 - bq)];
        b0[pidx(N - bq)] = make_float2(w * (2.f * SA.x - l.x), w * (2.f * SA.y - l.y));
        b0[pidx(nu - 1 + bq)] = make_float2(w * (2.f * SE.x - r.x), w * (2.f * SE.y - r.y));
      }
      __syncthreads();
    }
    float2 * X = fft_chain<N, T, 1>(b0, b1, tws);
    float2 * other = (X == b0) ? b1 : b0;
    // multiply by the real, even kernel and conjugate: the inverse transform is
    // conj(FFT(conj(K X))) / N
    for (int f = threadIdx.x; f < N; f += blockDim.x)
    {
      const float  k = Ks[min(f, N - f)];
      const float2 z = X[pidx(f)];
      X[pidx(f)] = make_float2(z.x * k, -z.y * k);
    }
    __syncthreads();
    float2 * W = fft_chain<N, T, 1>(X, other, tws);
    for (int c = threadIdx.x; c < nu; c += blockDim.x)
    {
      const float2 z = W[pidx(c)];
      a.out[ra * nu + c] = z.x * inv;
      if (hb)
        a.out[rb * nu + c] = -z.y * inv;
    }
  }
}

// Ramp filter of one stack, persistent: each CTA loads the pass twiddles and
// the ramp kernel into shared memory once, then filters row pairs until the
// stack is done.  The stack's description is a kernel parameter.
// 128 registers per thread at most: (threads x 128) x (512 / threads) = 64 K
template <int N>
__global__ void __launch_bounds__(kRampThreads<N>, 512 / kRampThreads<N>)
ramp_fft_kernel(FilterArgs a, int tw_len)
{
  constexpr int P = pidx(N);
  extern __shared__ float2 sbuf[];
  float2 *      tws = sbuf + 2 * P;
  float *       Ks = reinterpret_cast<float *>(tws + tw_len);
  for (int i = threadIdx.x; i < tw_len; i += blockDim.x)
    tws[i] = a.tw[i];
  for (int i = threadIdx.x; i <= N / 2; i += blockDim.x)
    Ks[i] = a.K[i];
  const long long pairs = ((long long)a.nv * a.np + 1) / 2;
  ramp_pairs<N>(a, blockIdx.x, pairs, gridDim.x, sbuf, sbuf + P, tws, Ks);
}

// Ramp filter of many stacks of one padded length N, persistent: the global
// row-pair range of stack q is [pair_begin[q], pair_begin[q + 1]); a CTA takes
// the pairs blockIdx.x + k gridDim.x, stack after stack, loading each stack's
// description (into shared memory) and ramp kernel when it reaches it.  The
// pass twiddles are shared by every stack of the launch.
template <int N>
__global__ void __launch_bounds__(kRampThreads<N>, 512 / kRampThreads<N>)
ramp_fft_batch_kernel(const FilterArgs * __restrict__ probs, const long long * __restrict__ pair_begin, int nprob,
                      const float2 * __restrict__ tw, int tw_len)
{
  constexpr int P = pidx(N);
  extern __shared__ float2 sbuf[];
  __shared__ FilterArgs cur;
  float2 *              tws = sbuf + 2 * P;
  float *               Ks = reinterpret_cast<float *>(tws + tw_len);
  for (int i = threadIdx.x; i < tw_len; i += blockDim.x)
    tws[i] = tw[i];
  for (int q = 0; q < nprob; q++)
  {
    const long long lo = pair_begin[q], hi = pair_begin[q + 1];
    // this CTA's first pair at or after lo, as an index of stack q
    const long long first = (((long long)blockIdx.x - lo) % gridDim.x + gridDim.x) % gridDim.x;
    if (lo + first >= hi)
      continue;
    __syncthreads(); // the previous stack's last pair has been stored
    if (threadIdx.x == 0)
      cur = probs[q];
    for (int i = threadIdx.x; i <= N / 2; i += blockDim.x)
      Ks[i] = probs[q].K[i];
    __syncthreads();
    ramp_pairs<N>(cur, first, hi - lo, gridDim.x, sbuf, sbuf + P, tws, Ks);
  }
}

// Twiddle rows of every pass of a length-N transform, in pass order, FP64
// values stored as float2 (see fft_pass).
static void
pass_twiddles(int N, std::vector<float> & tw)
{
  tw.clear();
  for (int Ns = 1; Ns < N;)
  {
    const int rem = N / Ns;
    const int R = rem >= 16 ? 16 : rem;
    const int nrows = R == 16 ? 4 : R == 8 ? 3 : R == 4 ? 2 : 1;
    if (Ns > 1)
      for (int row = 0; row < nrows; row++)
      {
        const int pw = 1 << row;
        for (int k = 0; k < Ns; k++)
        {
          const double ang = -2. * 3.14159265358979323846 * (double)pw * (double)k / ((double)Ns * R);
          tw.push_back((float)std::cos(ang));
          tw.push_back((float)std::sin(ang));
        }
      }
    Ns *= R;
  }
}

// Grid of a persistent ramp launch: as many CTAs as fit on the GPU, at most
// one per row pair.
template <typename K>
static cudaError_t
ramp_grid(K kern, int threads, size_t smem, long long pairs, long long & grid)
{
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int         dev = 0, sms = 0, per_sm = 0;
  if (e == cudaSuccess)
    e = cudaGetDevice(&dev);
  if (e == cudaSuccess)
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
  grid = std::min<long long>(pairs, (long long)sms * std::max(per_sm, 1));
  return e;
}

template <int N>
static size_t
ramp_smem(int tw_len)
{
  return (2 * (size_t)pidx(N) + tw_len) * sizeof(float2) + ((size_t)N / 2 + 1) * sizeof(float);
}

template <int N>
static cudaError_t
launch_ramp(const FilterArgs & a, int tw_len, long long pairs, cudaStream_t st)
{
  long long   grid = 0;
  cudaError_t e = ramp_grid(ramp_fft_kernel<N>, kRampThreads<N>, ramp_smem<N>(tw_len), pairs, grid);
  if (e == cudaSuccess && pairs > 0)
  {
    ramp_fft_kernel<N><<<(unsigned)grid, kRampThreads<N>, ramp_smem<N>(tw_len), st>>>(a, tw_len);
    e = cudaGetLastError();
  }
  return e;
}

template <int N>
static cudaError_t
launch_ramp_batch(const FilterArgs * d_probs, const long long * d_begin, int nprob, long long pairs,
                  const float2 * d_tw, int tw_len, cudaStream_t st)
{
  long long   grid = 0;
  cudaError_t e = ramp_grid(ramp_fft_batch_kernel<N>, kRampThreads<N>, ramp_smem<N>(tw_len), pairs, grid);
  if (e == cudaSuccess && pairs > 0)
  {
    ramp_fft_batch_kernel<N><<<(unsigned)grid, kRampThreads<N>, ramp_smem<N>(tw_len), st>>>(d_probs, d_begin, nprob,
                                                                                           d_tw, tw_len);
    e = cudaGetLastError();
  }
  return e;
}

// One stack (d_probs == nullptr: a) or a table of nprob stacks of length N.
static cudaError_t
launch_ramp_n(int N, const FilterArgs & a, const FilterArgs * d_probs, const long long * d_begin, int nprob,
              long long pairs, const float2 * d_tw, int tw_len, cudaStream_t st)
{
#define RTKB_RAMP_CASE(n)                                                                                              \
  case n:                                                                                                              \
    return d_probs ? launch_ramp_batch<n>(d_probs, d_begin, nprob, pairs, d_tw, tw_len, st)                            \
                   : launch_ramp<n>(a, tw_len, pairs, st)
  switch (N)
  {
    RTKB_RAMP_CASE(2);
    RTKB_RAMP_CASE(4);
    RTKB_RAMP_CASE(8);
    RTKB_RAMP_CASE(16);
    RTKB_RAMP_CASE(32);
    RTKB_RAMP_CASE(64);
    RTKB_RAMP_CASE(128);
    RTKB_RAMP_CASE(256);
    RTKB_RAMP_CASE(512);
    RTKB_RAMP_CASE(1024);
    RTKB_RAMP_CASE(2048);
    RTKB_RAMP_CASE(4096);
    default:
      return d_probs ? launch_ramp_batch<8192>(d_probs, d_begin, nprob, pairs, d_tw, tw_len, st)
                     : launch_ramp<8192>(a, tw_len, pairs, st);
  }
#undef RTKB_RAMP_CASE
}

struct Options
{
  bool             displaced = false, pad = true, parker = false, fdk = false, ramp = false;
  double           threshold = 3.14159265358979323846 / 9;
  rtkb_ramp_params rp{};
};

template <typename T>
static size_t
append(std::vector<unsigned char> & blob, const std::vector<T> & v)
{
  size_t off = (blob.size() + 255) & ~size_t(255);
  blob.resize(off + v.size() * sizeof(T));
  if (!v.empty())
    std::memcpy(blob.data() + off, v.data(), v.size() * sizeof(T));
  return off;
}

// Host half of the weighting and ramp filters of one stack: argument checks,
// the output region, the FP64 weight tables, the ramp kernel, the twiddles and
// the truncation weights, gathered into P.blob for one upload; P.a holds the
// sizes and, after bind_filters, the device pointers.
struct Prepared
{
  FilterArgs                 a{};
  std::vector<unsigned char> blob;
  size_t                     o_fdk = 0, o_colw = 0, o_K = 0, o_tw = 0, o_mw = 0;
  bool                       h_fdk = false, h_colw = false, h_K = false, h_tw = false, h_mw = false;
  int                        tw_len = 0;
  long long                  pairs = 0;
  bool                       ramp = false;
};

int
prepare_filters(const rtkb_geometry * g, const rtkb_image_desc * in, const Options & o, rtkb_image_desc * out_desc,
                const float * d_in, float * d_out, int * is_short, Prepared & P)
{
  using namespace rtkb;
  std::string why;
  if (!g)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "Geometry has not been set.");
  if (!desc_valid(in, why))
    return fail(RTKB_ERR_INVALID_ARGUMENT, why);
  const Geometry & G = g->g;
  if (in->index[2] < 0 || (long long)in->index[2] + in->size[2] > (long long)G.p.size())
    return fail(RTKB_ERR_INVALID_ARGUMENT, "Mismatch between the number of projections and the geometry entries.");
  if (o.displaced && (G.radius_cylindrical != 0. || (!G.p.empty() && G.p[0].sdd == 0.)))
    return fail(RTKB_ERR_UNSUPPORTED, "Displaced detector cannot handle cylindrical detector or parallel geometry");

  rtkb_image_desc    out = *in;
  int                shift = 0;
  std::vector<float> wd, wp, colw;
  if (o.displaced)
  {
    DisplacedInfo info;
    int           rc = displaced_region(G, *in, o.pad, info);
    if (rc != RTKB_OK)
      return rc;
    if (info.weighted)
    {
      out = info.out;
      shift = info.shift;
      displaced_weights(G, *in, info, wd);
    }
  }
  bool short_scan = false;
  if (o.parker)
    short_scan = parker_weights(G, out, o.threshold, wp);
  if (is_short)
    *is_short = short_scan ? 1 : 0;
  if (out_desc)
    *out_desc = out;
  const int nu_in = in->size[0], nu_out = out.size[0], nv = in->size[1], np = in->size[2];
  if (!d_in || !d_out)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null buffer");
  if (d_in == d_out && nu_out != nu_in)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "the padded displaced-detector output cannot be computed in place");
  if (nv > 65535 || np > 65535)
    return fail(RTKB_ERR_UNSUPPORTED, "projection stacks of more than 65535 rows or projections per call");
  if (!wd.empty() || short_scan)
  {
    colw.assign((size_t)np * nu_out, 1.f);
    for (int s = 0; s < np; s++)
      for (int c = 0; c < nu_out; c++)
      {
        float       w = 1.f;
        const int   ci = c - shift;
        if (!wd.empty())
          w *= (ci >= 0 && ci < nu_in) ? wd[(size_t)s * nu_in + ci] : 0.f;
        if (short_scan)
          w *= wp[(size_t)s * nu_out + c];
        colw[(size_t)s * nu_out + c] = w;
      }
  }
  std::vector<double> fdkp;
  if (o.fdk)
    fdk_weight_params(G, out, fdkp);

  FilterArgs a{};
  a.nu_in = nu_in;
  a.nu_out = nu_out;
  a.nv = nv;
  a.np = np;
  a.shift = shift;
  std::vector<float> K, tw, mw;
  if (o.ramp)
  {
    if (o.rp.greatest_prime_factor != 2 && o.rp.greatest_prime_factor != 0)
      return fail(RTKB_ERR_UNSUPPORTED, "the GPU ramp filter pads to powers of two (greatest prime factor 2)");
    const int N = ramp_padded_size(nu_out, o.rp);
    if ((N & (N - 1)) != 0 || N > kMaxFFT || N < 2)
      return fail(RTKB_ERR_UNSUPPORTED, "padded row length must be a power of two <= 8192");
    std::vector<double> Kd;
    ramp_kernel(N, out.spacing[0], o.rp, Kd);
    K.assign(Kd.begin(), Kd.end());
    pass_twiddles(N, tw);
    int next = (int)std::floor(o.rp.truncation_correction * nu_out);
    next = std::min(next, (N - nu_out) / 2);
    if (next == 1)
      return fail(RTKB_ERR_INVALID_ARGUMENT, "truncation correction extent of one pixel is undefined");
    if (next > 0)
      truncation_mirror_weights(next, mw);
    a.N = N;
    a.next = next;
  }
  P.blob.clear();
  P.o_fdk = append(P.blob, fdkp);
  P.o_colw = append(P.blob, colw);
  P.o_K = append(P.blob, K);
  P.o_tw = append(P.blob, tw);
  P.o_mw = append(P.blob, mw);
  P.h_fdk = !fdkp.empty();
  P.h_colw = !colw.empty();
  P.h_K = !K.empty();
  P.h_tw = !tw.empty();
  P.h_mw = !mw.empty();
  P.tw_len = (int)(tw.size() / 2);
  P.pairs = ((long long)nv * np + 1) / 2;
  P.ramp = o.ramp;
  a.in = d_in;
  a.out = d_out;
  P.a = a;
  return RTKB_OK;
}

// Points P.a's tables at the device copy of P.blob that starts at base.
void
bind_filters(Prepared & P, char * base)
{
  P.a.fdkp = P.h_fdk ? reinterpret_cast<const double *>(base + P.o_fdk) : nullptr;
  P.a.colw = P.h_colw ? reinterpret_cast<const float *>(base + P.o_colw) : nullptr;
  P.a.K = P.h_K ? reinterpret_cast<const float *>(base + P.o_K) : nullptr;
  P.a.tw = P.h_tw ? reinterpret_cast<const float2 *>(base + P.o_tw) : nullptr;
  P.a.mw = P.h_mw ? reinterpret_cast<const float *>(base + P.o_mw) : nullptr;
}

size_t
align256(size_t x)
{
  return (x + 255) & ~size_t(255);
}

int
run_filters(const rtkb_geometry * g, const rtkb_image_desc * in, const Options & o, rtkb_image_desc * out_desc,
            const float * d_in, float * d_out, cudaStream_t st, int * is_short)
{
  using namespace rtkb;
  Prepared P;
  int      rc = prepare_filters(g, in, o, out_desc, d_in, d_out, is_short, P);
  if (rc != RTKB_OK)
    return rc;
  void * scratch = nullptr;
  if (!P.blob.empty())
    RTKB_CUDA_TRY(rtkb::scratch_malloc(&scratch, P.blob.size(), st));
  bind_filters(P, static_cast<char *>(scratch));
  cudaError_t e = scratch ? cudaMemcpyAsync(scratch, P.blob.data(), P.blob.size(), cudaMemcpyHostToDevice, st)
                          : cudaSuccess;
  if (e != cudaSuccess)
    rc = cuda_fail(e, "cudaMemcpyAsync");
  else if (P.ramp)
  {
    e = launch_ramp_n(P.a.N, P.a, nullptr, nullptr, 1, P.pairs, P.a.tw, P.tw_len, st);
    if (e != cudaSuccess)
      rc = cuda_fail(e, "ramp_fft_kernel launch");
  }
  else
  {
    const dim3 grid((unsigned)((P.a.nu_out + 255) / 256), (unsigned)P.a.nv, (unsigned)P.a.np);
    weight_kernel<<<grid, 256, 0, st>>>(P.a);
    e = cudaGetLastError();
    if (e != cudaSuccess)
      rc = cuda_fail(e, "weight_kernel launch");
  }
  if (scratch)
  {
    cudaError_t fe = rtkb::scratch_free(scratch, st);
    if (rc == RTKB_OK && fe != cudaSuccess)
      rc = cuda_fail(fe, "cudaFreeAsync");
  }
  return rc;
}

template <typename F>
int
guarded(F && f)
{
  try
  {
    return f();
  }
  catch (...)
  {
    return rtkb::fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

} // namespace

extern "C" int
rtkb_fdk_weight(const rtkb_geometry * g, const rtkb_image_desc * proj, const float * d_in, float * d_out,
                void * stream)
{
  RTKB_TRACE();
  return guarded([&] {
    Options o;
    o.fdk = true;
    return run_filters(g, proj, o, nullptr, d_in, d_out, static_cast<cudaStream_t>(stream), nullptr);
  });
}

extern "C" int
rtkb_parker_short_scan(const rtkb_geometry * g, const rtkb_image_desc * proj, double threshold, const float * d_in,
                       float * d_out, void * stream, int * is_short_scan)
{
  RTKB_TRACE();
  return guarded([&] {
    if (!std::isfinite(threshold))
      return rtkb::fail(RTKB_ERR_INVALID_ARGUMENT, "invalid angular gap threshold");
    Options o;
    o.parker = true;
    o.threshold = threshold;
    return run_filters(g, proj, o, nullptr, d_in, d_out, static_cast<cudaStream_t>(stream), is_short_scan);
  });
}

extern "C" int
rtkb_displaced_detector_region(const rtkb_geometry * g, const rtkb_image_desc * proj, int pad, rtkb_image_desc * out,
                               int * weighted)
{
  RTKB_TRACE();
  return guarded([&] {
    std::string why;
    if (!g || !out)
      return rtkb::fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
    if (!rtkb::desc_valid(proj, why))
      return rtkb::fail(RTKB_ERR_INVALID_ARGUMENT, why);
    rtkb::DisplacedInfo info;
    int                 rc = rtkb::displaced_region(g->g, *proj, pad != 0, info);
    if (rc != RTKB_OK)
      return rc;
    *out = info.weighted ? info.out : *proj;
    if (weighted)
      *weighted = info.weighted ? 1 : 0;
    return RTKB_OK;
  });
}

extern "C" int
rtkb_displaced_detector(const rtkb_geometry * g, const rtkb_image_desc * proj, int pad, const float * d_in,
                        float * d_out, void * stream)
{
  RTKB_TRACE();
  return guarded([&] {
    Options o;
    o.displaced = true;
    o.pad = pad != 0;
    return run_filters(g, proj, o, nullptr, d_in, d_out, static_cast<cudaStream_t>(stream), nullptr);
  });
}

extern "C" int
rtkb_ramp_kernel(int nu, double spacing, const rtkb_ramp_params * p, int * padded, double * kernel)
{
  RTKB_TRACE();
  return guarded([&] {
    if (nu <= 0 || !p || !padded || !std::isfinite(spacing) || spacing == 0.)
      return rtkb::fail(RTKB_ERR_INVALID_ARGUMENT, "invalid ramp kernel arguments");
    const int N = rtkb::ramp_padded_size(nu, *p);
    *padded = N;
    if (kernel)
    {
      if ((N & (N - 1)) != 0)
        return rtkb::fail(RTKB_ERR_UNSUPPORTED, "kernel evaluation needs a power-of-two padded size");
      std::vector<double> K;
      rtkb::ramp_kernel(N, spacing, *p, K);
      std::copy(K.begin(), K.end(), kernel);
    }
    return RTKB_OK;
  });
}

extern "C" int
rtkb_ramp_filter(const rtkb_image_desc * proj, const rtkb_ramp_params * p, const float * d_in, float * d_out,
                 void * stream)
{
  RTKB_TRACE();
  return guarded([&] {
    if (!p)
      return rtkb::fail(RTKB_ERR_INVALID_ARGUMENT, "null ramp parameters");
    std::string why;
    if (!rtkb::desc_valid(proj, why))
      return rtkb::fail(RTKB_ERR_INVALID_ARGUMENT, why);
    // the ramp needs no geometry: use a placeholder with enough projections
    rtkb_geometry g;
    const int     total = proj->index[2] + proj->size[2];
    if (proj->index[2] < 0)
      return rtkb::fail(RTKB_ERR_INVALID_ARGUMENT, "negative projection index");
    g.g.p.resize(total);
    Options o;
    o.ramp = true;
    o.rp = *p;
    return run_filters(&g, proj, o, nullptr, d_in, d_out, static_cast<cudaStream_t>(stream), nullptr);
  });
}

extern "C" int
rtkb_fdk_preprocess(const rtkb_geometry * g, const rtkb_image_desc * proj, const rtkb_fdk_preprocess_params * p,
                    rtkb_image_desc * out, const float * d_in, float * d_out, void * stream)
{
  RTKB_TRACE();
  return guarded([&] {
    if (!p)
      return rtkb::fail(RTKB_ERR_INVALID_ARGUMENT, "null preprocessing parameters");
    Options o;
    o.displaced = p->displaced_detector != 0;
    o.pad = p->pad_on_truncated_side != 0;
    o.parker = p->short_scan != 0;
    o.threshold = p->angular_gap_threshold > 0. ? p->angular_gap_threshold : 3.14159265358979323846 / 9;
    o.fdk = true;
    o.ramp = true;
    o.rp = p->ramp;
    return run_filters(g, proj, o, out, d_in, d_out, static_cast<cudaStream_t>(stream), nullptr);
  });
}

extern "C" int
rtkb_fdk_preprocess_batch(rtkb_fdk_preprocess_problem * problems, int n, const rtkb_fdk_preprocess_params * p,
                          void * stream)
{
  RTKB_TRACE();
  return guarded([&] {
    using namespace rtkb;
    if (!p)
      return fail(RTKB_ERR_INVALID_ARGUMENT, "null preprocessing parameters");
    if (n < 0 || (n > 0 && !problems))
      return fail(RTKB_ERR_INVALID_ARGUMENT, "invalid problem list");
    Options o;
    o.displaced = p->displaced_detector != 0;
    o.pad = p->pad_on_truncated_side != 0;
    o.parker = p->short_scan != 0;
    o.threshold = p->angular_gap_threshold > 0. ? p->angular_gap_threshold : 3.14159265358979323846 / 9;
    o.fdk = true;
    o.ramp = true;
    o.rp = p->ramp;
    // every problem's host half first: nothing is launched unless all are valid
    std::vector<Prepared> P(n);
    for (int i = 0; i < n; i++)
    {
      const rtkb_fdk_preprocess_problem & q = problems[i];
      const int rc = prepare_filters(q.geometry, &q.proj, o, &problems[i].out, q.d_in, q.d_out, nullptr, P[i]);
      if (rc != RTKB_OK)
        return rc;
    }
    if (n == 0)
      return (int)RTKB_OK;
    // one device block: every problem's tables, then per padded length N a
    // problem table and its pair ranges (one launch per N)
    struct Group
    {
      int              N;
      std::vector<int> idx;
      size_t           o_args = 0, o_begin = 0;
      long long        pairs = 0;
    };
    std::vector<Group> groups;
    for (int i = 0; i < n; i++)
    {
      auto it = std::find_if(groups.begin(), groups.end(), [&](const Group & gr) { return gr.N == P[i].a.N; });
      if (it == groups.end())
      {
        groups.push_back(Group{ P[i].a.N, {} });
        it = groups.end() - 1;
      }
      it->idx.push_back(i);
    }
    std::vector<size_t> offs(n);
    size_t              off = 0;
    for (int i = 0; i < n; i++)
    {
      offs[i] = off;
      off = align256(off + P[i].blob.size());
    }
    for (Group & gr : groups)
    {
      gr.o_args = off;
      off = align256(off + gr.idx.size() * sizeof(FilterArgs));
      gr.o_begin = off;
      off = align256(off + (gr.idx.size() + 1) * sizeof(long long));
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    void *       scratch = nullptr;
    RTKB_CUDA_TRY(rtkb::scratch_malloc(&scratch, off, st));
    char *                     base = static_cast<char *>(scratch);
    std::vector<unsigned char> host(off, 0);
    for (int i = 0; i < n; i++)
    {
      if (!P[i].blob.empty())
        std::memcpy(host.data() + offs[i], P[i].blob.data(), P[i].blob.size());
      bind_filters(P[i], base + offs[i]);
    }
    for (Group & gr : groups)
    {
      long long acc = 0;
      for (size_t k = 0; k < gr.idx.size(); k++)
      {
        std::memcpy(host.data() + gr.o_args + k * sizeof(FilterArgs), &P[gr.idx[k]].a, sizeof(FilterArgs));
        std::memcpy(host.data() + gr.o_begin + k * sizeof(long long), &acc, sizeof(long long));
        acc += P[gr.idx[k]].pairs;
      }
      std::memcpy(host.data() + gr.o_begin + gr.idx.size() * sizeof(long long), &acc, sizeof(long long));
      gr.pairs = acc;
    }
    int         rc = RTKB_OK;
    cudaError_t e = cudaMemcpyAsync(scratch, host.data(), off, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess)
      rc = cuda_fail(e, "cudaMemcpyAsync");
    for (size_t k = 0; k < groups.size() && rc == RTKB_OK; k++)
    {
      const Group &    gr = groups[k];
      const Prepared & f = P[gr.idx[0]]; // the group's pass twiddles (one set per N)
      e = launch_ramp_n(gr.N, f.a, reinterpret_cast<const FilterArgs *>(base + gr.o_args),
                        reinterpret_cast<const long long *>(base + gr.o_begin), (int)gr.idx.size(), gr.pairs, f.a.tw,
                        f.tw_len, st);
      if (e != cudaSuccess)
        rc = cuda_fail(e, "ramp_fft_kernel launch");
    }
    // (a copy from pageable memory returns once its source has been staged)
    cudaError_t fe = rtkb::scratch_free(scratch, st);
    if (rc == RTKB_OK && fe != cudaSuccess)
      rc = cuda_fail(fe, "cudaFreeAsync");
    return rc;
  });
}

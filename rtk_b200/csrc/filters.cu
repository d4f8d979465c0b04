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
// while the current one is transformed.  With N/16 threads per CTA (N >= 1024)
// a thread's 16 columns are both the inputs of its first-pass butterfly and
// the outputs of its last-pass butterflies, so the load, the kernel product
// and the store never touch shared memory; butterfly sums and differences use
// packed FP32 pairs (FADD2 / FFMA2).  FDK cos(gamma) weights come from
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
  int            period; // RTK's padded length: the circular convolution's period (N, or <= (N+1)/2 when embedded)
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

// T[s][c][r] = A[s][r][c] for r < rows, c < cols: 32 x 32 tiles through shared
// memory, so that both the reads and the writes are coalesced.
// grid: (column tiles, row tiles, projections), block 32 x 8
__global__ void __launch_bounds__(256)
transpose_rc_kernel(const float * __restrict__ A, float * __restrict__ T, int rows, int cols)
{
  __shared__ float tile[32][33];
  const long long base = (long long)blockIdx.z * rows * cols;
  const int       c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += 8)
  {
    const int r = r0 + k, c = c0 + threadIdx.x;
    if (r < rows && c < cols)
      tile[k][threadIdx.x] = A[base + (long long)r * cols + c];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += 8)
  {
    const int c = c0 + k, r = r0 + threadIdx.x;
    if (r < rows && c < cols)
      T[base + (long long)c * rows + r] = tile[threadIdx.x][k];
  }
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

// Complex sum and difference as packed FP32 pairs (one FADD2 / FFMA2 each
// instead of two scalar instructions; x - y = fma(y, -1, x) rounds once, so
// both are bit-identical to the scalar forms).
__device__ __forceinline__ float2
cadd(float2 x, float2 y)
{
  return __fadd2_rn(x, y);
}

__device__ __forceinline__ float2
csub(float2 x, float2 y)
{
  return __ffma2_rn(y, make_float2(-1.f, -1.f), x);
}

// (x - y) e^{-2 pi i j / L} for the constant twiddles of a size-L (2, 4, 8)
// DFT; the -i rotation is formed directly from x and y.
__device__ __forceinline__ float2
diff_rot(float2 x, float2 y, int j, int L)
{
  constexpr float c = 0.70710678118654752440f; // sqrt(1/2)
  if (L == 2 || j == 0)
    return csub(x, y);
  if (L == 4 || j == 2)
    return make_float2(x.y - y.y, y.x - x.x);
  const float2 d = csub(x, y);
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
        v[i + j] = cadd(x, y);
        v[i + j + half] = diff_rot(x, y, j, 2 * half);
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

// W16^j = e^{-2 pi i j/16}, j = 0..7
__device__ __forceinline__ float2
w16(float2 d, int j)
{
  constexpr float c[8] = { 1.f, 0.92387953251128675613f, 0.70710678118654752440f, 0.38268343236508977173f,
                           0.f, -0.38268343236508977173f, -0.70710678118654752440f, -0.92387953251128675613f };
  constexpr float sn[8] = { 0.f, 0.38268343236508977173f, 0.70710678118654752440f, 0.92387953251128675613f,
                            1.f, 0.92387953251128675613f, 0.70710678118654752440f, 0.38268343236508977173f };
  return make_float2(d.x * c[j] + d.y * sn[j], d.y * c[j] - d.x * sn[j]);
}

// Stages 2-4 of the 16-point DFT (three radix-2 levels) and the 4-bit reversal.
__device__ __forceinline__ void
dft16_tail(float2 (&v)[16])
{
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
        v[i + j] = cadd(x, y);
        v[i + j + half] = diff_rot(x, y, j, 2 * half);
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

// In-register forward DFT of size 16 (radix-2 decimation in frequency with the
// W16^j constants, then the 4-bit reversal).
__device__ __forceinline__ void
dft16(float2 (&v)[16])
{
#pragma unroll
  for (int j = 0; j < 8; j++)
  {
    const float2 x = v[j], y = v[j + 8];
    v[j] = cadd(x, y);
    if (j == 0)
      v[j + 8] = csub(x, y);
    else if (j == 4)
      v[j + 8] = make_float2(x.y - y.y, y.x - x.x); // -i (x - y)
    else
      v[j + 8] = w16(csub(x, y), j);
  }
  dft16_tail(v);
}

// The same DFT of an input whose upper half v[8..15] is zero: the first
// stage's sums are the inputs themselves (bit-identical: x + 0 = x).
__device__ __forceinline__ void
dft16_upper_zero(float2 (&v)[16])
{
#pragma unroll
  for (int j = 0; j < 8; j++)
  {
    const float2 x = v[j];
    if (j == 0)
      v[j + 8] = x;
    else if (j == 4)
      v[j + 8] = make_float2(x.y, -x.x);
    else
      v[j + 8] = w16(x, j);
  }
  dft16_tail(v);
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

// v[r] *= w^r for r = 1..R-1, w = e^{-2 pi i k / (Ns R)}: the powers 1, 2, 4
// and 8 from the pass's twiddle rows, the others as their products.
template <int R, int Ns>
__device__ __forceinline__ void
twiddle(float2 (&v)[R], const float2 * __restrict__ twp, int k)
{
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
    twiddle<R, Ns>(v, twp, k);
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

// First pass (Ns = 1, radix 16) from registers: v holds the columns
// threadIdx.x + i N/16, which are exactly this thread's butterfly inputs.
template <int N, bool UPPER_ZERO = false>
__device__ __forceinline__ void
fft_first_regs(float2 (&v)[16], float2 * __restrict__ dst)
{
  if constexpr (UPPER_ZERO)
    dft16_upper_zero(v);
  else
    dft16(v);
#pragma unroll
  for (int r = 0; r < 16; r++)
    dst[pidx(16 * threadIdx.x + r)] = v[r];
}

// Last pass (Ns R = N) into registers: with T = N/16 threads a thread does
// 16/R butterflies j = threadIdx.x + jj T (k = j), whose outputs j + r Ns are
// the columns threadIdx.x + m T, m = jj + r 16/R -- the same column set as
// the first pass reads.
template <int N, int T, int Ns, int R>
__device__ __forceinline__ void
fft_last_regs(const float2 * __restrict__ src, const float2 * __restrict__ twp, float2 (&out)[16])
{
  constexpr int per = Ns / T;
  static_assert(Ns * R == N && per * R == 16, "last pass covers the row with 16 outputs per thread");
#pragma unroll
  for (int jj = 0; jj < per; jj++)
  {
    const int j = threadIdx.x + jj * T;
    float2    v[R];
#pragma unroll
    for (int r = 0; r < R; r++)
      v[r] = src[pidx(j + r * Ns)];
    twiddle<R, Ns>(v, twp, j);
    dft_any<R>(v);
#pragma unroll
    for (int r = 0; r < R; r++)
      out[jj + r * per] = v[r];
  }
}

// Passes Ns, 16 Ns, ... of a length-N transform whose first pass is done:
// radix-16 passes through shared memory, the last one into registers.
// `spare` receives the buffer the last pass did not read (free to write
// without a barrier).
template <int N, int T, int Ns>
__device__ __forceinline__ void
fft_rest_regs(float2 * src, float2 * dst, const float2 * tw, float2 (&out)[16], float2 *& spare)
{
  if constexpr (N / Ns <= 16)
  {
    fft_last_regs<N, T, Ns, N / Ns>(src, tw, out);
    spare = dst;
  }
  else
  {
    fft_pass_c<N, T, Ns, 16>(src, dst, tw);
    __syncthreads();
    fft_rest_regs<N, T, Ns * 16>(dst, src, tw + 4 * Ns, out, spare);
  }
}

// The two rows of row pair pr (the second absent past the last row of an odd
// stack): projection and row indices.
struct PairRows
{
  int  sa, ra, sb, rb;
  bool hb;
};

__device__ __forceinline__ PairRows
pair_rows(const FilterArgs & a, int pr)
{
  const unsigned row = 2u * (unsigned)pr, nv = (unsigned)a.nv;
  PairRows       q;
  q.sa = (int)(row / nv);
  q.ra = (int)(row - (unsigned)q.sa * nv);
  q.hb = (long long)row + 1 < (long long)a.nv * a.np;
  q.sb = q.sa;
  q.rb = q.ra + 1;
  if (q.rb == a.nv)
  {
    q.sb = q.sa + 1;
    q.rb = 0;
  }
  if (!q.hb)
  {
    q.sb = q.sa;
    q.rb = q.ra;
  }
  return q;
}

// Ohnesorge mirror extrapolation (PadInputImageRegion :218-258) in the
// shared row b0 (the row at columns 0..nu-1, zeros after): left values wrap
// to the end of the convolution's period (the buffer's end unless the period
// is embedded in a longer FFT).
__device__ __forceinline__ void
mirror_pad(const FilterArgs & a, float2 * b0, int nu)
{
  const float2 SA = b0[pidx(1)], SE = b0[pidx(nu - 1)];
  for (int bq = 1 + threadIdx.x; bq <= a.next; bq += blockDim.x)
  {
    const float  w = __ldg(a.mw + bq);
    const float2 l = b0[pidx(bq)], r = b0[pidx(nu - 1 - bq)];
    b0[pidx(a.period - bq)] = make_float2(w * (2.f * SA.x - l.x), w * (2.f * SA.y - l.y));
    b0[pidx(nu - 1 + bq)] = make_float2(w * (2.f * SE.x - r.x), w * (2.f * SE.y - r.y));
  }
}

// Ramp filter of the row pairs first, first + stride, ... < pairs of one stack
// (two real rows as one complex sequence); the pass twiddles and the stack's
// ramp kernel, pre-scaled by 1/N (a power of two: exact), are in shared
// memory already.  The next pair's raw pixels are prefetched into registers
// while the current pair is transformed.  With N/16 threads (N >= 1024) the
// row pair stays in registers from the load to the first pass, from the last
// forward pass through the kernel product to the first inverse pass, and from
// the last inverse pass to the store.  UZ (upper zero): the row occupies at
// most the lower half of the padded buffer and nothing is mirrored, so the
// upper 8 of a thread's 16 columns are zero on input and unused on output.
template <int N, bool UZ>
__device__ __forceinline__ void
ramp_pairs(const FilterArgs & a, int first, int pairs, int stride, float2 * b0, float2 * b1, const float2 * tws,
           const float * Ks)
{
  constexpr int  T = kRampThreads<N>;
  constexpr bool kRegs = (T == N / 16);
  static_assert(kRegs || !UZ, "the upper-zero form needs N/16 threads");
  constexpr int  kCols = UZ ? 8 : 16;
  const int      nu = a.nu_out;
  // columns threadIdx.x + i T; T >= N / 16, so 16 columns per thread cover the row
  float          pa[kCols], pb[kCols];
  auto           prefetch = [&](const PairRows & q) {
#pragma unroll
    for (int i = 0; i < kCols; i++)
    {
      const int c = threadIdx.x + i * T;
      pa[i] = (c < nu) ? raw_pixel(a, q.sa, q.ra, c) : 0.f;
      pb[i] = (c < nu && q.hb) ? raw_pixel(a, q.sb, q.rb, c) : 0.f;
    }
  };
  PairRows q{};
  if (first < pairs)
  {
    q = pair_rows(a, first);
    prefetch(q);
  }
  for (int pr = first; pr < pairs; pr += stride)
  {
    const PairRows  cur = q;
    const RowWeight wa = row_weight(a, cur.sa, cur.ra);
    const RowWeight wb = row_weight(a, cur.sb, cur.rb);
    float2          v[16];
#pragma unroll
    for (int i = 0; i < kCols; i++)
    {
      const int c = threadIdx.x + i * T;
      v[i] = make_float2((c < nu) ? apply_weights(a, wa, cur.sa, c, pa[i]) : 0.f,
                         (c < nu && cur.hb) ? apply_weights(a, wb, cur.sb, c, pb[i]) : 0.f);
    }
    if (pr + stride < pairs)
    {
      q = pair_rows(a, pr + stride);
      prefetch(q);
    }
    float * oa = a.out + ((long long)cur.sa * a.nv + cur.ra) * nu;
    float * ob = a.out + ((long long)cur.sb * a.nv + cur.rb) * nu;
    __syncthreads(); // the previous pair's last pass has read the shared buffers
    if constexpr (kRegs)
    {
      if (!UZ && a.next > 0)
      {
#pragma unroll
        for (int i = 0; i < 16; i++)
          b0[pidx(threadIdx.x + i * T)] = v[i];
        __syncthreads();
        mirror_pad(a, b0, nu);
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 16; i++)
          v[i] = b0[pidx(threadIdx.x + i * T)];
        __syncthreads();
      }
      fft_first_regs<N, UZ>(v, b0);
      __syncthreads();
      float2 * spare;
      fft_rest_regs<N, T, 16>(b0, b1, tws, v, spare);
      // times the real, even kernel, conjugated: the inverse transform is
      // conj(FFT(conj(K X))) (the 1/N is in K)
#pragma unroll
      for (int m = 0; m < 16; m++)
      {
        const int   f = threadIdx.x + m * T;
        const float k = Ks[min(f, N - f)];
        v[m] = make_float2(v[m].x * k, -v[m].y * k);
      }
      fft_first_regs<N>(v, spare);
      __syncthreads();
      float2 * unused;
      fft_rest_regs<N, T, 16>(spare, spare == b0 ? b1 : b0, tws, v, unused);
#pragma unroll
      for (int m = 0; m < kCols; m++)
      {
        const int c = threadIdx.x + m * T;
        if (c < nu)
        {
          oa[c] = v[m].x;
          if (cur.hb)
            ob[c] = -v[m].y;
        }
      }
    }
    else
    {
#pragma unroll
      for (int i = 0; i < 16; i++)
      {
        const int c = threadIdx.x + i * T;
        if (c < N)
          b0[pidx(c)] = v[i];
      }
      __syncthreads();
      if (a.next > 0)
      {
        mirror_pad(a, b0, nu);
        __syncthreads();
      }
      float2 * X = fft_chain<N, T, 1>(b0, b1, tws);
      float2 * other = (X == b0) ? b1 : b0;
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
        oa[c] = z.x;
        if (cur.hb)
          ob[c] = -z.y;
      }
    }
  }
}

// Shared-memory ramp kernel of one stack, times 1/N (exact: N is a power of two)
template <int N>
__device__ __forceinline__ void
load_kernel(const float * __restrict__ K, float * Ks)
{
  constexpr float inv = 1.f / (float)N;
  for (int i = threadIdx.x; i <= N / 2; i += blockDim.x)
    Ks[i] = K[i] * inv;
}

// Ramp filter of one stack, persistent: each CTA loads the pass twiddles and
// the ramp kernel into shared memory once, then filters row pairs until the
// stack is done.  The stack's description is a kernel parameter.
// 128 registers per thread at most: (threads x 128) x (512 / threads) = 64 K
template <int N, bool UZ>
__global__ void __launch_bounds__(kRampThreads<N>, 512 / kRampThreads<N>)
ramp_fft_kernel(FilterArgs a, int tw_len)
{
  constexpr int P = pidx(N);
  extern __shared__ float2 sbuf[];
  float2 *      tws = sbuf + 2 * P;
  float *       Ks = reinterpret_cast<float *>(tws + tw_len);
  for (int i = threadIdx.x; i < tw_len; i += blockDim.x)
    tws[i] = a.tw[i];
  load_kernel<N>(a.K, Ks);
  const int pairs = (a.nv * a.np + 1) / 2;
  ramp_pairs<N, UZ>(a, blockIdx.x, pairs, gridDim.x, sbuf, sbuf + P, tws, Ks);
}

// Ramp filter of many stacks of one padded length N, persistent: the global
// row-pair range of stack q is [pair_begin[q], pair_begin[q + 1]); a CTA takes
// the pairs blockIdx.x + k gridDim.x, stack after stack, loading each stack's
// description (into shared memory) and ramp kernel when it reaches it.  The
// pass twiddles are shared by every stack of the launch.
template <int N, bool UZ>
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
    load_kernel<N>(probs[q].K, Ks);
    __syncthreads();
    ramp_pairs<N, UZ>(cur, (int)first, (int)(hi - lo), gridDim.x, sbuf, sbuf + P, tws, Ks);
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

template <int N, bool UZ>
static cudaError_t
launch_ramp_uz(const FilterArgs & a, int tw_len, long long pairs, cudaStream_t st)
{
  long long   grid = 0;
  cudaError_t e = ramp_grid(ramp_fft_kernel<N, UZ>, kRampThreads<N>, ramp_smem<N>(tw_len), pairs, grid);
  if (e == cudaSuccess && pairs > 0)
  {
    ramp_fft_kernel<N, UZ><<<(unsigned)grid, kRampThreads<N>, ramp_smem<N>(tw_len), st>>>(a, tw_len);
    e = cudaGetLastError();
  }
  return e;
}

// The upper-zero form exists for N/16-thread CTAs (N >= 1024) only.
template <int N>
static cudaError_t
launch_ramp(const FilterArgs & a, int tw_len, long long pairs, bool uz, cudaStream_t st)
{
  if constexpr (kRampThreads<N> == N / 16)
    if (uz)
      return launch_ramp_uz<N, true>(a, tw_len, pairs, st);
  return launch_ramp_uz<N, false>(a, tw_len, pairs, st);
}

template <int N, bool UZ>
static cudaError_t
launch_ramp_batch_uz(const FilterArgs * d_probs, const long long * d_begin, int nprob, long long pairs,
                     const float2 * d_tw, int tw_len, cudaStream_t st)
{
  long long   grid = 0;
  cudaError_t e = ramp_grid(ramp_fft_batch_kernel<N, UZ>, kRampThreads<N>, ramp_smem<N>(tw_len), pairs, grid);
  if (e == cudaSuccess && pairs > 0)
  {
    ramp_fft_batch_kernel<N, UZ><<<(unsigned)grid, kRampThreads<N>, ramp_smem<N>(tw_len), st>>>(d_probs, d_begin, nprob,
                                                                                           d_tw, tw_len);
    e = cudaGetLastError();
  }
  return e;
}

template <int N>
static cudaError_t
launch_ramp_batch(const FilterArgs * d_probs, const long long * d_begin, int nprob, long long pairs,
                  const float2 * d_tw, int tw_len, bool uz, cudaStream_t st)
{
  if constexpr (kRampThreads<N> == N / 16)
    if (uz)
      return launch_ramp_batch_uz<N, true>(d_probs, d_begin, nprob, pairs, d_tw, tw_len, st);
  return launch_ramp_batch_uz<N, false>(d_probs, d_begin, nprob, pairs, d_tw, tw_len, st);
}

// Whether a stack's rows fit the upper-zero form: at most N/2 columns and no
// mirror extrapolation (the N/16-thread condition is the launcher's).
static bool
upper_zero(const FilterArgs & a)
{
  return a.next == 0 && 2 * a.nu_out <= a.N;
}

// One stack (d_probs == nullptr: a) or a table of nprob stacks of length N;
// uz: every stack has upper_zero().
static cudaError_t
launch_ramp_n(int N, const FilterArgs & a, const FilterArgs * d_probs, const long long * d_begin, int nprob,
              long long pairs, const float2 * d_tw, int tw_len, bool uz, cudaStream_t st)
{
#define RTKB_RAMP_CASE(n)                                                                                              \
  case n:                                                                                                              \
    return d_probs ? launch_ramp_batch<n>(d_probs, d_begin, nprob, pairs, d_tw, tw_len, uz, st)                        \
                   : launch_ramp<n>(a, tw_len, pairs, uz, st)
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
      return d_probs ? launch_ramp_batch<8192>(d_probs, d_begin, nprob, pairs, d_tw, tw_len, uz, st)
                     : launch_ramp<8192>(a, tw_len, pairs, uz, st);
  }
#undef RTKB_RAMP_CASE
}

struct Options
{
  bool             displaced = false, pad = true, parker = false, fdk = false, ramp = false;
  bool             offset_fov = false; // DisplacedDetectorForOffsetFieldOfViewImageFilter
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
  // 2-D kernel (HannCutFrequencyY): the column pass's arguments (rows = the
  // stack's columns, N = padded height; in/out set when it runs) and tables
  FilterArgs                 col{};
  size_t                     o_Ky = 0, o_twy = 0;
  int                        tw_len_y = 0;
  long long                  col_pairs = 0;
  bool                       colpass = false;
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
    int           rc = o.offset_fov ? offset_fov_region(G, *in, info) : displaced_region(G, *in, o.pad, info);
    if (rc != RTKB_OK)
      return rc;
    if (info.weighted)
    {
      out = info.out;
      shift = info.shift;
      if (o.offset_fov)
        offset_fov_weights(G, *in, info, wd);
      else
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
    // RTK's padded length P is the period of the circular convolution; a P
    // that is not a power of two (greatest prime factor above 2, RTK built
    // with FFTW) is embedded in a power-of-two FFT of length >= 2P - 1
    const int P = ramp_padded_size(nu_out, o.rp);
    const int N = P >= 1 ? fft_length_for_period(P) : 0;
    if (P < 2 || N > kMaxFFT)
      return fail(RTKB_ERR_UNSUPPORTED, "the ramp filter's FFT length (the padded row length, a power of two, or "
                                        "the power of two >= twice it otherwise) must be <= 8192");
    if ((long long)nv * np > 0x7ffffffe)
      return fail(RTKB_ERR_UNSUPPORTED, "the ramp filter indexes rows in 32 bits: nv * np must be < 2^31");
    std::vector<double> Kd, KM;
    ramp_kernel(P, out.spacing[0], o.rp, Kd);
    if (N != P)
      embed_spectrum(P, N, Kd, KM);
    K.assign(N != P ? KM.begin() : Kd.begin(), N != P ? KM.end() : Kd.end());
    pass_twiddles(N, tw);
    // the weights follow the full extent floor(t * nu) (UpdateTruncationMirrorWeights
    // :345-355); the mirror covers at most the zero padding (PadInputImageRegion :215-216)
    const int extent = (int)std::floor(o.rp.truncation_correction * nu_out);
    const int next = std::min(extent, (P - nu_out) / 2);
    if (next > 0 && extent == 1)
      return fail(RTKB_ERR_INVALID_ARGUMENT, "truncation correction extent of one pixel is undefined");
    if (next > 0)
      truncation_mirror_weights(extent, mw);
    a.N = N;
    a.period = P;
    a.next = next;
  }
  std::vector<float> Ky, twy;
  P.colpass = o.ramp && o.rp.hann_cut_y > 0.;
  if (P.colpass)
  {
    const int H = ramp_padded_size_y(nv, o.rp);
    const int M = H >= 1 ? fft_length_for_period(H) : 0;
    if (H < 2 || M > kMaxFFT)
      return fail(RTKB_ERR_UNSUPPORTED, "the 2-D kernel's column FFT length (the padded height, a power of two, or "
                                        "the power of two >= twice it otherwise) must be <= 8192");
    if ((long long)nu_out * np > 0x7ffffffe)
      return fail(RTKB_ERR_UNSUPPORTED, "the 2-D ramp kernel indexes columns in 32 bits: nu * np must be < 2^31");
    std::vector<double> Wd, WM;
    ramp_window_y(H, o.rp, Wd);
    if (M != H)
      embed_spectrum(H, M, Wd, WM);
    Ky.assign(M != H ? WM.begin() : Wd.begin(), M != H ? WM.end() : Wd.end());
    pass_twiddles(M, twy);
    FilterArgs c{};
    c.nu_in = nv;
    c.nu_out = nv;
    c.nv = nu_out;
    c.np = np;
    c.N = M;
    c.period = H;
    P.col = c;
    P.col_pairs = ((long long)nu_out * np + 1) / 2;
  }
  P.blob.clear();
  P.o_fdk = append(P.blob, fdkp);
  P.o_colw = append(P.blob, colw);
  P.o_K = append(P.blob, K);
  P.o_tw = append(P.blob, tw);
  P.o_mw = append(P.blob, mw);
  P.o_Ky = append(P.blob, Ky);
  P.o_twy = append(P.blob, twy);
  P.tw_len_y = (int)(twy.size() / 2);
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
  if (P.colpass)
  {
    P.col.K = reinterpret_cast<const float *>(base + P.o_Ky);
    P.col.tw = P.tw_len_y ? reinterpret_cast<const float2 *>(base + P.o_twy) : nullptr;
  }
}

// The vertical part of the 2-D kernel (HannCutFrequencyY).  The kernel is the
// 1-D ramp kernel times a window of the rows' frequency, so the 2-D
// convolution (FFTProjectionsConvolutionImageFilter::ThreadedGenerateData with
// the 2-D kernel, include/rtkFFTProjectionsConvolutionImageFilter.hxx:121-198)
// is the row filter followed by a circular convolution of every column,
// zero-padded to the padded height H, with the window's inverse transform.  The
// columns of d_out become rows of a transposed copy, which the ramp FFT kernel
// filters in place with the window as its (real, even) kernel, and the result
// is transposed back into d_out.
int
column_pass(Prepared & P, float * d_out, cudaStream_t st)
{
  using namespace rtkb;
  const int nu = P.a.nu_out, nv = P.a.nv, np = P.a.np;
  void *    t = nullptr;
  RTKB_CUDA_TRY(rtkb::scratch_malloc(&t, (size_t)nu * nv * np * sizeof(float), st));
  float *     T = static_cast<float *>(t);
  int         rc = RTKB_OK;
  const dim3  blk(32, 8);
  transpose_rc_kernel<<<dim3((unsigned)((nu + 31) / 32), (unsigned)((nv + 31) / 32), (unsigned)np), blk, 0, st>>>(
    d_out, T, nv, nu);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
  {
    P.col.in = T;
    P.col.out = T;
    e = launch_ramp_n(P.col.N, P.col, nullptr, nullptr, 1, P.col_pairs, P.col.tw, P.tw_len_y, upper_zero(P.col), st);
  }
  if (e == cudaSuccess)
  {
    transpose_rc_kernel<<<dim3((unsigned)((nv + 31) / 32), (unsigned)((nu + 31) / 32), (unsigned)np), blk, 0, st>>>(
      T, d_out, nu, nv);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess)
    rc = cuda_fail(e, "2-D ramp kernel column pass");
  const cudaError_t fe = rtkb::scratch_free(t, st);
  if (rc == RTKB_OK && fe != cudaSuccess)
    rc = cuda_fail(fe, "cudaFreeAsync");
  return rc;
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
    e = launch_ramp_n(P.a.N, P.a, nullptr, nullptr, 1, P.pairs, P.a.tw, P.tw_len, upper_zero(P.a), st);
    if (e != cudaSuccess)
      rc = cuda_fail(e, "ramp_fft_kernel launch");
    else if (P.colpass)
      rc = column_pass(P, d_out, st);
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
rtkb_displaced_detector_offset_fov_region(const rtkb_geometry * g, const rtkb_image_desc * proj, rtkb_image_desc * out,
                                          int * weighted)
{
  RTKB_TRACE();
  return guarded([&] {
    std::string why;
    if (!g || !out)
      return rtkb::fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
    if (!rtkb::desc_valid(proj, why))
      return rtkb::fail(RTKB_ERR_INVALID_ARGUMENT, why);
    if (g->g.radius_cylindrical != 0. || (!g->g.p.empty() && g->g.p[0].sdd == 0.))
      return rtkb::fail(RTKB_ERR_UNSUPPORTED, "Displaced detector cannot handle cylindrical detector or parallel geometry");
    rtkb::DisplacedInfo info;
    int                 rc = rtkb::offset_fov_region(g->g, *proj, info);
    if (rc != RTKB_OK)
      return rc;
    *out = info.weighted ? info.out : *proj;
    if (weighted)
      *weighted = info.weighted ? 1 : 0;
    return RTKB_OK;
  });
}

extern "C" int
rtkb_displaced_detector_offset_fov(const rtkb_geometry * g, const rtkb_image_desc * proj, const float * d_in,
                                   float * d_out, void * stream)
{
  RTKB_TRACE();
  return guarded([&] {
    Options o;
    o.displaced = true;
    o.offset_fov = true;
    return run_filters(g, proj, o, nullptr, d_in, d_out, static_cast<cudaStream_t>(stream), nullptr);
  });
}

extern "C" int
rtkb_field_of_view_radius(const rtkb_geometry * g, const rtkb_image_desc * proj, int type, double * x, double * z,
                          double * r)
{
  RTKB_TRACE();
  return guarded([&] {
    std::string why;
    if (!g || !x || !z || !r || type < 0 || type > 2)
      return rtkb::fail(RTKB_ERR_INVALID_ARGUMENT, "invalid field-of-view arguments");
    if (!rtkb::desc_valid(proj, why))
      return rtkb::fail(RTKB_ERR_INVALID_ARGUMENT, why);
    const int rc = rtkb::fov_radius(g->g, *proj, type, *x, *z, *r);
    return rc == RTKB_OK || rc == RTKB_ERR_UNSUPPORTED
             ? rc
             : rtkb::fail(RTKB_ERR_INVALID_ARGUMENT, "no disc is seen by every projection (the programme has no solution)");
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
    o.offset_fov = p->displaced_detector == 2;
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
    o.offset_fov = p->displaced_detector == 2;
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
      bool             uz = true;
      for (int i : gr.idx)
        uz = uz && upper_zero(P[i].a);
      e = launch_ramp_n(gr.N, f.a, reinterpret_cast<const FilterArgs *>(base + gr.o_args),
                        reinterpret_cast<const long long *>(base + gr.o_begin), (int)gr.idx.size(), gr.pairs, f.a.tw,
                        f.tw_len, uz, st);
      if (e != cudaSuccess)
        rc = cuda_fail(e, "ramp_fft_kernel launch");
    }
    for (int i = 0; i < n && rc == RTKB_OK; i++)
      if (P[i].colpass)
        rc = column_pass(P[i], problems[i].d_out, st);
    // (a copy from pageable memory returns once its source has been staged)
    cudaError_t fe = rtkb::scratch_free(scratch, st);
    if (rc == RTKB_OK && fe != cudaSuccess)
      rc = cuda_fail(fe, "cudaFreeAsync");
    return rc;
  });
}

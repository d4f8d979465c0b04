// preprocess.cu -- raw detector counts to line integrals, upstream of the
// projectors: rtk::I0EstimationProjectionFilter
// (include/rtkI0EstimationProjectionFilter.hxx) and
// rtk::LUTbasedVariableI0RawToAttenuationImageFilter
// (include/rtkLUTbasedVariableI0RawToAttenuationImageFilter.hxx), the two
// filters rtk::ProjectionsReader chains for 16-bit raw projections.
//
// I0 estimation: a histogram of raw >> bitShift (16-bit input: 65536 >>
// bitShift bins) is built on the GPU, each CTA counting into its own copy in
// shared memory and adding it to the global histogram once; RTK's integer
// search for the dynamic range and the background mode then runs on the host
// on the 64 KB histogram, step for step (including the 16-bit type of the
// mode's count and of the bounds, as the filter declares them).
//
// Conversion: RTK builds a 65536-entry float lookup table
//   lut[r] = float(log(max(I0 - IDark, 1))) - float(log(double(max(float(r) - float(IDark), 1.f))))
// (ITK's subtract, threshold-below-1 and log image filters applied to the ramp
// 0..65535); the table is built the same way on the host and the GPU gathers
// from it (the first 224 KB staged in each CTA's shared memory, the rest read
// from L2): 2 bytes read and 4 written per pixel.
#include "rtkb200.h"
#include "rtkb_internal.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace
{
using rtkb::fail;

constexpr int kLutSize = 65536;

// Histogram of (raw >> shift) into hist (nbins <= 16384 with shift >= 2);
// per-CTA copy in shared memory.
__global__ void __launch_bounds__(512)
raw_histogram_kernel(const uint16_t * __restrict__ raw, long long n, int shift, int nbins,
                     unsigned int * __restrict__ hist)
{
  extern __shared__ unsigned int h[];
  for (int b = threadIdx.x; b < nbins; b += blockDim.x)
    h[b] = 0u;
  __syncthreads();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    atomicAdd(&h[raw[i] >> shift], 1u);
  __syncthreads();
  for (int b = threadIdx.x; b < nbins; b += blockDim.x)
    if (h[b])
      atomicAdd(&hist[b], h[b]);
}

// The same without a shared-memory copy (bit shifts below 2: up to 65536 bins)
__global__ void __launch_bounds__(256)
raw_histogram_global_kernel(const uint16_t * __restrict__ raw, long long n, int shift, unsigned int * __restrict__ hist)
{
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    atomicAdd(&hist[raw[i] >> shift], 1u);
}

// out = lut[raw], eight pixels per 16-byte load where the buffers allow it.
// Random 4-byte gathers from a 256 KB table in L2 move a 32-byte sector each;
// so each CTA (one per SM) first copies the table's first kSmemLut entries
// into shared memory and gathers from there, and only larger raw values read
// the table in global memory.
constexpr int kSmemLut = 57344; // 224 KB of the 227 KB a CTA may have

__device__ __forceinline__ float
lut_at(const float * __restrict__ s, const float * __restrict__ lut, unsigned r)
{
  return r < (unsigned)kSmemLut ? s[r] : __ldg(lut + r);
}

__global__ void __launch_bounds__(1024)
raw_lut_kernel(const uint16_t * __restrict__ raw, long long n, const float * __restrict__ lut, float * __restrict__ out)
{
  extern __shared__ float4 s4[];
  const float4 * g4 = reinterpret_cast<const float4 *>(lut);
  for (int k = threadIdx.x; k < kSmemLut / 4; k += blockDim.x)
    s4[k] = g4[k];
  __syncthreads();
  const float *   s = reinterpret_cast<const float *>(s4);
  const long long stride = (long long)gridDim.x * blockDim.x;
  const bool      vec = ((reinterpret_cast<uintptr_t>(raw) | reinterpret_cast<uintptr_t>(out)) & 15) == 0;
  const long long n8 = vec ? n / 8 : 0;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n8; q += stride)
  {
    const uint4 r = reinterpret_cast<const uint4 *>(raw)[q];
    float4      a, b;
    a.x = lut_at(s, lut, r.x & 0xffffu);
    a.y = lut_at(s, lut, r.x >> 16);
    a.z = lut_at(s, lut, r.y & 0xffffu);
    a.w = lut_at(s, lut, r.y >> 16);
    b.x = lut_at(s, lut, r.z & 0xffffu);
    b.y = lut_at(s, lut, r.z >> 16);
    b.z = lut_at(s, lut, r.w & 0xffffu);
    b.w = lut_at(s, lut, r.w >> 16);
    reinterpret_cast<float4 *>(out)[2 * q] = a;
    reinterpret_cast<float4 *>(out)[2 * q + 1] = b;
  }
  for (long long i = n8 * 8 + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride)
    out[i] = lut_at(s, lut, raw[i]);
}

// Water precorrection with at least 3 coefficients, in RTK's arithmetic: the
// products of the double coefficients and the float powers in double, the
// running sum rounded to float after each term, powers of v in float.  No
// fused multiply-adds, as an x86 build of the filter computes it.
constexpr int kMaxWaterCoefficients = 16;
struct WaterCoeffs
{
  double c[kMaxWaterCoefficients];
  int    n;
};

__global__ void __launch_bounds__(256)
water_precorrection_kernel(const float * in, float * out, long long n, WaterCoeffs k)
{
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
  {
    const float v = in[i];
    float       o = (float)__dadd_rn(k.c[0], __dmul_rn(k.c[1], (double)v));
    float       bpow = __fmul_rn(v, v);
    for (int j = 2; j < k.n; j++)
    {
      o = (float)__dadd_rn((double)o, __dmul_rn(k.c[j], (double)bpow));
      bpow = __fmul_rn(bpow, v);
    }
    out[i] = o;
  }
}

// two coefficients (not the identity): out = float(c0 + c1 v); one non-zero coefficient: out = c0
__global__ void __launch_bounds__(256)
water_affine_kernel(const float * in, float * out, long long n, double c0, double c1, bool constant)
{
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = constant ? (float)c0 : (float)__dadd_rn(c0, __dmul_rn(c1, (double)in[i]));
}

unsigned
grid_of(long long n)
{
  return (unsigned)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148LL * 8));
}
} // namespace

namespace rtkb
{
// RTK's search on the histogram (ThreadedGenerateData's last-thread block and
// AfterThreadedGenerateData), with the filter's types: Imin, Imax, I0, the
// mode's count and the half-maximum are of the 16-bit pixel type.
void
i0_search(const std::vector<unsigned int> & hist, int shift, unsigned int dyn_threshold, rtkb_i0_estimate & out)
{
  const size_t nbins = hist.size();
  size_t       imax = nbins - 1;
  while (hist[imax] <= dyn_threshold && imax > 0)
    --imax;
  // back to a non-empty bin.  RTK's loop runs past the end only when every bin
  // is empty, i.e. for an empty image, which the entry point refuses (image
  // sizes must be positive); for every other histogram the bound never binds.
  while (hist[imax] == 0 && imax + 1 < nbins)
    ++imax;
  size_t imin = 0;
  while (hist[imin] <= dyn_threshold && imin < imax)
    ++imin;
  while (hist[imin] == 0 && imin > 0)
    --imin;
  const uint16_t Imin = (uint16_t)(imin << shift), Imax = (uint16_t)(imax << shift);
  const unsigned start = (3u * (unsigned)(Imax >> 2)) >> shift;
  unsigned       idx = start, max_id = start;
  uint16_t       max_val = (uint16_t)hist[start];
  while (idx < (unsigned)(Imax >> shift))
  {
    if (hist[idx] >= max_val)
    {
      max_val = (uint16_t)hist[idx];
      max_id = idx;
    }
    ++idx;
  }
  const uint16_t I0 = (uint16_t)(max_id << shift);
  const uint16_t width = (uint16_t)(float)(max_val >> 1);
  unsigned       low = max_id;
  while (hist[low] > width && low > 0)
    --low;
  unsigned high = max_id;
  while (hist[high] > width && high < Imax && high + 1 < nbins)
    ++high;
  out.i0 = I0;
  out.i0_fwhm = (uint16_t)((high - low) << shift);
  out.imin = Imin;
  out.imax = Imax;
  out.low_bound = low << shift;
  out.high_bound = high << shift;
}

// lut[r] as RTK's LUT pipeline computes it (float ramp minus float(IDark),
// values below 1 set to 1, log in double rounded to float, subtracted from
// float(log(max(I0 - IDark, 1))))
void
raw_to_attenuation_lut(double i0, double idark, std::vector<float> & lut)
{
  lut.resize(kLutSize);
  const float c = (float)std::log(std::max(i0 - idark, 1.));
  const float d = (float)idark;
  for (int r = 0; r < kLutSize; r++)
  {
    float v = (float)r - d;
    if (v < 1.f)
      v = 1.f;
    lut[r] = c - (float)std::log((double)v);
  }
}
} // namespace rtkb

extern "C" int
rtkb_i0_estimation(const rtkb_image_desc * desc, const unsigned short * d_raw, int bit_shift,
                   unsigned int dyn_threshold, rtkb_i0_estimate * out, void * stream)
{
  RTKB_TRACE();
  using namespace rtkb;
  std::string why;
  if (!desc || !d_raw || !out)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  if (!desc_valid(desc, why))
    return fail(RTKB_ERR_INVALID_ARGUMENT, why);
  if (bit_shift < 0 || bit_shift > 8)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "bit shift must lie in 0..8");
  try
  {
    cudaStream_t    st = static_cast<cudaStream_t>(stream);
    const long long n = num_pixels(*desc);
    const int       nbins = kLutSize >> bit_shift;
    unsigned int *  d_hist = nullptr;
    RTKB_CUDA_TRY(scratch_malloc(&d_hist, (size_t)nbins * 4, st));
    cudaError_t e = cudaMemsetAsync(d_hist, 0, (size_t)nbins * 4, st);
    if (e == cudaSuccess && n > 0)
    {
      if (bit_shift >= 2)
      {
        const size_t smem = (size_t)nbins * 4;
        static_cast<void>(cudaFuncSetAttribute(raw_histogram_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)smem));
        const unsigned blocks = (unsigned)std::max<long long>(1, std::min<long long>((n + 511) / 512, 148LL * 2));
        raw_histogram_kernel<<<blocks, 512, smem, st>>>(d_raw, n, bit_shift, nbins, d_hist);
      }
      else
        raw_histogram_global_kernel<<<grid_of(n), 256, 0, st>>>(d_raw, n, bit_shift, d_hist);
      e = cudaGetLastError();
    }
    std::vector<unsigned int> hist(nbins);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(hist.data(), d_hist, (size_t)nbins * 4, cudaMemcpyDeviceToHost, st);
    const cudaError_t fe = scratch_free(d_hist, st);
    if (e == cudaSuccess)
      e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
      return cuda_fail(e, "I0 estimation");
    if (fe != cudaSuccess)
      return cuda_fail(fe, "cudaFreeAsync");
    i0_search(hist, bit_shift, dyn_threshold, *out);
    return RTKB_OK;
  }
  catch (...)
  {
    return fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

extern "C" int
rtkb_raw_to_attenuation(const rtkb_image_desc * desc, const unsigned short * d_raw, double i0, double idark,
                        float * d_out, void * stream)
{
  RTKB_TRACE();
  using namespace rtkb;
  std::string why;
  if (!desc || !d_raw || !d_out)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  if (!desc_valid(desc, why))
    return fail(RTKB_ERR_INVALID_ARGUMENT, why);
  if (!std::isfinite(i0) || !std::isfinite(idark))
    return fail(RTKB_ERR_INVALID_ARGUMENT, "I0 and IDark must be finite");
  try
  {
    std::vector<float> lut;
    raw_to_attenuation_lut(i0, idark, lut);
    cudaStream_t    st = static_cast<cudaStream_t>(stream);
    const long long n = num_pixels(*desc);
    float *         d_lut = nullptr;
    RTKB_CUDA_TRY(scratch_malloc(&d_lut, (size_t)kLutSize * 4, st));
    cudaError_t e = cudaMemcpyAsync(d_lut, lut.data(), (size_t)kLutSize * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && n > 0)
    {
      const size_t smem = (size_t)kSmemLut * 4;
      e = cudaFuncSetAttribute(raw_lut_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e == cudaSuccess)
      {
        const unsigned blocks = (unsigned)std::max<long long>(1, std::min<long long>((n + 8191) / 8192, 148));
        raw_lut_kernel<<<blocks, 1024, smem, st>>>(d_raw, n, d_lut, d_out);
        e = cudaGetLastError();
      }
    }
    const cudaError_t fe = scratch_free(d_lut, st);
    if (e != cudaSuccess)
      return cuda_fail(e, "raw to attenuation");
    return fe == cudaSuccess ? RTKB_OK : cuda_fail(fe, "cudaFreeAsync");
  }
  catch (...)
  {
    return fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

extern "C" int
rtkb_water_precorrection(const rtkb_image_desc * desc, const float * d_in, float * d_out, const double * coefficients,
                         int n_coefficients, void * stream)
{
  RTKB_TRACE();
  // WaterPrecorrectionImageFilter::DynamicThreadedGenerateData
  // (include/rtkWaterPrecorrectionImageFilter.hxx:14-62), an in-place filter:
  // the cases it leaves untouched (no coefficients, the identity (0, 1), a
  // single zero) pass the input through.
  using namespace rtkb;
  std::string why;
  if (!desc || !d_in || !d_out || (n_coefficients > 0 && !coefficients))
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  if (!desc_valid(desc, why))
    return fail(RTKB_ERR_INVALID_ARGUMENT, why);
  if (n_coefficients < 0 || n_coefficients > kMaxWaterCoefficients)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "water precorrection takes at most 16 coefficients");
  cudaStream_t    st = static_cast<cudaStream_t>(stream);
  const long long n = num_pixels(*desc);
  const double *  c = coefficients;
  cudaError_t     e = cudaSuccess;
  if (n_coefficients >= 3)
  {
    WaterCoeffs k{};
    for (int j = 0; j < n_coefficients; j++)
      k.c[j] = c[j];
    k.n = n_coefficients;
    water_precorrection_kernel<<<grid_of(n), 256, 0, st>>>(d_in, d_out, n, k);
    e = cudaGetLastError();
  }
  else if (n_coefficients == 2 && (c[0] != 0. || c[1] != 1.))
  {
    water_affine_kernel<<<grid_of(n), 256, 0, st>>>(d_in, d_out, n, c[0], c[1], false);
    e = cudaGetLastError();
  }
  else if (n_coefficients == 1 && c[0] != 0.)
  {
    water_affine_kernel<<<grid_of(n), 256, 0, st>>>(d_in, d_out, n, c[0], 0., true);
    e = cudaGetLastError();
  }
  else if (d_out != d_in)
    e = cudaMemcpyAsync(d_out, d_in, (size_t)n * 4, cudaMemcpyDeviceToDevice, st);
  return e == cudaSuccess ? RTKB_OK : cuda_fail(e, "water precorrection");
}

// regularized_cg.cu -- rtk::RegularizedConjugateGradientConeBeamReconstructionFilter
// (include/rtkRegularizedConjugateGradientConeBeamReconstructionFilter.hxx)
// on the conjugate-gradient plan (Joseph pair), with the regularisation steps
// it chains after each CG run: positivity (itk::ThresholdImageFilter,
// ThresholdBelow(0), outside value 0), total-variation denoising
// (rtk::TotalVariationDenoisingBPDQImageFilter) and soft thresholding of the
// image (rtk::SoftThresholdImageFilter); and rtk::TotalVariationImageFilter,
// the total-variation measure RTK's tests check the denoiser with.
//
// TV denoising by basis pursuit dequantisation
// (include/rtkDenoisingBPDQImageFilter.hxx:60-148), d processed dimensions:
//   beta = 0.9 minSpacing / 2^d   (minSpacing: the smallest spacing over the
//                                  processed dimensions and dimension 0)
//   z = P(grad(beta f))                            iteration 0
//   z = P(z - grad(beta minSpacing (f - div z)))   iterations 1..n-1
//   out = f - div z
// grad: forward differences, zero-flux Neumann boundary, spacing-scaled
// (rtk::ForwardDifferenceGradientImageFilter); div: backward differences, zero
// before the first voxel (rtk::BackwardDifferenceDivergenceImageFilter); P
// scales vectors longer than gamma back to gamma
// (rtk::MagnitudeThresholdImageFilter, in place: shorter ones unchanged).
// The divergence filter's AfterThreadedGenerateData subtracts z_k / s_k on the
// last slice along k (as coded, for one voxel of it); z_k is exactly zero
// there in this iteration (the forward difference vanishes on that slice, and
// P and z - grad keep it zero), so the divergence below, which drops z_k on
// that slice, gives the same values.
//
// Layout: the dual field z is one float plane per processed dimension (SoA,
// coalesced along x); each BPDQ iteration is two passes over the volume, the
// divergence/subtract/scale pass and the gradient/subtract/threshold pass,
// 48 bytes per voxel of HBM traffic.
#include "rtkb200.h"
#include "rtkb_internal.h"

#include <algorithm>
#include <cmath>
#include <vector>

namespace
{
using rtkb::fail;

struct TvDims
{
  int   nd;        // processed dimensions
  int   dk[3];     // their indices, packed
  float inv_s[3];  // 1 / spacing of each packed dimension
  int   n[3];      // volume size
};

dim3
row_grid(const rtkb_image_desc & v)
{
  return dim3((unsigned)((v.size[0] + 127) / 128), (unsigned)std::min(v.size[1], 65535),
              (unsigned)std::min(v.size[2], 65535));
}

#define FOR_EACH_ROW_VOXEL(n)                                                                                         \
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;                                                               \
  if (ix < n[0])                                                                                                      \
    for (int iz = blockIdx.z; iz < n[2]; iz += gridDim.z)                                                             \
      for (int iy = blockIdx.y; iy < n[1]; iy += gridDim.y)

__device__ __forceinline__ long long
stride_of(const TvDims & t, int k)
{
  return k == 0 ? 1LL : (k == 1 ? (long long)t.n[0] : (long long)t.n[0] * t.n[1]);
}

// z_j = P_gamma(z_j - grad_j w) (kSubtract) or P_gamma(grad_j w), with w read
// as scale * src (scale = beta in iteration 0, where src is f; 1 afterwards).
template <bool kSubtract>
__global__ void __launch_bounds__(128)
tv_gradient_kernel(const float * __restrict__ src, float scale, float * __restrict__ Z, TvDims t, float gamma)
{
  const long long nvox = (long long)t.n[0] * t.n[1] * t.n[2];
  FOR_EACH_ROW_VOXEL(t.n)
  {
    const long long i = ((long long)iz * t.n[1] + iy) * t.n[0] + ix;
    const int       c[3] = { ix, iy, iz };
    const float     w0 = src[i] * scale;
    float           v[3] = { 0.f, 0.f, 0.f };
    double          nn = 0.;
#pragma unroll
    for (int j = 0; j < 3; j++)
    {
      if (j >= t.nd)
        break;
      const int k = t.dk[j];
      const float g = c[k] < t.n[k] - 1 ? (src[i + stride_of(t, k)] * scale - w0) * t.inv_s[j] : 0.f;
      v[j] = kSubtract ? Z[j * nvox + i] - g : g;
      nn += (double)v[j] * v[j];
    }
    const double norm = sqrt(nn);
    const bool   clip = norm > (double)gamma;
#pragma unroll
    for (int j = 0; j < 3; j++)
    {
      if (j >= t.nd)
        break;
      Z[j * nvox + i] = clip ? gamma * v[j] / (float)norm : v[j];
    }
  }
}

// out = f - div z (kFinal) or scale (f - div z).  out may alias f.
template <bool kFinal>
__global__ void __launch_bounds__(128)
tv_divergence_kernel(const float * f, const float * __restrict__ Z, float * out, TvDims t, float scale)
{
  const long long nvox = (long long)t.n[0] * t.n[1] * t.n[2];
  FOR_EACH_ROW_VOXEL(t.n)
  {
    const long long i = ((long long)iz * t.n[1] + iy) * t.n[0] + ix;
    const int       c[3] = { ix, iy, iz };
    float           div = 0.f;
#pragma unroll
    for (int j = 0; j < 3; j++)
    {
      if (j >= t.nd)
        break;
      const int   k = t.dk[j];
      const float here = c[k] < t.n[k] - 1 ? Z[j * nvox + i] : 0.f;
      const float prev = c[k] > 0 ? Z[j * nvox + i - stride_of(t, k)] : 0.f;
      div += (here - prev) * t.inv_s[j];
    }
    const float u = f[i] - div;
    out[i] = kFinal ? u : u * scale;
  }
}

// x = max(x, 0) (ThresholdBelow(0), outside value 0) and / or
// x = sgn(x) max(|x| - t, 0)
__global__ void __launch_bounds__(256)
pointwise_kernel(float * __restrict__ x, long long n, bool positivity, bool soft, float t)
{
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
  {
    float v = x[i];
    if (positivity && v < 0.f)
      v = 0.f;
    if (soft)
    {
      const float a = fmaxf(fabsf(v) - t, 0.f);
      v = v > 0.f ? a : (v < 0.f ? -a : 0.f);
    }
    x[i] = v;
  }
}

// Per-block partial sums of the forward-difference gradient norms
// (TotalVariationImageFilter: float differences, float sum of squares, the
// square roots accumulated in double).
constexpr int kTvBlocks = 148 * 8;
__global__ void __launch_bounds__(256)
tv_measure_kernel(const float * __restrict__ x, int nx, int ny, int nz, float isx, float isy, float isz,
                  double * __restrict__ partial)
{
  const long long sxy = (long long)nx * ny, n = sxy * nz;
  double          acc = 0.;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
  {
    const int   ix = (int)(i % nx), iy = (int)((i / nx) % ny), iz = (int)(i / sxy);
    const float v = x[i];
    const float dx = ix < nx - 1 ? (x[i + 1] - v) * isx : 0.f;
    const float dy = iy < ny - 1 ? (x[i + nx] - v) * isy : 0.f;
    const float dz = iz < nz - 1 ? (x[i + sxy] - v) * isz : 0.f;
    acc += sqrt((double)(dx * dx + dy * dy + dz * dz));
  }
  __shared__ double red[256];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1)
  {
    if ((int)threadIdx.x < s)
      red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    partial[blockIdx.x] = red[0];
}

__global__ void
sum_partials_kernel(const double * __restrict__ partial, int n, double * __restrict__ out)
{
  if (threadIdx.x == 0 && blockIdx.x == 0)
  {
    double s = 0.;
    for (int b = 0; b < n; b++)
      s += partial[b];
    *out = s;
  }
}

unsigned
flat_grid(long long n)
{
  return (unsigned)std::min<long long>((n + 255) / 256, 148LL * 16);
}

bool
tv_dims(const rtkb_image_desc & v, const int * dims, TvDims & t, double & min_spacing)
{
  t.nd = 0;
  min_spacing = v.spacing[0];
  for (int d = 0; d < 3; d++)
  {
    t.n[d] = v.size[d];
    if (dims[d])
    {
      t.dk[t.nd] = d;
      t.inv_s[t.nd] = (float)(1. / v.spacing[d]);
      t.nd++;
      min_spacing = std::min(min_spacing, v.spacing[d]);
    }
  }
  return true;
}

// BPDQ TV denoising of f into out (out may equal f); Z: nd * nvox floats, w: nvox floats.
cudaError_t
tv_bpdq(const rtkb_image_desc & v, const float * f, float * out, double gamma, int niter, const int * dims, float * Z,
        float * w, cudaStream_t st)
{
  TvDims t;
  double minsp = 0.;
  tv_dims(v, dims, t, minsp);
  const long long nvox = (long long)v.size[0] * v.size[1] * v.size[2];
  const double    beta = 1. / std::pow(2., (double)t.nd) * 0.9 * minsp;
  const float     g = (float)gamma, b0 = (float)beta, b1 = (float)(beta * minsp);
  const dim3      grid = row_grid(v);
  if (t.nd == 0)
    return f == out ? cudaSuccess : cudaMemcpyAsync(out, f, (size_t)nvox * 4, cudaMemcpyDeviceToDevice, st);
  tv_gradient_kernel<false><<<grid, 128, 0, st>>>(f, b0, Z, t, g);
  for (int it = 1; it < niter; it++)
  {
    tv_divergence_kernel<false><<<grid, 128, 0, st>>>(f, Z, w, t, b1);
    tv_gradient_kernel<true><<<grid, 128, 0, st>>>(w, 1.f, Z, t, g);
  }
  tv_divergence_kernel<true><<<grid, 128, 0, st>>>(f, Z, out, t, 1.f);
  return cudaGetLastError();
}

size_t
up256(size_t b)
{
  return (b + 255) & ~size_t(255);
}
} // namespace

extern "C" int
rtkb_tv_denoising_bpdq(const rtkb_image_desc * vol, const float * d_in, float * d_out, double gamma, int niter,
                       const int dims_processed[3], void * stream)
{
  using namespace rtkb;
  std::string why;
  if (!vol || !d_in || !d_out)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  if (!desc_valid(vol, why))
    return fail(RTKB_ERR_INVALID_ARGUMENT, why);
  if (niter < 1 || !std::isfinite(gamma) || gamma < 0.)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "TV denoising needs niter >= 1 and a finite gamma >= 0");
  const int       all[3] = { 1, 1, 1 };
  const int *     dims = dims_processed ? dims_processed : all;
  const long long nvox = num_pixels(*vol);
  if (nvox == 0)
    return RTKB_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  void *       mem = nullptr;
  RTKB_CUDA_TRY(scratch_malloc(&mem, 4 * up256((size_t)nvox * 4), st));
  float *     Z = static_cast<float *>(mem);
  float *     w = reinterpret_cast<float *>(static_cast<char *>(mem) + 3 * up256((size_t)nvox * 4));
  cudaError_t e = tv_bpdq(*vol, d_in, d_out, gamma, niter, dims, Z, w, st);
  cudaError_t fe = scratch_free(mem, st);
  if (e != cudaSuccess)
    return cuda_fail(e, "TV denoising");
  return fe == cudaSuccess ? RTKB_OK : cuda_fail(fe, "cudaFreeAsync");
}

extern "C" int
rtkb_total_variation(const rtkb_image_desc * vol, const float * d_in, double * tv, void * stream)
{
  using namespace rtkb;
  std::string why;
  if (!vol || !d_in || !tv)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  if (!desc_valid(vol, why))
    return fail(RTKB_ERR_INVALID_ARGUMENT, why);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double *     d = nullptr;
  RTKB_CUDA_TRY(scratch_malloc(&d, sizeof(double) * (kTvBlocks + 1), st));
  tv_measure_kernel<<<kTvBlocks, 256, 0, st>>>(d_in, vol->size[0], vol->size[1], vol->size[2],
                                               (float)(1. / vol->spacing[0]), (float)(1. / vol->spacing[1]),
                                               (float)(1. / vol->spacing[2]), d);
  sum_partials_kernel<<<1, 32, 0, st>>>(d, kTvBlocks, d + kTvBlocks);
  cudaError_t e = cudaGetLastError();
  double      h = 0.;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&h, d + kTvBlocks, sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaError_t fe = scratch_free(d, st);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(st);
  if (e != cudaSuccess)
    return cuda_fail(e, "total variation");
  if (fe != cudaSuccess)
    return cuda_fail(fe, "cudaFreeAsync");
  *tv = h;
  return RTKB_OK;
}

extern "C" int
rtkb_regularized_cg(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                    const float * d_proj, const float * d_weights, float * d_x,
                    const rtkb_regularized_cg_params * prm, void * stream)
{
  using namespace rtkb;
  std::string why;
  if (!g || !vol || !proj || !d_proj || !d_x || !prm)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  if (!desc_valid(vol, why) || !desc_valid(proj, why))
    return fail(RTKB_ERR_INVALID_ARGUMENT, why);
  if (prm->main_loop_iterations < 0 || prm->cg_iterations < 0 ||
      (prm->tv && (prm->tv_iterations < 1 || !std::isfinite(prm->gamma_tv) || prm->gamma_tv < 0.)) ||
      (prm->soft_threshold_on_image && !(prm->soft_threshold >= 0.)))
    return fail(RTKB_ERR_INVALID_ARGUMENT, "invalid regularised CG parameters");
  const long long nvox = num_pixels(*vol);
  if (prm->main_loop_iterations == 0 || nvox == 0)
    return RTKB_OK;
  cudaStream_t   st = static_cast<cudaStream_t>(stream);
  rtkb_cg_params cp = {};
  cp.tikhonov = prm->tikhonov;
  cp.use_cuda_graph = 1;
  cp.storage = 0;
  cp.gamma = prm->gamma;
  rtkb_cg * plan = nullptr;
  int       rc = rtkb_cg_create(g, vol, proj, &cp, &plan);
  if (rc != RTKB_OK)
    return rc;
  const size_t vb = up256((size_t)nvox * 4);
  void *       mem = nullptr;
  cudaError_t  e = scratch_malloc(&mem, (prm->tv ? 5 : 1) * vb, st);
  if (e != cudaSuccess)
  {
    rtkb_cg_destroy(plan);
    return cuda_fail(e, "scratch allocation");
  }
  float *   b = static_cast<float *>(mem);
  float *   Z = prm->tv ? reinterpret_cast<float *>(static_cast<char *>(mem) + vb) : nullptr;
  float *   w = prm->tv ? reinterpret_cast<float *>(static_cast<char *>(mem) + 4 * vb) : nullptr;
  const int all[3] = { 1, 1, 1 };
  int       dims[3];
  for (int d = 0; d < 3; d++)
    dims[d] = prm->tv_dimensions ? prm->tv_dimensions[d] : all[d];
  // b = BP(W .* p) once: every CG run of the main loop solves the same normal equations
  rc = cg_rhs(plan, d_proj, d_weights, !prm->disable_displaced_detector, b, st);
  for (int m = 0; m < prm->main_loop_iterations && rc == RTKB_OK; m++)
  {
    rc = rtkb_cg_start_rhs(plan, b, d_x, stream);
    if (rc == RTKB_OK)
      rc = rtkb_cg_iterate(plan, prm->cg_iterations, stream);
    if (rc != RTKB_OK)
      break;
    if (prm->positivity)
    {
      pointwise_kernel<<<flat_grid(nvox), 256, 0, st>>>(d_x, nvox, true, false, 0.f);
      if ((e = cudaGetLastError()) != cudaSuccess)
        rc = cuda_fail(e, "positivity");
    }
    if (rc == RTKB_OK && prm->tv && (e = tv_bpdq(*vol, d_x, d_x, prm->gamma_tv, prm->tv_iterations, dims, Z, w, st)) !=
                                      cudaSuccess)
      rc = cuda_fail(e, "TV denoising");
    if (rc == RTKB_OK && prm->soft_threshold_on_image)
    {
      pointwise_kernel<<<flat_grid(nvox), 256, 0, st>>>(d_x, nvox, false, true, (float)prm->soft_threshold);
      if ((e = cudaGetLastError()) != cudaSuccess)
        rc = cuda_fail(e, "soft threshold");
    }
  }
  e = scratch_free(mem, st);
  if (rc == RTKB_OK && e != cudaSuccess)
    rc = cuda_fail(e, "cudaFreeAsync");
  if (rc == RTKB_OK && (e = cudaStreamSynchronize(st)) != cudaSuccess)
    rc = cuda_fail(e, "regularised CG");
  rtkb_cg_destroy(plan);
  return rc;
}

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
// coalesced along x), ping-ponged between two buffers.  Each BPDQ iteration
// after the first is ONE pass: a thread recomputes w = beta' (f - div z) at
// its voxel and at its forward neighbours from cached loads of f and z (the
// same float operations in the same order as a separate pass would do), so an
// iteration moves 28 bytes per voxel of HBM traffic (f and z in, z out).
// RTK's default, all three dimensions processed, has kernels of its own with
// the directions fixed at compile time and 32-bit offsets where the volume
// allows (the generic kernels spend most of their time on index arithmetic).
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

// coordinate and size along dimension k (selects: no local-memory arrays)
__device__ __forceinline__ int
coord_of(int x, int y, int z, int k)
{
  return k == 0 ? x : (k == 1 ? y : z);
}

__device__ __forceinline__ int
size_of(const TvDims & t, int k)
{
  return k == 0 ? t.n[0] : (k == 1 ? t.n[1] : t.n[2]);
}

// div z at voxel i: backward differences, zero before the first voxel, z_k
// dropped on the last slice along k.
__device__ __forceinline__ float
div_at(const float * __restrict__ Z, const TvDims & t, int x, int y, int z, long long i, long long nvox)
{
  float div = 0.f;
#pragma unroll
  for (int j = 0; j < 3; j++)
  {
    if (j >= t.nd)
      break;
    const int   k = t.dk[j], ck = coord_of(x, y, z, k);
    const float here = ck < size_of(t, k) - 1 ? Z[j * nvox + i] : 0.f;
    const float prev = ck > 0 ? Z[j * nvox + i - stride_of(t, k)] : 0.f;
    div += (here - prev) * t.inv_s[j];
  }
  return div;
}

// P_gamma: vectors longer than gamma scaled back to gamma
__device__ __forceinline__ void
clip3(float & a, float & b, float & c, float gamma)
{
  const float norm = sqrtf(a * a + b * b + c * c);
  if (norm > gamma)
  {
    a = gamma * a / norm;
    b = gamma * b / norm;
    c = gamma * c / norm;
  }
}

// Iteration 0 (generic dimensions): z = P_gamma(grad(beta f)).
__global__ void __launch_bounds__(128)
tv_first_kernel(const float * __restrict__ f, float beta, float * __restrict__ Z, TvDims t, float gamma)
{
  const long long nvox = (long long)t.n[0] * t.n[1] * t.n[2];
  FOR_EACH_ROW_VOXEL(t.n)
  {
    const long long i = ((long long)iz * t.n[1] + iy) * t.n[0] + ix;
    const float     w0 = f[i] * beta;
    float           v[3] = { 0.f, 0.f, 0.f };
#pragma unroll
    for (int j = 0; j < 3; j++)
    {
      if (j >= t.nd)
        break;
      const int k = t.dk[j];
      v[j] = coord_of(ix, iy, iz, k) < size_of(t, k) - 1 ? (f[i + stride_of(t, k)] * beta - w0) * t.inv_s[j] : 0.f;
    }
    clip3(v[0], v[1], v[2], gamma);
#pragma unroll
    for (int j = 0; j < 3; j++)
      if (j < t.nd)
        Z[j * nvox + i] = v[j];
  }
}

// Iterations 1..n-1 (generic dimensions), fused: Zout = P_gamma(Zin - grad w),
// w = beta1 (f - div Zin) evaluated at the voxel and at each forward neighbour.
__global__ void __launch_bounds__(128)
tv_iterate_kernel(const float * __restrict__ f, const float * __restrict__ Zin, float * __restrict__ Zout, TvDims t,
                  float beta1, float gamma)
{
  const long long nvox = (long long)t.n[0] * t.n[1] * t.n[2];
  FOR_EACH_ROW_VOXEL(t.n)
  {
    const long long i = ((long long)iz * t.n[1] + iy) * t.n[0] + ix;
    const float     w0 = (f[i] - div_at(Zin, t, ix, iy, iz, i, nvox)) * beta1;
    float           v[3] = { 0.f, 0.f, 0.f };
#pragma unroll
    for (int j = 0; j < 3; j++)
    {
      if (j >= t.nd)
        break;
      const int k = t.dk[j];
      float     g = 0.f;
      if (coord_of(ix, iy, iz, k) < size_of(t, k) - 1)
      {
        const long long i1 = i + stride_of(t, k);
        const float     w1 =
          (f[i1] - div_at(Zin, t, ix + (k == 0), iy + (k == 1), iz + (k == 2), i1, nvox)) * beta1;
        g = (w1 - w0) * t.inv_s[j];
      }
      v[j] = Zin[j * nvox + i] - g;
    }
    clip3(v[0], v[1], v[2], gamma);
#pragma unroll
    for (int j = 0; j < 3; j++)
      if (j < t.nd)
        Zout[j * nvox + i] = v[j];
  }
}

// out = f - div z (generic dimensions).  out may alias f.
__global__ void __launch_bounds__(128)
tv_final_kernel(const float * f, const float * __restrict__ Z, float * out, TvDims t)
{
  const long long nvox = (long long)t.n[0] * t.n[1] * t.n[2];
  FOR_EACH_ROW_VOXEL(t.n)
  {
    const long long i = ((long long)iz * t.n[1] + iy) * t.n[0] + ix;
    out[i] = f[i] - div_at(Z, t, ix, iy, iz, i, nvox);
  }
}

// ---- all three dimensions processed (RTK's default) ----
template <typename Off>
struct Vol3
{
  int   n[3];
  Off   sy, sz; // strides of y and z
  float isx, isy, isz;
};

template <typename Off>
__device__ __forceinline__ float
div3(const float * __restrict__ zx, const float * __restrict__ zy, const float * __restrict__ zz, const Vol3<Off> & v,
     int x, int y, int z, Off p)
{
  float r = ((x < v.n[0] - 1 ? zx[p] : 0.f) - (x > 0 ? zx[p - 1] : 0.f)) * v.isx;
  r += ((y < v.n[1] - 1 ? zy[p] : 0.f) - (y > 0 ? zy[p - v.sy] : 0.f)) * v.isy;
  r += ((z < v.n[2] - 1 ? zz[p] : 0.f) - (z > 0 ? zz[p - v.sz] : 0.f)) * v.isz;
  return r;
}

template <typename Off>
__global__ void __launch_bounds__(128)
tv3_first_kernel(const float * __restrict__ f, float beta, float * __restrict__ Z, Vol3<Off> v, float gamma)
{
  const Off nvox = v.sz * v.n[2];
  float *   zx = Z;
  float *   zy = Z + nvox;
  float *   zz = Z + 2 * nvox;
  FOR_EACH_ROW_VOXEL(v.n)
  {
    const Off   p = (Off)iz * v.sz + (Off)iy * v.sy + ix;
    const float w0 = f[p] * beta;
    float       a = ix < v.n[0] - 1 ? (f[p + 1] * beta - w0) * v.isx : 0.f;
    float       b = iy < v.n[1] - 1 ? (f[p + v.sy] * beta - w0) * v.isy : 0.f;
    float       c = iz < v.n[2] - 1 ? (f[p + v.sz] * beta - w0) * v.isz : 0.f;
    clip3(a, b, c, gamma);
    zx[p] = a;
    zy[p] = b;
    zz[p] = c;
  }
}

template <typename Off>
__global__ void __launch_bounds__(128)
tv3_iterate_kernel(const float * __restrict__ f, const float * __restrict__ Zin, float * __restrict__ Zout,
                   Vol3<Off> v, float beta1, float gamma)
{
  const Off     nvox = v.sz * v.n[2];
  const float * zx = Zin;
  const float * zy = Zin + nvox;
  const float * zz = Zin + 2 * nvox;
  FOR_EACH_ROW_VOXEL(v.n)
  {
    const Off   p = (Off)iz * v.sz + (Off)iy * v.sy + ix;
    const float w0 = (f[p] - div3(zx, zy, zz, v, ix, iy, iz, p)) * beta1;
    float       a = zx[p], b = zy[p], c = zz[p];
    if (ix < v.n[0] - 1)
      a -= ((f[p + 1] - div3(zx, zy, zz, v, ix + 1, iy, iz, p + 1)) * beta1 - w0) * v.isx;
    if (iy < v.n[1] - 1)
      b -= ((f[p + v.sy] - div3(zx, zy, zz, v, ix, iy + 1, iz, p + v.sy)) * beta1 - w0) * v.isy;
    if (iz < v.n[2] - 1)
      c -= ((f[p + v.sz] - div3(zx, zy, zz, v, ix, iy, iz + 1, p + v.sz)) * beta1 - w0) * v.isz;
    clip3(a, b, c, gamma);
    Zout[p] = a;
    Zout[nvox + p] = b;
    Zout[2 * nvox + p] = c;
  }
}

template <typename Off>
__global__ void __launch_bounds__(128)
tv3_final_kernel(const float * f, const float * __restrict__ Z, float * out, Vol3<Off> v)
{
  const Off     nvox = v.sz * v.n[2];
  const float * zx = Z;
  const float * zy = Z + nvox;
  const float * zz = Z + 2 * nvox;
  FOR_EACH_ROW_VOXEL(v.n)
  {
    const Off p = (Off)iz * v.sz + (Off)iy * v.sy + ix;
    out[p] = f[p] - div3(zx, zy, zz, v, ix, iy, iz, p);
  }
}

template <typename Off>
void
tv3_run(const rtkb_image_desc & vd, const TvDims & t, const float * f, float * out, int niter, float b0, float b1,
        float g, float * Z, dim3 grid, cudaStream_t st)
{
  Vol3<Off> v;
  for (int d = 0; d < 3; d++)
    v.n[d] = vd.size[d];
  v.sy = (Off)vd.size[0];
  v.sz = (Off)vd.size[0] * vd.size[1];
  v.isx = t.inv_s[0];
  v.isy = t.inv_s[1];
  v.isz = t.inv_s[2];
  const long long nvox = (long long)vd.size[0] * vd.size[1] * vd.size[2];
  float *         za = Z;
  float *         zb = Z + 3 * nvox;
  tv3_first_kernel<Off><<<grid, 128, 0, st>>>(f, b0, za, v, g);
  for (int it = 1; it < niter; it++)
  {
    tv3_iterate_kernel<Off><<<grid, 128, 0, st>>>(f, za, zb, v, b1, g);
    std::swap(za, zb);
  }
  tv3_final_kernel<Off><<<grid, 128, 0, st>>>(f, za, out, v);
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

void
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
}

// BPDQ TV denoising of f into out (out may equal f); Z: two buffers of three
// planes of nvox floats.
cudaError_t
tv_bpdq(const rtkb_image_desc & v, const float * f, float * out, double gamma, int niter, const int * dims, float * Z,
        cudaStream_t st)
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
  if (t.nd == 3)
  {
    if (nvox < (1LL << 31) - (1LL << 20))
      tv3_run<int>(v, t, f, out, niter, b0, b1, g, Z, grid, st);
    else
      tv3_run<long long>(v, t, f, out, niter, b0, b1, g, Z, grid, st);
    return cudaGetLastError();
  }
  float * za = Z;
  float * zb = Z + 3 * nvox;
  tv_first_kernel<<<grid, 128, 0, st>>>(f, b0, za, t, g);
  for (int it = 1; it < niter; it++)
  {
    tv_iterate_kernel<<<grid, 128, 0, st>>>(f, za, zb, t, b1, g);
    std::swap(za, zb);
  }
  tv_final_kernel<<<grid, 128, 0, st>>>(f, za, out, t);
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
  RTKB_TRACE();
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
  RTKB_CUDA_TRY(scratch_malloc(&mem, (size_t)6 * nvox * 4, st));
  cudaError_t e = tv_bpdq(*vol, d_in, d_out, gamma, niter, dims, static_cast<float *>(mem), st);
  cudaError_t fe = scratch_free(mem, st);
  if (e != cudaSuccess)
    return cuda_fail(e, "TV denoising");
  return fe == cudaSuccess ? RTKB_OK : cuda_fail(fe, "cudaFreeAsync");
}

extern "C" int
rtkb_total_variation(const rtkb_image_desc * vol, const float * d_in, double * tv, void * stream)
{
  RTKB_TRACE();
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
  RTKB_TRACE();
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
  cp.backprojector = 1; // BP_JOSEPH: the regularised CG runs on the Joseph pair
  rtkb_cg * plan = nullptr;
  int       rc = rtkb_cg_create(g, vol, proj, &cp, &plan);
  if (rc != RTKB_OK)
    return rc;
  if (prm->support_mask && (rc = rtkb_cg_set_support_mask(plan, prm->support_mask)) != RTKB_OK)
  {
    rtkb_cg_destroy(plan);
    return rc;
  }
  const size_t vb = up256((size_t)nvox * 4);
  void *       mem = nullptr;
  cudaError_t  e = scratch_malloc(&mem, vb + (prm->tv ? (size_t)6 * nvox * 4 : 0), st);
  if (e != cudaSuccess)
  {
    rtkb_cg_destroy(plan);
    return cuda_fail(e, "scratch allocation");
  }
  float *   b = static_cast<float *>(mem);
  float *   Z = prm->tv ? reinterpret_cast<float *>(static_cast<char *>(mem) + vb) : nullptr;
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
    if (rc == RTKB_OK)
      rc = rtkb_cg_finish(plan, stream); // the CG filter's output times the support mask
    if (rc != RTKB_OK)
      break;
    if (prm->positivity)
    {
      pointwise_kernel<<<flat_grid(nvox), 256, 0, st>>>(d_x, nvox, true, false, 0.f);
      if ((e = cudaGetLastError()) != cudaSuccess)
        rc = cuda_fail(e, "positivity");
    }
    if (rc == RTKB_OK && prm->tv && (e = tv_bpdq(*vol, d_x, d_x, prm->gamma_tv, prm->tv_iterations, dims, Z, st)) !=
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

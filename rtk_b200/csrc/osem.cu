// osem.cu -- rtk::OSEMConeBeamReconstructionFilter
// (include/rtkOSEMConeBeamReconstructionFilter.hxx) and
// rtk::DePierroRegularizationImageFilter
// (include/rtkDePierroRegularizationImageFilter.hxx) on the projector pair:
// the Joseph forward projector and the voxel-based (RTK's default) or Joseph
// back projector.
//
// For each subset S of the processing order (the order is drawn once, before
// the iterations):
//   r_s = p_s / FP_s(x)       (1 where |FP_s(x)| < 1e-5: DivideOrZeroOut, constant 1)
//   B   = sum_{s in S} BP_s(r_s)
//   N   = sum_{s in S} BP_s(1)            (kept per subset after the first
//                                          iteration when normalisation images are stored)
//   M   = B x
//   R   = (A + sqrt(A^2 + 8 beta 26 M)) / 2,  A = N - beta K(x)
//   x   = M / R               (0 where |R| < 1e-5: DivideOrZeroOut, constant 0)
// K is the 3x3x3 neighbourhood sum with weight 26 at the centre and 1 at the
// 26 neighbours, zero outside the volume (itk::ConstantBoundaryCondition);
// with beta = 0, R = N and the update is the classic ML-EM one, x B / N.
// The 1e-5 thresholds are ITK's itk::DivideOrZeroOutImageFilter default
// (ITK >= 5.1, the version RTK requires), which RTK's OSEM filter keeps.
//
// B200 layout: x only changes at the end of a subset, so the subset's
// projections are projected and back projected together.  The stack and its
// geometry entries are permuted once into processing order; every subset is
// then a contiguous sub-stack, one forward-projection call, one ratio kernel,
// one back-projection call and one fused De Pierro/update kernel.  This needs
// a projection direction that keeps the stack axis apart from the detector
// axes (block-diagonal, as RTK's stacks have), because the Joseph and voxel
// projectors take the stack index of a projection through the projection
// image's index-to-physical matrix; other directions run projection by
// projection on the original stack.
#include "rtkb200.h"
#include "rtkb_internal.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace
{
using rtkb::fail;

constexpr float kDivideThreshold = 1e-5f; // itk::Functor::DivideOrZeroOut's default threshold

unsigned
grid_for(long long n)
{
  return (unsigned)std::min<long long>((n + 255) / 256, 148LL * 16);
}

__global__ void __launch_bounds__(256)
ones_kernel(float * __restrict__ out, long long n)
{
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = 1.f;
}

// fp = p / fp, or 1 where |fp| < threshold
__global__ void __launch_bounds__(256)
osem_ratio_kernel(const float * __restrict__ p, float * __restrict__ fp, long long n)
{
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
  {
    const float d = fp[i];
    fp[i] = fabsf(d) < kDivideThreshold ? 1.f : p[i] / d;
  }
}

// De Pierro's regularisation factor R at voxel (ix, iy, iz), in the operation
// order of rtk::DePierroRegularizationImageFilter: the 27-tap neighbourhood
// inner product in double (itk::NeighborhoodOperatorImageFilter's real type
// for a float image), rounded to float, times beta; A = N - that; B = M times
// float(8 beta 26); R = (A + sqrt(A A + B)) / 2 in float.
template <bool kStencil>
__device__ __forceinline__ float
de_pierro_factor(const float * __restrict__ x, int ix, int iy, int iz, int nx, int ny, int nz, float n, float m,
                 float beta, float c2)
{
  float a = n;
  if (kStencil)
  {
    const long long sxy = (long long)nx * ny;
    double          s = 0.;
#pragma unroll
    for (int dz = -1; dz <= 1; dz++)
    {
      const int z = iz + dz;
      if (z < 0 || z >= nz)
        continue;
#pragma unroll
      for (int dy = -1; dy <= 1; dy++)
      {
        const int y = iy + dy;
        if (y < 0 || y >= ny)
          continue;
        const float * row = x + (long long)z * sxy + (long long)y * nx;
#pragma unroll
        for (int dx = -1; dx <= 1; dx++)
        {
          const int xx = ix + dx;
          if (xx < 0 || xx >= nx)
            continue;
          const double w = (dx == 0 && dy == 0 && dz == 0) ? 26. : 1.;
          s += w * (double)__ldg(row + xx);
        }
      }
    }
    a = n - (float)s * beta;
  }
  const float b = m * c2;
  return (a + sqrtf(a * a + b)) / 2.f;
}

// Voxel rows: threads along x, blocks over (x tiles, y, z), striding over y and
// z beyond the grid's limits.
#define FOR_EACH_VOXEL(nx, ny, nz)                                                                                    \
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;                                                               \
  if (ix < nx)                                                                                                        \
    for (int iz = blockIdx.z; iz < nz; iz += gridDim.z)                                                               \
      for (int iy = blockIdx.y; iy < ny; iy += gridDim.y)

dim3
voxel_grid(const rtkb_image_desc & v)
{
  return dim3((unsigned)((v.size[0] + 127) / 128), (unsigned)std::min(v.size[1], 65535),
              (unsigned)std::min(v.size[2], 65535));
}

// OSEM update without the neighbourhood term (beta = 0), in place:
// x = DivideOrZeroOut(B x, R), R = (N + sqrt(N N + 0)) / 2.
__global__ void __launch_bounds__(128)
osem_update_kernel(float * x, const float * __restrict__ B, const float * __restrict__ N, int nx, int ny, int nz,
                   float beta, float c2)
{
  FOR_EACH_VOXEL(nx, ny, nz)
  {
    const long long i = ((long long)iz * ny + iy) * nx + ix;
    const float     m = B[i] * x[i];
    const float     r = de_pierro_factor<false>(x, ix, iy, iz, nx, ny, nz, N[i], m, beta, c2);
    x[i] = fabsf(r) < kDivideThreshold ? 0.f : m / r;
  }
}

// OSEM update with the neighbourhood term, marching along z: a thread owns one
// (x, y) column over a chunk of slices and slides three 3x3 in-plane sums of x
// (slices z-1, z, z+1) through registers, so each slice's sum is loaded once
// and used three times.  K = (3x3x3 box sum) + 25 x_c, summed in double; a
// double sum of at most 27 floats whose magnitudes lie within 2^24 of one
// another is exact, so K equals the filter's raster-order double inner
// product, rounded to float, for such volumes.
__device__ __forceinline__ double
plane_sum3(const float * __restrict__ x, int ix, int iy, int z, int nx, int ny, int nz)
{
  if (z < 0 || z >= nz)
    return 0.;
  const float * slice = x + (long long)z * nx * ny;
  double        s = 0.;
#pragma unroll
  for (int dy = -1; dy <= 1; dy++)
  {
    const int y = iy + dy;
    if (y < 0 || y >= ny)
      continue;
    const float * row = slice + (long long)y * nx;
#pragma unroll
    for (int dx = -1; dx <= 1; dx++)
    {
      const int xx = ix + dx;
      if (xx >= 0 && xx < nx)
        s += (double)__ldg(row + xx);
    }
  }
  return s;
}

constexpr int kZChunk = 16;

__global__ void __launch_bounds__(128)
osem_update_stencil_kernel(const float * __restrict__ x, const float * __restrict__ B, const float * __restrict__ N,
                           float * __restrict__ x_out, int nx, int ny, int nz, float beta, float c2)
{
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  if (ix >= nx)
    return;
  const int z0 = blockIdx.z * kZChunk, z1 = min(nz, z0 + kZChunk);
  for (int iy = blockIdx.y; iy < ny; iy += gridDim.y)
  {
    double sm = plane_sum3(x, ix, iy, z0 - 1, nx, ny, nz), s0 = plane_sum3(x, ix, iy, z0, nx, ny, nz);
    for (int iz = z0; iz < z1; iz++)
    {
      const double    sp = plane_sum3(x, ix, iy, iz + 1, nx, ny, nz);
      const long long i = ((long long)iz * ny + iy) * nx + ix;
      const float     xc = x[i];
      const float     m = B[i] * xc;
      const double    k = sm + s0 + sp + 25. * (double)xc;
      const float     a = N[i] - (float)k * beta;
      const float     r = (a + sqrtf(a * a + m * c2)) / 2.f;
      x_out[i] = fabsf(r) < kDivideThreshold ? 0.f : m / r;
      sm = s0;
      s0 = sp;
    }
  }
}

// rtk::DePierroRegularizationImageFilter alone: out = R(x_k, update, norm);
// norm == nullptr stands for the default normalisation volume of ones.
template <bool kStencil>
__global__ void __launch_bounds__(128)
de_pierro_kernel(const float * __restrict__ xk, const float * upd, const float * norm, float * out, int nx, int ny,
                 int nz, float beta, float c2)
{
  FOR_EACH_VOXEL(nx, ny, nz)
  {
    const long long i = ((long long)iz * ny + iy) * nx + ix;
    out[i] = de_pierro_factor<kStencil>(xk, ix, iy, iz, nx, ny, nz, norm ? norm[i] : 1.f, upd[i], beta, c2);
  }
}

bool
block_diagonal(const double * d)
{
  return d[2] == 0. && d[5] == 0. && d[6] == 0. && d[7] == 0.;
}

size_t
up256(size_t b)
{
  return (b + 255) & ~size_t(255);
}

// One projection group of a subset: a contiguous range of a stack (its
// geometry, description and data).
struct Group
{
  const rtkb_geometry * g;
  rtkb_image_desc       d;
  const float *         meas; // measured projections of the group
  float *               work; // forward projections, then ratios
};
} // namespace

extern "C" int
rtkb_de_pierro_regularization(const rtkb_image_desc * vol, const float * d_xk, const float * d_update,
                              const float * d_norm, double beta, float * d_out, void * stream)
{
  RTKB_TRACE();
  using namespace rtkb;
  std::string why;
  if (!vol || !d_xk || !d_update || !d_out)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  if (!desc_valid(vol, why))
    return fail(RTKB_ERR_INVALID_ARGUMENT, why);
  if (!std::isfinite(beta))
    return fail(RTKB_ERR_INVALID_ARGUMENT, "beta must be finite");
  if (d_out == d_xk && beta != 0.)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "the output must not alias x_k (neighbourhood term)");
  cudaStream_t    st = static_cast<cudaStream_t>(stream);
  const long long n = num_pixels(*vol);
  if (n == 0)
    return RTKB_OK;
  const float fb = (float)beta, c2 = (float)(4. * 2. * beta * 26.);
  if (beta != 0.)
    de_pierro_kernel<true><<<voxel_grid(*vol), 128, 0, st>>>(d_xk, d_update, d_norm, d_out, vol->size[0],
                                                              vol->size[1], vol->size[2], fb, c2);
  else
    de_pierro_kernel<false><<<voxel_grid(*vol), 128, 0, st>>>(d_xk, d_update, d_norm, d_out, vol->size[0],
                                                               vol->size[1], vol->size[2], fb, c2);
  cudaError_t ce = cudaGetLastError();
  return ce == cudaSuccess ? RTKB_OK : cuda_fail(ce, "De Pierro regularisation");
}

extern "C" int
rtkb_osem(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj, const float * d_proj,
          float * d_x, const rtkb_osem_params * prm, void * stream)
{
  RTKB_TRACE();
  using namespace rtkb;
  std::string why;
  if (!g || !vol || !proj || !d_proj || !d_x || !prm)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  if (!desc_valid(vol, why) || !desc_valid(proj, why))
    return fail(RTKB_ERR_INVALID_ARGUMENT, why);
  const int np = proj->size[2];
  if (prm->niter < 0 || prm->projections_per_subset < 1 || !std::isfinite(prm->beta) ||
      (prm->backprojector != RTKB_OSEM_BP_VOXEL && prm->backprojector != RTKB_OSEM_BP_JOSEPH))
    return fail(RTKB_ERR_INVALID_ARGUMENT, "invalid OSEM parameters");
  if (proj->index[2] < 0 || (long long)proj->index[2] + np > (long long)g->g.p.size())
    return fail(RTKB_ERR_INVALID_ARGUMENT, "Mismatch between the number of projections and the geometry entries.");
  const long long per = (long long)proj->size[0] * proj->size[1], nvox = num_pixels(*vol);
  if (prm->niter == 0 || np == 0 || nvox == 0)
    return RTKB_OK;
  try
  {
    std::vector<int> order;
    if (prm->order)
    {
      order.assign(prm->order, prm->order + np);
      std::vector<char> seen(np, 0);
      for (int s : order)
      {
        if (s < 0 || s >= np || seen[s])
          return fail(RTKB_ERR_INVALID_ARGUMENT, "OSEM order must be a permutation of the stack's projections");
        seen[s] = 1;
      }
    }
    else
      seeded_order(np, prm->seed, order);

    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int    pps = std::min(prm->projections_per_subset, np);
    const int    nsub = (np + pps - 1) / pps;
    const bool   gathered = block_diagonal(proj->direction);
    const bool   stencil = prm->beta != 0.;
    const bool   store = prm->store_normalization != 0 && prm->niter > 1;
    const size_t vb = up256((size_t)nvox * 4), gb = up256((size_t)per * pps * 4);
    const size_t stack_b = gathered ? up256((size_t)per * np * 4) : 0;
    const size_t total = stack_b + 2 * gb + vb /*B*/ + (store ? 0 : vb) /*N*/ + (stencil ? vb : 0) /*x ping-pong*/;
    void *       mem = nullptr;
    RTKB_CUDA_TRY(rtkb::scratch_malloc(&mem, total, st));
    void * norms = nullptr;
    if (store)
    {
      cudaError_t ce = rtkb::scratch_malloc(&norms, vb * (size_t)nsub, st);
      if (ce != cudaSuccess)
      {
        cudaGetLastError();
        rtkb::scratch_free(mem, st);
        return fail(RTKB_ERR_OUT_OF_MEMORY, "no room for " + std::to_string(nsub) +
                                                " stored normalisation volumes; set store_normalization to 0");
      }
    }
    char *  m = static_cast<char *>(mem);
    float * stack = gathered ? reinterpret_cast<float *>(m) : nullptr;
    float * work = reinterpret_cast<float *>(m + stack_b);
    float * ones = reinterpret_cast<float *>(m + stack_b + gb);
    float * B = reinterpret_cast<float *>(m + stack_b + 2 * gb);
    float * Nscr = store ? nullptr : reinterpret_cast<float *>(m + stack_b + 2 * gb + vb);
    float * xalt = stencil ? reinterpret_cast<float *>(m + stack_b + 2 * gb + vb + (store ? 0 : vb)) : nullptr;

    int           rc = RTKB_OK;
    rtkb_geometry pg; // geometry entries in processing order
    auto          cuda_step = [&](cudaError_t ce, const char * what) {
      if (ce != cudaSuccess && rc == RTKB_OK)
        rc = cuda_fail(ce, what);
    };
    if (gathered)
    {
      pg.g.radius_cylindrical = g->g.radius_cylindrical;
      pg.g.p.reserve(np);
      for (int i = 0; i < np && rc == RTKB_OK; i++)
      {
        pg.g.p.push_back(g->g.p[proj->index[2] + order[i]]);
        cuda_step(cudaMemcpyAsync(stack + (size_t)i * per, d_proj + (size_t)order[i] * per, (size_t)per * 4,
                                  cudaMemcpyDeviceToDevice, st),
                  "cudaMemcpyAsync");
      }
    }
    if (rc == RTKB_OK)
    {
      ones_kernel<<<grid_for(per * pps), 256, 0, st>>>(ones, per * pps);
      cuda_step(cudaGetLastError(), "fill");
    }

    std::vector<Group> groups;
    auto               make_groups = [&](int first, int k) {
      groups.clear();
      if (gathered)
      {
        rtkb_image_desc d = *proj;
        d.index[2] = first;
        d.size[2] = k;
        groups.push_back({ &pg, d, stack + (size_t)first * per, work });
      }
      else
        for (int t = 0; t < k; t++)
        {
          const int       s = order[first + t];
          rtkb_image_desc d = *proj;
          d.index[2] = proj->index[2] + s;
          d.size[2] = 1;
          groups.push_back({ g, d, d_proj + (size_t)s * per, work + (size_t)t * per });
        }
    };
    auto backproject = [&](const Group & G, const float * src, float * acc) {
      return prm->backprojector == RTKB_OSEM_BP_JOSEPH
               ? rtkb_joseph_back_project(G.g, vol, &G.d, src, acc, acc, stream)
               : rtkb_voxel_backproject(G.g, vol, &G.d, src, acc, acc, stream);
    };

    float *     x = d_x;
    const float fb = (float)prm->beta, c2 = (float)(4. * 2. * prm->beta * 26.);
    for (int it = 0; it < prm->niter && rc == RTKB_OK; it++)
      for (int j = 0; j < nsub && rc == RTKB_OK; j++)
      {
        const int first = j * pps, k = std::min(pps, np - first);
        make_groups(first, k);
        cuda_step(cudaMemsetAsync(work, 0, (size_t)per * k * 4, st), "cudaMemsetAsync");
        for (const Group & G : groups)
        {
          if (rc == RTKB_OK)
            rc = rtkb_joseph_forward_project(G.g, vol, &G.d, x, G.work, G.work, stream);
          if (rc == RTKB_OK)
          {
            const long long n = per * G.d.size[2];
            osem_ratio_kernel<<<grid_for(n), 256, 0, st>>>(G.meas, G.work, n);
            cuda_step(cudaGetLastError(), "OSEM ratio");
          }
        }
        cuda_step(cudaMemsetAsync(B, 0, (size_t)nvox * 4, st), "cudaMemsetAsync");
        for (const Group & G : groups)
          if (rc == RTKB_OK)
            rc = backproject(G, G.work, B);
        float * N = store ? reinterpret_cast<float *>(static_cast<char *>(norms) + vb * (size_t)j) : Nscr;
        if (it == 0 || !store)
        {
          cuda_step(cudaMemsetAsync(N, 0, (size_t)nvox * 4, st), "cudaMemsetAsync");
          for (const Group & G : groups)
            if (rc == RTKB_OK)
              rc = backproject(G, ones, N);
        }
        if (rc != RTKB_OK)
          break;
        const int nx = vol->size[0], ny = vol->size[1], nz = vol->size[2];
        if (stencil)
        {
          float * xo = (x == d_x) ? xalt : d_x;
          const dim3 sg((unsigned)((nx + 127) / 128), (unsigned)std::min(ny, 65535),
                        (unsigned)((nz + kZChunk - 1) / kZChunk));
          osem_update_stencil_kernel<<<sg, 128, 0, st>>>(x, B, N, xo, nx, ny, nz, fb, c2);
          x = xo;
        }
        else
          osem_update_kernel<<<voxel_grid(*vol), 128, 0, st>>>(x, B, N, nx, ny, nz, fb, c2);
        cuda_step(cudaGetLastError(), "OSEM update");
      }
    if (rc == RTKB_OK && x != d_x)
      cuda_step(cudaMemcpyAsync(d_x, x, (size_t)nvox * 4, cudaMemcpyDeviceToDevice, st), "cudaMemcpyAsync");
    cudaError_t fe = rtkb::scratch_free(mem, st);
    if (norms)
    {
      cudaError_t fe2 = rtkb::scratch_free(norms, st);
      if (fe == cudaSuccess)
        fe = fe2;
    }
    if (rc == RTKB_OK && fe != cudaSuccess)
      rc = cuda_fail(fe, "cudaFreeAsync");
    return rc;
  }
  catch (...)
  {
    return fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

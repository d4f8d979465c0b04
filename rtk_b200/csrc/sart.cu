// sart.cu -- rtk::SARTConeBeamReconstructionFilter
// (include/rtkSARTConeBeamReconstructionFilter.hxx) on the projector pair:
// the Joseph forward projector, RTK's default for SART, and the voxel-based
// back projector, its default back projector.
//
// For each projection s of the processing order:
//   e = lambda (p_s - FP_s(x)) / raybox_s   (0 where raybox_s < threshold)
//   e weighted by the displaced-detector filter (no padding)
//   B += BP_s(e), N += BP_s(1)
// and after every `projections_per_subset` projections (and after the last
// one) x += B / N (0 where N < threshold), then x = max(x, 0) with
// positivity.  raybox_s is RayBoxIntersectionImageFilter's length (mm) of
// the source-to-pixel ray inside the box BoxShape::SetBoxFromImage(volume,
// false) spans: from the origin to origin + D (spacing x (size - 1)).  RTK
// draws the projection order with std::shuffle on a default-constructed
// std::default_random_engine, whose sequence the C++ standard leaves to
// the implementation; the order is an input here (or a seeded Fisher-Yates
// shuffle), so that the oracle can follow the same one.
#include "rtkb200.h"
#include "rtkb_internal.h"

#include <algorithm>
#include <cfloat>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

namespace
{
using rtkb::fail;

struct RayTab
{
  double m[12];  // projection index -> world (rows 0-2)
  double src[3];   // source position (world); parallel beam: pixel - source
  double parallel; // 1: parallel beam (the source moves with the pixel, RTK's parallel ray iterator)
};

struct Box
{
  double D[9];      // volume direction, row-major
  double mn[3], mx[3]; // box corners in the frame rotated by D^T, ordered
};

// BoxShape::IsIntersectedByRay (src/rtkBoxShape.cxx:47-97) along the
// normalised source-to-pixel direction, density 1
__global__ void __launch_bounds__(256)
ray_box_kernel(const RayTab * __restrict__ P, Box b, int nu, int nv, int pidx0, int pidx1, int pidx2, float * out)
{
  const int u = blockIdx.x * 32 + (threadIdx.x & 31), v = blockIdx.y * 8 + (threadIdx.x >> 5), s = blockIdx.z;
  if (u >= nu || v >= nv)
    return;
  const RayTab & q = P[s];
  const double   iu = u + pidx0, iv = v + pidx1, ik = s + pidx2;
  double         d[3], src[3];
#pragma unroll
  for (int a = 0; a < 3; a++)
  {
    const double pix = q.m[a * 4 + 0] * iu + q.m[a * 4 + 1] * iv + q.m[a * 4 + 2] * ik + q.m[a * 4 + 3];
    src[a] = q.parallel != 0. ? pix - q.src[a] : q.src[a];
    d[a] = pix - src[a];
  }
  const double len = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  double       inf = -DBL_MAX, sup = DBL_MAX;
  bool         hit = true;
#pragma unroll
  for (int a = 0; a < 3; a++)
  {
    const double org = b.D[0 * 3 + a] * src[0] + b.D[1 * 3 + a] * src[1] + b.D[2 * 3 + a] * src[2];
    const double dir = (b.D[0 * 3 + a] * d[0] + b.D[1 * 3 + a] * d[1] + b.D[2 * 3 + a] * d[2]) / len;
    if (!hit)
      continue;
    if (dir == 0. && (org < b.mn[a] || org > b.mx[a]))
    {
      hit = false;
      continue;
    }
    const double inv = 1. / dir;
    double       t1 = (b.mn[a] - org) * inv, t2 = (b.mx[a] - org) * inv;
    if (t1 > t2)
    {
      const double t = t1;
      t1 = t2;
      t2 = t;
    }
    inf = fmax(t1, inf);
    sup = fmin(t2, sup);
    if (inf > sup || sup < 0.)
      hit = false;
  }
  out[((long long)s * nv + v) * nu + u] = hit ? (float)(sup - inf) : 0.f;
}

// e = lambda (p - fp) / rb, or 0 where rb < threshold (DivideOrZeroOut)
__global__ void __launch_bounds__(256)
sart_error_kernel(const float * __restrict__ p, const float * __restrict__ fp, const float * __restrict__ rb,
                  float * __restrict__ e, long long n, float lambda, float threshold)
{
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
  {
    const float den = rb[i];
    e[i] = den < threshold ? 0.f : lambda * (p[i] - fp[i]) / den;
  }
}

// x += B / N (0 where N < threshold), then max(x, 0) with positivity
__global__ void __launch_bounds__(256)
sart_update_kernel(float * __restrict__ x, const float * __restrict__ B, const float * __restrict__ N, long long n,
                   float threshold, bool positivity)
{
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
  {
    float v = x[i] + (N[i] < threshold ? 0.f : B[i] / N[i]);
    if (positivity && v < 0.f)
      v = 0.f;
    x[i] = v;
  }
}

// ThresholdBelow(0) with outside value 0
__global__ void __launch_bounds__(256)
positivity_kernel(float * __restrict__ x, long long n)
{
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (x[i] < 0.f)
      x[i] = 0.f;
}

__global__ void __launch_bounds__(256)
fill_value_kernel(float * __restrict__ out, float v, long long n)
{
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = v;
}

unsigned
grid_of(long long n)
{
  return (unsigned)std::min<long long>((n + 255) / 256, 148LL * 16);
}


int
ray_box_lengths(const rtkb_geometry * g, const rtkb_image_desc & vol, const rtkb_image_desc & proj, float * d_out,
                cudaStream_t st, const double * corners = nullptr)
{
  using namespace rtkb;
  if (g->g.radius_cylindrical != 0.)
    return fail(RTKB_ERR_UNSUPPORTED, "ray-box lengths are computed for flat panels only");
  std::vector<RayTab> tab(proj.size[2]);
  double              pi2pp[16];
  index_to_physical(proj, pi2pp);
  for (int s = 0; s < proj.size[2]; s++)
  {
    double p2f[16], m[16], src[4];
    g->g.proj_coords_to_fixed(proj.index[2] + s, p2f);
    mat_mul(p2f, pi2pp, m, 4, 4, 4);
    g->g.source_position(proj.index[2] + s, src);
    std::memcpy(tab[s].m, m, 12 * sizeof(double));
    tab[s].src[0] = src[0];
    tab[s].src[1] = src[1];
    tab[s].src[2] = src[2];
    tab[s].parallel = g->g.parallel_source_to_pixel(proj.index[2] + s, tab[s].src) ? 1. : 0.;
  }
  Box b;
  if (corners)
  {
    // SetBoxMin / SetBoxMax: identity direction, the two corners ordered
    const double I[9] = { 1., 0., 0., 0., 1., 0., 0., 0., 1. };
    std::memcpy(b.D, I, sizeof(b.D));
    for (int a = 0; a < 3; a++)
    {
      b.mn[a] = std::min(corners[a], corners[3 + a]);
      b.mx[a] = std::max(corners[a], corners[3 + a]);
    }
  }
  const double * D = vol.direction;
  double       ext[3], bmin[3], bmax[3];
  if (!corners)
    std::memcpy(b.D, D, sizeof(b.D));
  for (int a = 0; a < 3; a++)
    ext[a] = vol.spacing[a] * (vol.size[a] - 1);
  for (int r = 0; r < 3; r++)
  {
    bmin[r] = vol.origin[r];
    bmax[r] = vol.origin[r] + D[3 * r + 0] * ext[0] + D[3 * r + 1] * ext[1] + D[3 * r + 2] * ext[2];
  }
  for (int a = 0; a < 3 && !corners; a++)
  {
    b.mn[a] = D[0 * 3 + a] * bmin[0] + D[1 * 3 + a] * bmin[1] + D[2 * 3 + a] * bmin[2];
    b.mx[a] = D[0 * 3 + a] * bmax[0] + D[1 * 3 + a] * bmax[1] + D[2 * 3 + a] * bmax[2];
    if (b.mn[a] > b.mx[a])
      std::swap(b.mn[a], b.mx[a]);
  }
  void * d_tab = nullptr;
  RTKB_CUDA_TRY(rtkb::scratch_malloc(&d_tab, tab.size() * sizeof(RayTab), st));
  cudaError_t e = cudaMemcpyAsync(d_tab, tab.data(), tab.size() * sizeof(RayTab), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
  {
    const dim3 grid((unsigned)((proj.size[0] + 31) / 32), (unsigned)((proj.size[1] + 7) / 8), (unsigned)proj.size[2]);
    ray_box_kernel<<<grid, 256, 0, st>>>(static_cast<const RayTab *>(d_tab), b, proj.size[0], proj.size[1],
                                         proj.index[0], proj.index[1], proj.index[2], d_out);
    e = cudaGetLastError();
  }
  int         rc = (e == cudaSuccess) ? RTKB_OK : cuda_fail(e, "ray-box lengths");
  cudaError_t fe = rtkb::scratch_free(d_tab, st);
  if (rc == RTKB_OK && fe != cudaSuccess)
    rc = cuda_fail(fe, "cudaFreeAsync");
  return rc;
}
} // namespace

namespace rtkb
{
// SplitMix64 (Steele, Lea and Flood 2014) driving a Fisher-Yates shuffle
void
seeded_order(int n, unsigned long long seed, std::vector<int> & order)
{
  order.resize(n);
  std::iota(order.begin(), order.end(), 0);
  uint64_t state = seed;
  auto     next = [&]() {
    uint64_t z = (state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  for (int i = n - 1; i > 0; i--)
  {
    const int j = (int)(next() % (uint64_t)(i + 1));
    std::swap(order[i], order[j]);
  }
}
} // namespace rtkb

extern "C" int
rtkb_ray_box_lengths(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj, float * d_out,
                     void * stream)
{
  RTKB_TRACE();
  using namespace rtkb;
  std::string why;
  if (!g || !vol || !proj || !d_out)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  if (!desc_valid(vol, why) || !desc_valid(proj, why))
    return fail(RTKB_ERR_INVALID_ARGUMENT, why);
  if (proj->index[2] < 0 || (long long)proj->index[2] + proj->size[2] > (long long)g->g.p.size())
    return fail(RTKB_ERR_INVALID_ARGUMENT, "Mismatch between the number of projections and the geometry entries.");
  if (proj->size[1] > 65535 * 8 || proj->size[2] > 65535)
    return fail(RTKB_ERR_UNSUPPORTED, "projection stack too large for one launch");
  try
  {
    return ray_box_lengths(g, *vol, *proj, d_out, static_cast<cudaStream_t>(stream));
  }
  catch (...)
  {
    return fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

extern "C" int
rtkb_sart(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj, const float * d_proj,
          float * d_x, const rtkb_sart_params * prm, void * stream)
{
  RTKB_TRACE();
  using namespace rtkb;
  std::string why;
  if (!g || !vol || !proj || !d_proj || !d_x || !prm)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  if (!desc_valid(vol, why) || !desc_valid(proj, why))
    return fail(RTKB_ERR_INVALID_ARGUMENT, why);
  const int np = proj->size[2];
  if (prm->niter < 0 || prm->projections_per_subset < 1 || !(prm->division_threshold >= 0.))
    return fail(RTKB_ERR_INVALID_ARGUMENT, "invalid SART parameters");
  if (proj->index[2] < 0 || (long long)proj->index[2] + np > (long long)g->g.p.size())
    return fail(RTKB_ERR_INVALID_ARGUMENT, "Mismatch between the number of projections and the geometry entries.");
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
          return fail(RTKB_ERR_INVALID_ARGUMENT, "SART order must be a permutation of the stack's projections");
        seen[s] = 1;
      }
    }
    else
      seeded_order(np, prm->seed, order);
    cudaStream_t    st = static_cast<cudaStream_t>(stream);
    const long long per = (long long)proj->size[0] * proj->size[1], nvox = num_pixels(*vol);
    const size_t    vb = ((size_t)nvox * 4 + 255) & ~size_t(255), pb = ((size_t)per * 4 + 255) & ~size_t(255);
    const size_t    rbb = ((size_t)per * np * 4 + 255) & ~size_t(255);
    void *          mem = nullptr;
    RTKB_CUDA_TRY(rtkb::scratch_malloc(&mem, 2 * vb + rbb + 4 * pb, st));
    char *  m = static_cast<char *>(mem);
    float * B = reinterpret_cast<float *>(m);
    float * N = reinterpret_cast<float *>(m + vb);
    float * rb = reinterpret_cast<float *>(m + 2 * vb);
    float * fp = reinterpret_cast<float *>(m + 2 * vb + rbb);
    float * e = reinterpret_cast<float *>(m + 2 * vb + rbb + pb);
    float * e2 = reinterpret_cast<float *>(m + 2 * vb + rbb + 2 * pb);
    float * ones = reinterpret_cast<float *>(m + 2 * vb + rbb + 3 * pb);
    int     rc = ray_box_lengths(g, *vol, *proj, rb, st);
    if (rc == RTKB_OK)
    {
      fill_value_kernel<<<grid_of(per), 256, 0, st>>>(ones, 1.f, per);
      cudaError_t ce = cudaGetLastError();
      if (ce != cudaSuccess)
        rc = cuda_fail(ce, "fill");
    }
    for (int it = 0; it < prm->niter && rc == RTKB_OK; it++)
    {
      int count = 0;
      for (int i = 0; i < np && rc == RTKB_OK; i++)
      {
        const int       s = order[i];
        rtkb_image_desc p1 = *proj;
        p1.size[2] = 1;
        p1.index[2] = proj->index[2] + s;
        cudaError_t ce = cudaMemsetAsync(fp, 0, (size_t)per * 4, st);
        if (ce != cudaSuccess)
        {
          rc = cuda_fail(ce, "cudaMemsetAsync");
          break;
        }
        rc = rtkb_joseph_forward_project(g, vol, &p1, d_x, fp, fp, stream);
        if (rc != RTKB_OK)
          break;
        sart_error_kernel<<<grid_of(per), 256, 0, st>>>(d_proj + (size_t)s * per, fp, rb + (size_t)s * per, e, per,
                                                        (float)prm->lambda, (float)prm->division_threshold);
        if ((ce = cudaGetLastError()) != cudaSuccess)
        {
          rc = cuda_fail(ce, "SART error");
          break;
        }
        const float * eb = e;
        if (!prm->disable_displaced_detector)
        {
          rc = rtkb_displaced_detector(g, &p1, 0, e, e2, stream);
          eb = e2;
          if (rc != RTKB_OK)
            break;
        }
        if (count == 0)
        {
          ce = cudaMemsetAsync(B, 0, 2 * vb, st); // B and N
          if (ce != cudaSuccess)
          {
            rc = cuda_fail(ce, "cudaMemsetAsync");
            break;
          }
        }
        rc = rtkb_voxel_backproject(g, vol, &p1, eb, B, B, stream);
        if (rc == RTKB_OK)
          rc = rtkb_voxel_backproject(g, vol, &p1, ones, N, N, stream);
        if (rc != RTKB_OK)
          break;
        if (++count == prm->projections_per_subset || i == np - 1)
        {
          sart_update_kernel<<<grid_of(nvox), 256, 0, st>>>(d_x, B, N, nvox, (float)prm->division_threshold,
                                                            prm->positivity != 0);
          if ((ce = cudaGetLastError()) != cudaSuccess)
            rc = cuda_fail(ce, "SART update");
          count = 0;
        }
      }
    }
    cudaError_t fe = rtkb::scratch_free(mem, st);
    if (rc == RTKB_OK && fe != cudaSuccess)
      rc = cuda_fail(fe, "cudaFreeAsync");
    return rc;
  }
  catch (...)
  {
    return fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

extern "C" int
rtkb_iterative_fdk(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                   const float * d_proj, float * d_x, const rtkb_iterative_fdk_params * prm, void * stream)
{
  RTKB_TRACE();
  // IterativeFDKConeBeamReconstructionFilter::GenerateData
  // (include/rtkIterativeFDKConeBeamReconstructionFilter.hxx:171-218):
  // x += FDK(p); then niter - 1 times x += FDK(lambda (p - JosephFP(x)) / raybox)
  // (DivideOrZeroOut below 1e-5, the box from the volume's origin to origin +
  // size x spacing), each result thresholded below 0 with positivity.  FDK is
  // the displaced-detector, Parker, weighting and ramp chain, then the FDK
  // back projector, adding to x.
  using namespace rtkb;
  std::string why;
  if (!g || !vol || !proj || !d_proj || !d_x || !prm)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  if (!desc_valid(vol, why) || !desc_valid(proj, why))
    return fail(RTKB_ERR_INVALID_ARGUMENT, why);
  if (prm->niter < 1 || !std::isfinite(prm->lambda))
    return fail(RTKB_ERR_INVALID_ARGUMENT, "invalid iterative FDK parameters");
  if (proj->index[2] < 0 || (long long)proj->index[2] + proj->size[2] > (long long)g->g.p.size())
    return fail(RTKB_ERR_INVALID_ARGUMENT, "Mismatch between the number of projections and the geometry entries.");
  try
  {
    cudaStream_t    st = static_cast<cudaStream_t>(stream);
    rtkb_image_desc cd = *proj; // the filtered stack (padded on the truncated side when the detector is displaced)
    int             rc = RTKB_OK;
    if (prm->fdk.displaced_detector)
    {
      int weighted = 0;
      rc = rtkb_displaced_detector_region(g, proj, prm->fdk.pad_on_truncated_side, &cd, &weighted);
      if (rc != RTKB_OK)
        return rc;
    }
    const long long n = num_pixels(*proj), nc = num_pixels(cd), nvox = num_pixels(*vol);
    const size_t    pb = ((size_t)n * 4 + 255) & ~size_t(255), cb = ((size_t)nc * 4 + 255) & ~size_t(255);
    void *          mem = nullptr;
    RTKB_CUDA_TRY(rtkb::scratch_malloc(&mem, 3 * pb + cb, st));
    char *  m = static_cast<char *>(mem);
    float * rb = reinterpret_cast<float *>(m);
    float * fp = reinterpret_cast<float *>(m + pb);
    float * e = reinterpret_cast<float *>(m + 2 * pb);
    float * c = reinterpret_cast<float *>(m + 3 * pb);
    double  corners[6];
    for (int a = 0; a < 3; a++)
    {
      corners[a] = vol->origin[a];
      corners[3 + a] = vol->origin[a] + vol->size[a] * vol->spacing[a];
    }
    auto fdk_add = [&](const float * stack) {
      rtkb_image_desc od{};
      int             r = rtkb_fdk_preprocess(g, proj, &prm->fdk, &od, stack, c, stream);
      if (r == RTKB_OK)
        r = rtkb_fdk_backproject(g, vol, &od, c, d_x, d_x, stream);
      if (r == RTKB_OK && prm->positivity)
      {
        positivity_kernel<<<grid_of(nvox), 256, 0, st>>>(d_x, nvox);
        const cudaError_t ce = cudaGetLastError();
        if (ce != cudaSuccess)
          r = cuda_fail(ce, "positivity");
      }
      return r;
    };
    if (prm->niter > 1)
      rc = ray_box_lengths(g, *vol, *proj, rb, st, corners);
    if (rc == RTKB_OK)
      rc = fdk_add(d_proj);
    for (int it = 1; it < prm->niter && rc == RTKB_OK; it++)
    {
      cudaError_t ce = cudaMemsetAsync(fp, 0, (size_t)n * 4, st);
      if (ce != cudaSuccess)
      {
        rc = cuda_fail(ce, "cudaMemsetAsync");
        break;
      }
      rc = rtkb_joseph_forward_project(g, vol, proj, d_x, fp, fp, stream);
      if (rc != RTKB_OK)
        break;
      sart_error_kernel<<<grid_of(n), 256, 0, st>>>(d_proj, fp, rb, e, n, (float)prm->lambda, 1e-5f);
      if ((ce = cudaGetLastError()) != cudaSuccess)
      {
        rc = cuda_fail(ce, "iterative FDK correction");
        break;
      }
      rc = fdk_add(e);
    }
    const cudaError_t fe = rtkb::scratch_free(mem, st);
    if (rc == RTKB_OK && fe != cudaSuccess)
      rc = cuda_fail(fe, "cudaFreeAsync");
    return rc;
  }
  catch (...)
  {
    return fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

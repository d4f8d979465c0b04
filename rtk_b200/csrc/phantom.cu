// phantom.cu -- analytic projections of ellipsoid phantoms on the GPU.
//
// rtk::ProjectGeometricPhantomImageFilter / RayEllipsoidIntersectionImageFilter
// semantics (include/rtkRayConvexIntersectionImageFilter.hxx:57-84,
// src/rtkQuadricShape.cxx:43-140): every pixel receives, for each ellipsoid,
// density x length of the source-to-pixel segment inside it.  Used to
// synthesise benchmark inputs of the sizes the configurations name; FP64
// throughout.
#include "rtkb_internal.h"

#include <cstring>

namespace
{

struct PixProj
{
  double m[12];  // projection index -> world (rows 0-2)
  double src[3];   // source position (world); parallel beam: pixel - source
  double parallel; // 1: parallel beam (the source moves with the pixel, RTK's parallel ray iterator)
};

struct Ell
{
  double c[3], inva[3], Rt[9], density; // centre, 1/semi-axes, rotation transposed (world -> local)
};

__global__ void __launch_bounds__(256)
project_ellipsoids_kernel(const PixProj * __restrict__ P, const Ell * __restrict__ E, int ne, int nu, int nv,
                          int pidx0, int pidx1, int pidx2, float * out)
{
  const int u = blockIdx.x * 32 + (threadIdx.x & 31), v = blockIdx.y * 8 + (threadIdx.x >> 5), s = blockIdx.z;
  if (u >= nu || v >= nv)
    return;
  const PixProj & q = P[s];
  const double    iu = u + pidx0, iv = v + pidx1, ik = s + pidx2;
  double          d[3], src[3];
#pragma unroll
  for (int a = 0; a < 3; a++)
  {
    const double pix = q.m[a * 4 + 0] * iu + q.m[a * 4 + 1] * iv + q.m[a * 4 + 2] * ik + q.m[a * 4 + 3];
    src[a] = q.parallel != 0. ? pix - q.src[a] : q.src[a];
    d[a] = pix - src[a];
  }
  const double len = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  double       acc = 0.;
  for (int e = 0; e < ne; e++)
  {
    const Ell & el = E[e];
    double      o[3], dd[3];
    const double rel[3] = { src[0] - el.c[0], src[1] - el.c[1], src[2] - el.c[2] };
#pragma unroll
    for (int a = 0; a < 3; a++)
    {
      o[a] = (el.Rt[a * 3 + 0] * rel[0] + el.Rt[a * 3 + 1] * rel[1] + el.Rt[a * 3 + 2] * rel[2]) * el.inva[a];
      dd[a] = (el.Rt[a * 3 + 0] * d[0] + el.Rt[a * 3 + 1] * d[1] + el.Rt[a * 3 + 2] * d[2]) * el.inva[a];
    }
    const double A = dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2];
    const double B = 2 * (o[0] * dd[0] + o[1] * dd[1] + o[2] * dd[2]);
    const double C = o[0] * o[0] + o[1] * o[1] + o[2] * o[2] - 1.;
    const double disc = B * B - 4 * A * C;
    if (disc <= 0.)
      continue;
    const double sq = sqrt(disc);
    const double t1 = fmax((-B - sq) / (2 * A), 0.), t2 = fmin((-B + sq) / (2 * A), 1.);
    if (t2 > t1)
      acc += el.density * (t2 - t1) * len;
  }
  out[((long long)s * nv + v) * nu + u] = (float)acc;
}

} // namespace

extern "C" int
rtkb_project_ellipsoids(const rtkb_geometry * g, const rtkb_image_desc * proj, int n_ellipsoids,
                        const double * ellipsoids, float * d_out, void * stream)
{
  RTKB_TRACE();
  using namespace rtkb;
  std::string why;
  if (!g || !d_out || n_ellipsoids < 0 || (n_ellipsoids > 0 && !ellipsoids))
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  if (!desc_valid(proj, why))
    return fail(RTKB_ERR_INVALID_ARGUMENT, why);
  if (proj->index[2] < 0 || (long long)proj->index[2] + proj->size[2] > (long long)g->g.p.size())
    return fail(RTKB_ERR_INVALID_ARGUMENT, "Mismatch between the number of projections and the geometry entries.");
  if (proj->size[1] > 65535 * 8 || proj->size[2] > 65535)
    return fail(RTKB_ERR_UNSUPPORTED, "projection stack too large for one launch");
  if (g->g.radius_cylindrical != 0.)
    return fail(RTKB_ERR_UNSUPPORTED, "the phantom projector models flat panels only");
  try
  {
    std::vector<PixProj> tab(proj->size[2]);
    double               pi2pp[16];
    index_to_physical(*proj, pi2pp);
    for (int s = 0; s < proj->size[2]; s++)
    {
      double p2f[16], m[16], src[4];
      g->g.proj_coords_to_fixed(proj->index[2] + s, p2f);
      mat_mul(p2f, pi2pp, m, 4, 4, 4);
      g->g.source_position(proj->index[2] + s, src);
      std::memcpy(tab[s].m, m, 12 * sizeof(double));
      tab[s].src[0] = src[0];
      tab[s].src[1] = src[1];
      tab[s].src[2] = src[2];
      tab[s].parallel = g->g.parallel_source_to_pixel(proj->index[2] + s, tab[s].src) ? 1. : 0.;
    }
    std::vector<Ell> ell(n_ellipsoids > 0 ? n_ellipsoids : 1);
    for (int e = 0; e < n_ellipsoids; e++)
    {
      const double * in = ellipsoids + 16 * e; // centre, semi-axes, R (local -> world), density
      for (int a = 0; a < 3; a++)
      {
        if (!(in[3 + a] > 0.))
          return fail(RTKB_ERR_INVALID_ARGUMENT, "ellipsoid semi-axes must be positive");
        ell[e].c[a] = in[a];
        ell[e].inva[a] = 1. / in[3 + a];
        for (int b = 0; b < 3; b++)
          ell[e].Rt[a * 3 + b] = in[6 + b * 3 + a];
      }
      ell[e].density = in[15];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t tb = (tab.size() * sizeof(PixProj) + 255) & ~size_t(255), eb = ell.size() * sizeof(Ell);
    void *       scratch = nullptr;
    RTKB_CUDA_TRY(rtkb::scratch_malloc(&scratch, tb + eb, st));
    PixProj *   d_tab = static_cast<PixProj *>(scratch);
    Ell *       d_ell = reinterpret_cast<Ell *>(static_cast<char *>(scratch) + tb);
    cudaError_t e = cudaMemcpyAsync(d_tab, tab.data(), tab.size() * sizeof(PixProj), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_ell, ell.data(), eb, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
    {
      const dim3 grid((unsigned)((proj->size[0] + 31) / 32), (unsigned)((proj->size[1] + 7) / 8),
                      (unsigned)proj->size[2]);
      project_ellipsoids_kernel<<<grid, 256, 0, st>>>(d_tab, d_ell, n_ellipsoids, proj->size[0], proj->size[1],
                                                      proj->index[0], proj->index[1], proj->index[2], d_out);
      e = cudaGetLastError();
    }
    int         rc = (e == cudaSuccess) ? RTKB_OK : cuda_fail(e, "project ellipsoids");
    cudaError_t fe = rtkb::scratch_free(scratch, st);
    if (rc == RTKB_OK && fe != cudaSuccess)
      rc = cuda_fail(fe, "cudaFreeAsync");
    return rc;
  }
  catch (...)
  {
    return fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

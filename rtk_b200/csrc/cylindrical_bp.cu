// cylindrical_bp.cu -- the voxel-based back projector for a cylindrical
// detector centred on the source
// (rtk::BackProjectionImageFilter::CylindricalDetectorCenteredOnSourceBackprojection,
// include/rtkBackProjectionImageFilter.hxx:283-345; the matrices of :551-595).
//
// Per voxel x and projection s:
//   (a, b, c) = Mag Src Rot I2P_vol x   (physical detector point before the
//                                        projection translation, homogeneous)
//   u = a / c, v = b / c
//   u' = R atan2(u, R), v' = v R / sqrt(R^2 + u^2)  (arc length on the cylinder)
//   (i, j) = P2I_proj ProjT (u', v', 1)  (continuous projection index)
// and, when i and j lie in [start - 0.5, end + 0.5) of the projection
// (itk::LinearInterpolateImageFunction::IsInsideBuffer), the clamp-to-edge
// bilinear value is added to the voxel.  The projections are taken in stack
// order and each one's value is added in float, as RTK adds a projection at a
// time.  RTK accepts this geometry only when R equals the source-to-detector
// distance of the first projection; so does this entry point.
//
// A plain FP64 kernel (one thread per voxel row element, the projections in a
// loop); this path is not tuned.
#include "rtkb200.h"
#include "rtkb_internal.h"

#include <algorithm>
#include <cstring>
#include <vector>

namespace
{
using rtkb::fail;

struct CylBp
{
  double A[12]; // volume index -> (a, b, c)
  double B[6];  // rows 0-1 of P2I_proj ProjT: (u', v', 1) -> buffer index
};

__device__ __forceinline__ double
itk_bilinear(const float * __restrict__ p, int nu, int nv, double ci, double cj)
{
  // itk::LinearInterpolateImageFunction (2-D): base index floor(.), clamped
  // to the start; a neighbour past the end keeps the base value
  int          i0 = (int)floor(ci), j0 = (int)floor(cj);
  i0 = i0 < 0 ? 0 : i0;
  j0 = j0 < 0 ? 0 : j0;
  const double di = ci - i0, dj = cj - j0;
  const int    i1 = (di > 0. && i0 + 1 < nu) ? i0 + 1 : i0;
  const int    j1 = (dj > 0. && j0 + 1 < nv) ? j0 + 1 : j0;
  const double v00 = p[(long long)j0 * nu + i0], v10 = p[(long long)j0 * nu + i1];
  const double v01 = p[(long long)j1 * nu + i0], v11 = p[(long long)j1 * nu + i1];
  const double x0 = di > 0. ? v00 + (v10 - v00) * di : v00;
  const double x1 = di > 0. ? v01 + (v11 - v01) * di : v01;
  return dj > 0. ? x0 + (x1 - x0) * dj : x0;
}

__global__ void __launch_bounds__(128)
cyl_bp_kernel(const CylBp * __restrict__ T, int np, const float * __restrict__ proj, int nu, int nv,
              const float * vin, float * vout, int nx, int ny, int nz, int vx0, int vy0, int vz0, double radius)
{
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  if (ix >= nx)
    return;
  const long long per = (long long)nu * nv;
  for (int iz = blockIdx.z; iz < nz; iz += gridDim.z)
    for (int iy = blockIdx.y; iy < ny; iy += gridDim.y)
    {
      const long long o = ((long long)iz * ny + iy) * nx + ix;
      const double    x = ix + vx0, y = iy + vy0, z = iz + vz0;
      float           acc = vin[o];
      for (int s = 0; s < np; s++)
      {
        const CylBp & t = T[s];
        const double  c = t.A[8] * x + t.A[9] * y + t.A[10] * z + t.A[11];
        const double  persp = 1. / c;
        const double  u = (t.A[0] * x + t.A[1] * y + t.A[2] * z + t.A[3]) * persp;
        const double  v = (t.A[4] * x + t.A[5] * y + t.A[6] * z + t.A[7]) * persp;
        const double  u2 = radius * atan2(u, radius);
        const double  v2 = v * radius / sqrt(radius * radius + u * u);
        const double  ci = t.B[0] * u2 + t.B[1] * v2 + t.B[2];
        const double  cj = t.B[3] * u2 + t.B[4] * v2 + t.B[5];
        if (ci >= -0.5 && ci < nu - 0.5 && cj >= -0.5 && cj < nv - 0.5)
          acc = acc + (float)itk_bilinear(proj + s * per, nu, nv, ci, cj);
      }
      vout[o] = acc;
    }
}
} // namespace

namespace rtkb
{
int
cylindrical_backproject(const rtkb_geometry * g, const rtkb_image_desc & vol, const rtkb_image_desc & proj,
                        const float * d_proj, const float * d_vin, float * d_vout, cudaStream_t st)
{
  const Geometry & G = g->g;
  if (G.p.empty() || G.radius_cylindrical != G.p[0].sdd)
    return fail(RTKB_ERR_INVALID_ARGUMENT,
                "Voxel-based back projector can currently handle a cylindrical detector only when it is centered on "
                "the source.");
  if (vol.size[1] > 65535 || vol.size[2] > 65535)
    return fail(RTKB_ERR_UNSUPPORTED, "volume too large for one launch");
  const int np = proj.size[2];
  try
  {
    std::vector<CylBp> tab(np > 0 ? np : 1);
    double             i2p[16], p2i[16];
    index_to_physical(vol, i2p);
    if (!physical_to_index(proj, p2i))
      return fail(RTKB_ERR_INVALID_ARGUMENT, "singular projection direction");
    for (int s = 0; s < np; s++)
    {
      const Geometry::Proj & q = G.p[proj.index[2] + s];
      double                 t1[12], t2[12];
      mat_mul(q.mag, q.srct, t1, 3, 4, 4);
      mat_mul(t1, q.rot, t2, 3, 4, 4);
      mat_mul(t2, i2p, tab[s].A, 3, 4, 4);
      // the stack's physical-to-index matrix, its in-plane part, times ProjT;
      // then absolute index -> buffer index
      const double m[9] = { p2i[0], p2i[1], p2i[3], p2i[4], p2i[5], p2i[7], 0., 0., 1. };
      double       b[9];
      mat_mul(m, q.projt, b, 3, 3, 3);
      b[2] -= proj.index[0];
      b[5] -= proj.index[1];
      std::memcpy(tab[s].B, b, 6 * sizeof(double));
    }
    const long long nvox = num_pixels(vol);
    if (np == 0)
      return d_vin == d_vout ? RTKB_OK
                             : (cudaMemcpyAsync(d_vout, d_vin, (size_t)nvox * 4, cudaMemcpyDeviceToDevice, st) ==
                                    cudaSuccess
                                  ? RTKB_OK
                                  : fail(RTKB_ERR_CUDA, "cudaMemcpyAsync"));
    void * d_tab = nullptr;
    RTKB_CUDA_TRY(scratch_malloc(&d_tab, tab.size() * sizeof(CylBp), st));
    cudaError_t e = cudaMemcpyAsync(d_tab, tab.data(), tab.size() * sizeof(CylBp), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
    {
      const dim3 grid((unsigned)((vol.size[0] + 127) / 128), (unsigned)vol.size[1], (unsigned)vol.size[2]);
      cyl_bp_kernel<<<grid, 128, 0, st>>>(static_cast<const CylBp *>(d_tab), np, d_proj, proj.size[0], proj.size[1],
                                          d_vin, d_vout, vol.size[0], vol.size[1], vol.size[2], vol.index[0],
                                          vol.index[1], vol.index[2], G.radius_cylindrical);
      e = cudaGetLastError();
    }
    const cudaError_t fe = scratch_free(d_tab, st);
    if (e != cudaSuccess)
      return cuda_fail(e, "cylindrical back projection");
    return fe == cudaSuccess ? RTKB_OK : cuda_fail(fe, "cudaFreeAsync");
  }
  catch (...)
  {
    return fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}
} // namespace rtkb

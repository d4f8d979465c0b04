// joseph.cu -- Joseph forward projector and its exact adjoint on sm_100a.
//
// Restates rtk::JosephForwardProjectionImageFilter::ThreadedGenerateData
// (include/rtkJosephForwardProjectionImageFilter.hxx:182-427) and
// rtk::JosephBackProjectionImageFilter::GenerateData
// (include/rtkJosephBackProjectionImageFilter.hxx:57-323); replaces the ray
// marchers behind CUDA_forward_project and CUDA_ray_cast_back_project, which
// use fixed-step trilinear texture sampling instead of Joseph's scheme.
//
// One thread per detector pixel.  Both projectors' grids run every
// projection of a band of detector rows (8 by default, tunable) before the
// next band (blockIdx.y = projection, blockIdx.z = row band): detector rows
// run along the volume's y
// axis, so the blocks in flight touch one y-slab of the volume, which stays
// in L2 across projections (the quad copies and quad accumulators are 4x the
// volume).  The ray set-up
// (pixel and source in volume index coordinates, main direction, box
// clipping, rint() slice bounds, residual weights) is FP64 exactly as RTK
// computes it; the two border steps
// are FP64 with RTK's clamped taps; the middle steps run in FP32 with
// positions x0 + i*step (no accumulated drift).  Rays whose main direction is
// x read (or scatter into) a z<->x transposed copy of the volume, so that
// neighbouring rays touch neighbouring addresses for every main direction.
#include "rtkb_elem.cuh"
#include "rtkb_joseph.h"
#include "rtkb_ptx.cuh"

#include <algorithm>
#include <cfloat>
#include <cstring>

namespace
{
using rtkb::JosephArgs;
using rtkb::ld_elem;
using rtkb::st_elem;
using rtkb::RayProj;
using rtkb::CylProj;

struct Ray
{
  int    main, dinf, dsup;
  int    ns, fs, dz;
  double resB, resE, len0; // first/last step lengths in voxels (len0: single-step rays)
  double stepx, stepy, curx, cury, norm;
};

// RTK's ray set-up; forward selects the forward projector's acceptance test.
__device__ __forceinline__ bool
setup_ray(const JosephArgs & a, const RayProj & P, int u, int v, int s, bool forward, Ray & r)
{
  const double iu = u + a.pidx0, iv = v + a.pidx1, ik = s + a.pidx2;
  double       pix[3], dir[3];
  if (a.C)
  {
    // ProjectionsRegionConstIteratorRayBasedWithCylindricalPanel::NewPixel: the
    // flat-panel u is an arc length on the cylinder; its angle gives
    // u' = R sin(u / R), w' = w + R (1 - cos(u / R))
    const CylProj & C = a.C[s];
    double          pos[3];
#pragma unroll
    for (int q = 0; q < 3; q++)
      pos[q] = C.idx2det[q * 4 + 0] * iu + C.idx2det[q * 4 + 1] * iv + C.idx2det[q * 4 + 2] * ik + C.idx2det[q * 4 + 3];
    const double ang = (1. / a.radius) * pos[0];
    pos[0] = sin(ang) * a.radius;
    pos[2] += (1. - cos(ang)) * a.radius;
#pragma unroll
    for (int q = 0; q < 3; q++)
      pix[q] = C.det2vol[q * 4 + 3] + C.det2vol[q * 4 + 0] * pos[0] + C.det2vol[q * 4 + 1] * pos[1] +
               C.det2vol[q * 4 + 2] * pos[2];
  }
  else
  {
#pragma unroll
    for (int q = 0; q < 3; q++)
      pix[q] = P.pix2vol[q * 4 + 0] * iu + P.pix2vol[q * 4 + 1] * iv + P.pix2vol[q * 4 + 2] * ik + P.pix2vol[q * 4 + 3];
  }
  // dirVox = -SourceToPixel; a parallel beam's source moves with the pixel
  const bool par = P.parallel != 0.;
#pragma unroll
  for (int q = 0; q < 3; q++)
    dir[q] = par ? -P.src[q] : -(pix[q] - P.src[q]);
  int mainDir = 0;
  if (fabs(dir[1]) > fabs(dir[mainDir]))
    mainDir = 1;
  if (fabs(dir[2]) > fabs(dir[mainDir]))
    mainDir = 2;
  // BoxShape::IsIntersectedByRay, src/rtkBoxShape.cxx:47-97
  double infd = -DBL_MAX, supd = DBL_MAX;
#pragma unroll
  for (int q = 0; q < 3; q++)
  {
    double mn = a.bmin[q], mx = a.bmax[q];
    if (mn > mx)
    {
      const double t = mn;
      mn = mx;
      mx = t;
    }
    if (dir[q] == 0. && (pix[q] < mn || pix[q] > mx))
      return false;
    const double inv = 1 / dir[q];
    double       t1 = (mn - pix[q]) * inv, t2 = (mx - pix[q]) * inv;
    if (t1 > t2)
    {
      const double t = t1;
      t1 = t2;
      t2 = t;
    }
    infd = fmax(t1, infd);
    supd = fmin(t2, supd);
    if (infd > supd)
      return false;
    if (supd < 0.)
      return false;
  }
  if (forward)
  {
    infd = fmax(infd, 0.);
    supd = fmin(supd, 1.);
    if (!(supd > 0. && infd <= 1. && supd > infd))
      return false;
  }
  else
  {
    if (!(supd >= 0. && infd <= 1.))
      return false;
    infd = fmax(infd, 0.);
    supd = fmin(supd, 1.);
  }
  double npt[3], fpt[3];
#pragma unroll
  for (int q = 0; q < 3; q++)
  {
    npt[q] = pix[q] + infd * dir[q];
    fpt[q] = pix[q] + supd * dir[q];
  }
  r.main = mainDir;
  r.ns = (int)rint(npt[mainDir]);
  r.fs = (int)rint(fpt[mainDir]);
  int di = (mainDir + 1) % 3, ds = (mainDir + 2) % 3;
  if (di > ds)
  {
    const int t = di;
    di = ds;
    ds = t;
  }
  r.dinf = di;
  r.dsup = ds;
  double       resB = r.ns - npt[mainDir], resE = fpt[mainDir] - r.fs;
  const double nrm = 1. / dir[mainDir];
  double       stepx = dir[di] * nrm, stepy = dir[ds] * nrm;
  r.dz = 1;
  if (npt[mainDir] > fpt[mainDir])
  {
    resB = -resB;
    resE = -resE;
    stepx = -stepx;
    stepy = -stepy;
    r.dz = -1;
  }
  r.resB = resB;
  r.resE = resE;
  r.len0 = fabs(fpt[mainDir] - npt[mainDir]);
  r.stepx = stepx;
  r.stepy = stepy;
  r.curx = npt[di] + resB * stepx;
  r.cury = npt[ds] + resB * stepy;
  const double mx = a.spacing[di] * stepx, my = a.spacing[ds] * stepy, mz = a.spacing[mainDir];
  r.norm = sqrt(mx * mx + my * my + mz * mz);
  return true;
}

// Memory view of the plane interpolation for a ray: base of slice 0 and
// strides, in the layout chosen for its main direction.
struct View
{
  long long ox, oy, oz; // element strides of the inf/sup in-plane axes and the slice axis
  int       nxp, nyp;   // in-plane sizes (inf, sup)
  int       nzp;        // size along the main direction
  int       bx, by, bz; // region index of the inf/sup/main axes
  bool      transposed;
};

__device__ __forceinline__ View
view_for(const JosephArgs & a, const Ray & r)
{
  View      w;
  const int nx = a.n[0], ny = a.n[1], nz = a.n[2];
  w.transposed = (r.main == 0);
  if (r.main == 0)
  {
    // transposed copy T[x][y][z]: y stride nz, z stride 1, x stride ny*nz
    w.ox = nz;
    w.oy = 1;
    w.oz = (long long)ny * nz;
  }
  else
  {
    const long long st[3] = { 1, nx, (long long)nx * ny };
    w.ox = st[r.dinf];
    w.oy = st[r.dsup];
    w.oz = st[r.main];
  }
  w.nxp = a.n[r.dinf];
  w.nyp = a.n[r.dsup];
  w.nzp = a.n[r.main];
  w.bx = a.vidx[r.dinf];
  w.by = a.vidx[r.dsup];
  w.bz = a.vidx[r.main];
  return w;
}

// Border step (BilinearInterpolationOnBorders / BilinearSplatOnBorders): FP64
// position, taps clamped as RTK offsets them.  Returns buffer offsets and
// weights of the four taps.
__device__ __forceinline__ void
border_taps(const JosephArgs & a, const Ray & r, const View & w, int sl, double x, double y, long long o[4],
            double wt[4])
{
  const int    ix = (int)floor(x), iy = (int)floor(y);
  const double lx = x - ix, ly = y - iy, lxc = 1. - lx, lyc = 1. - ly;
  const double minx = a.bmin[r.dinf], miny = a.bmin[r.dsup], maxx = a.bmax[r.dinf], maxy = a.bmax[r.dsup];
  int          xi = ix, xs = ix + 1, yi = iy, ys = iy + 1;
  if (ix < minx)
    xi = ix + 1;
  if (iy < miny)
    yi = iy + 1;
  if (ix >= maxx)
    xs = ix;
  if (iy >= maxy)
    ys = iy;
  // buffer coordinates, clamped for memory safety (a no-op inside the box)
  xi = min(max(xi - w.bx, 0), w.nxp - 1);
  xs = min(max(xs - w.bx, 0), w.nxp - 1);
  yi = min(max(yi - w.by, 0), w.nyp - 1);
  ys = min(max(ys - w.by, 0), w.nyp - 1);
  const long long zo = (long long)min(max(sl - w.bz, 0), w.nzp - 1) * w.oz;
  o[0] = zo + xi * w.ox + yi * w.oy;
  o[1] = zo + xs * w.ox + yi * w.oy;
  o[2] = zo + xi * w.ox + ys * w.oy;
  o[3] = zo + xs * w.ox + ys * w.oy;
  wt[0] = lxc * lyc;
  wt[1] = lx * lyc;
  wt[2] = lxc * ly;
  wt[3] = lx * ly;
}

// The middle steps of rays whose main direction is z (or x) read one float4
// "quad" per step instead of four scattered taps: Q[e] holds the 2 x 2
// in-plane neighbourhood (f(a,b), f(a,b+1), f(a+1,b), f(a+1,b+1)) of element
// e of the volume (or of its transposed copy), with a the first in-plane axis
// and b the second, neighbours clamped at the last index.  Q uses the volume's
// own element indexing, so a step's quad sits at the offset of its first tap.
// Rays whose main direction is y (beyond 45 degrees of cone angle) keep the
// four-tap loop.
//
// Offsets are 32-bit (Off = int) when the volume has fewer than 2^31 voxels.
// 64 registers give 4 CTAs per SM: the loop is bound by gather latency, and
// the FP64 ray state is dead before it starts (the last border step is taken
// first; the sums are still added in ray order).
template <typename Off, typename TP, bool kQuads>
__global__ void __launch_bounds__(256, 4)
joseph_forward_kernel(JosephArgs a, const float * __restrict__ V, const float * __restrict__ Vt,
                      const float4 * __restrict__ QN, const float4 * __restrict__ QT, const TP * pin, TP * pout,
                      const float * __restrict__ weights, int rb)
{
  const int nub = (a.nu + 31) / 32;
  const int u = (int)(blockIdx.x % nub) * 32 + (threadIdx.x & 31);
  const int v = ((int)blockIdx.z * rb + (int)(blockIdx.x / nub)) * 8 + (threadIdx.x >> 5);
  const int s = blockIdx.y;
  if (u >= a.nu || v >= a.nv)
    return;
  const long long po = ((long long)s * a.nv + v) * a.nu + u;
  Ray             r;
  if (!setup_ray(a, a.P[s], u, v, s, true, r))
  {
    const float base = pin ? ld_elem(pin, po) : 0.f;
    st_elem(pout, po, weights ? base * __ldg(weights + po) : base);
    return;
  }
  const View    w = view_for(a, r);
  const float * vol = w.transposed ? Vt : V;
  long long     o[4];
  double        wt[4];
  double        sum = 0.;
  if (r.fs == r.ns)
  {
    border_taps(a, r, w, r.ns, r.curx, r.cury, o, wt);
    sum = r.len0 * (wt[0] * __ldg(vol + o[0]) + wt[2] * __ldg(vol + o[2]) + wt[1] * __ldg(vol + o[1]) +
                    wt[3] * __ldg(vol + o[3]));
  }
  else
  {
    border_taps(a, r, w, r.ns, r.curx, r.cury, o, wt);
    sum = (r.resB + 0.5) * (wt[0] * __ldg(vol + o[0]) + wt[2] * __ldg(vol + o[2]) + wt[1] * __ldg(vol + o[1]) +
                            wt[3] * __ldg(vol + o[3]));
    const int nmid = abs(r.fs - r.ns) - 1;
    const int last = r.ns + r.dz * (nmid + 1);
    border_taps(a, r, w, last, r.curx + (nmid + 1) * r.stepx, r.cury + (nmid + 1) * r.stepy, o, wt);
    const double lastv = (r.resE + 0.5) * (wt[0] * __ldg(vol + o[0]) + wt[2] * __ldg(vol + o[2]) +
                                           wt[1] * __ldg(vol + o[1]) + wt[3] * __ldg(vol + o[3]));
    // middle steps: FP32 positions relative to the buffer origin
    const float2    x0 = make_float2((float)(r.curx + r.stepx - w.bx), (float)(r.cury + r.stepy - w.by));
    const float2    sxy = make_float2((float)r.stepx, (float)r.stepy);
    const int       xmax = max(w.nxp - 2, 0), ymax = max(w.nyp - 2, 0);
    const Off       ox = (Off)w.ox, oy = (Off)w.oy;
    const long long first = (long long)(r.ns + r.dz - w.bz) * w.oz, dslice = r.dz * w.oz;
    const float2    m1 = make_float2(-1.f, -1.f);
    float           acc = 0.f;
    if (kQuads && r.main != 1)
    {
      const float4 * slice = (w.transposed ? QT : QN) + first;
      // four steps' quad loads in flight per thread (measured: 2 or none
      // 21.1 ms, 4 20.1 ms, 8 23.6 ms on 256^3 <- 360 x 512x384)
#pragma unroll 4
      for (int i = 0; i < nmid; i++, slice += dslice)
      {
        const float2 xy = __ffma2_rn(make_float2((float)i, (float)i), sxy, x0);
        const int    ix = min(max((int)floorf(xy.x), 0), xmax), iy = min(max((int)floorf(xy.y), 0), ymax);
        const float2 l = __ffma2_rn(m1, make_float2((float)ix, (float)iy), xy);
        const float4 t = __ldg(slice + ((Off)ix * ox + (Off)iy * oy));
        // x-lerps of rows y and y + 1 together, then the y-lerp
        const float2 lo = make_float2(t.x, t.y), hi = make_float2(t.z, t.w);
        const float2 a01 = __ffma2_rn(make_float2(l.x, l.x), __ffma2_rn(m1, lo, hi), lo);
        acc += fmaf(l.y, a01.y - a01.x, a01.x);
      }
    }
    else
    {
      const Off     ox1 = (w.nxp > 1) ? ox : 0, oy1 = (w.nyp > 1) ? oy : 0;
      const float * slice = vol + first;
      // two steps' taps in flight per thread (one projection: 0.254 -> 0.242 ms at 256^3 <- 512x384)
#pragma unroll 2
      for (int i = 0; i < nmid; i++, slice += dslice)
      {
        const float2  xy = __ffma2_rn(make_float2((float)i, (float)i), sxy, x0);
        const int     ix = min(max((int)floorf(xy.x), 0), xmax), iy = min(max((int)floorf(xy.y), 0), ymax);
        const float2  l = __ffma2_rn(m1, make_float2((float)ix, (float)iy), xy);
        const float * q = slice + ((Off)ix * ox + (Off)iy * oy);
        const float2  lo = make_float2(__ldg(q), __ldg(q + oy1)), hi = make_float2(__ldg(q + ox1), __ldg(q + ox1 + oy1));
        const float2  a01 = __ffma2_rn(make_float2(l.x, l.x), __ffma2_rn(m1, lo, hi), lo);
        acc += fmaf(l.y, a01.y - a01.x, a01.x);
      }
    }
    sum += acc;
    sum += lastv;
  }
  const float base = pin ? ld_elem(pin, po) : 0.f;
  const float val = base + (float)(sum * r.norm);
  st_elem(pout, po, weights ? val * __ldg(weights + po) : val);
}

// Quads of a volume laid out [k][m][f] (f fastest): element e = (k m_n + m)
// f_n + f.  inf_fast: the first in-plane axis a is f (natural volume, a = x,
// b = y); else a is m and b is f (transposed copy T[x][y][z], a = y, b = z).
__global__ void __launch_bounds__(256)
quad_kernel(const float * __restrict__ src, float4 * __restrict__ dst, int fn, int mn, int outer, bool inf_fast)
{
  // threads along the fast axis f, blocks over rows m and planes o (striding
  // past the grid's limits): no per-element division
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= fn)
    return;
  const long long df = (f + 1 < fn) ? 1 : 0;
  for (int o = blockIdx.z; o < outer; o += gridDim.z)
    for (int m = blockIdx.y; m < mn; m += gridDim.y)
    {
      const long long e = ((long long)o * mn + m) * fn + f;
      const long long dm = (m + 1 < mn) ? fn : 0;
      const long long da = inf_fast ? df : dm, db = inf_fast ? dm : df;
      dst[e] = make_float4(__ldg(src + e), __ldg(src + e + db), __ldg(src + e + da), __ldg(src + e + da + db));
    }
}

__device__ __forceinline__ void
red_add(float * p, float v)
{
  asm volatile("red.global.add.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}

__device__ __forceinline__ void
red_add4(float4 * p, float4 v)
{
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w)
               : "memory");
}

// Back projector: the border steps splat into the scalar accumulators A (or
// At, transposed); the middle steps of main-z (main-x) rays add their four
// weights with one 16-byte vector reduction into the quad accumulator QAN
// (QAT), laid out as the forward projector's quad copies: element e collects
// the contributions to (f(a,b), f(a,b+1), f(a+1,b), f(a+1,b+1)) of the 2 x 2
// neighbourhood at e.  The fold kernel adds each voxel's four quad entries.
// Rays with main direction y keep four scalar reductions into A.  64
// registers (4 CTAs per SM) keep more reductions in flight.
template <typename Off, typename TP>
__global__ void __launch_bounds__(256, 4)
joseph_back_kernel(JosephArgs a, const TP * __restrict__ proj, float * A, float * At, float4 * QAN, float4 * QAT,
                   int rb)
{
  const int nub = (a.nu + 31) / 32;
  const int u = (int)(blockIdx.x % nub) * 32 + (threadIdx.x & 31);
  const int v = ((int)blockIdx.z * rb + (int)(blockIdx.x / nub)) * 8 + (threadIdx.x >> 5);
  const int s = blockIdx.y;
  if (u >= a.nu || v >= a.nv)
    return;
  const float val = ld_elem(proj, ((long long)s * a.nv + v) * a.nu + u);
  Ray         r;
  if (!setup_ray(a, a.P[s], u, v, s, false, r))
    return;
  const View   w = view_for(a, r);
  float *      vol = w.transposed ? At : A;
  const double c = (double)val * r.norm;
  long long    o[4];
  double       wt[4];
  if (r.fs == r.ns)
  {
    border_taps(a, r, w, r.ns, r.curx, r.cury, o, wt);
    const double f = c * r.len0;
#pragma unroll
    for (int q = 0; q < 4; q++)
      red_add(vol + o[q], (float)(f * wt[q]));
    return;
  }
  border_taps(a, r, w, r.ns, r.curx, r.cury, o, wt);
  double f = c * (r.resB + 0.5);
#pragma unroll
  for (int q = 0; q < 4; q++)
    red_add(vol + o[q], (float)(f * wt[q]));
  const int nmid = abs(r.fs - r.ns) - 1;
  // the last border step goes first, so the FP64 ray state is dead in the loop
  const int last = r.ns + r.dz * (nmid + 1);
  border_taps(a, r, w, last, r.curx + (nmid + 1) * r.stepx, r.cury + (nmid + 1) * r.stepy, o, wt);
  f = c * (r.resE + 0.5);
#pragma unroll
  for (int q = 0; q < 4; q++)
    red_add(vol + o[q], (float)(f * wt[q]));
  const float     x0 = (float)(r.curx + r.stepx - w.bx), y0 = (float)(r.cury + r.stepy - w.by);
  const float     sx = (float)r.stepx, sy = (float)r.stepy, cf = (float)c;
  const int       xmax = max(w.nxp - 2, 0), ymax = max(w.nyp - 2, 0);
  const Off       ox = (Off)w.ox, oy = (Off)w.oy;
  const long long first = (long long)(r.ns + r.dz - w.bz) * w.oz, dslice = r.dz * w.oz;
  if (r.main != 1)
  {
    // one-voxel in-plane axes: the "+1" neighbour is the voxel itself
    const bool ca = w.nxp == 1, cb = w.nyp == 1;
    float4 *   slice = (w.transposed ? QAT : QAN) + first;
    for (int i = 0; i < nmid; i++, slice += dslice)
    {
      const float x = fmaf((float)i, sx, x0), y = fmaf((float)i, sy, y0);
      const int   ix = min(max((int)floorf(x), 0), xmax), iy = min(max((int)floorf(y), 0), ymax);
      const float lx = x - ix, ly = y - iy;
      const float cy0 = cf * (1.f - ly), cy1 = cf * ly;
      float4      q = make_float4(cy0 * (1.f - lx), cy1 * (1.f - lx), cy0 * lx, cy1 * lx);
      if (ca)
        q = make_float4(q.x + q.z, q.y + q.w, 0.f, 0.f);
      if (cb)
        q = make_float4(q.x + q.y, 0.f, q.z + q.w, 0.f);
      float4 *       dst = slice + ((Off)ix * ox + (Off)iy * oy);
      // lanes 2k and 2k+1 (neighbouring pixels of one row) often hit the same
      // quad: the even lane then adds both, the odd lane sends nothing
      const unsigned act = __activemask();
      const int      lane = threadIdx.x & 31;
      const bool     pa = (act >> (lane ^ 1)) & 1u;
      const unsigned long long pk = __shfl_xor_sync(act, (unsigned long long)dst, 1);
      const float4   pq = make_float4(__shfl_xor_sync(act, q.x, 1), __shfl_xor_sync(act, q.y, 1),
                                      __shfl_xor_sync(act, q.z, 1), __shfl_xor_sync(act, q.w, 1));
      const bool     same = pa && pk == (unsigned long long)dst;
      if (same && (lane & 1))
        continue;
      if (same)
        q = make_float4(q.x + pq.x, q.y + pq.y, q.z + pq.z, q.w + pq.w);
      red_add4(dst, q);
    }
  }
  else
  {
    const Off ox1 = (w.nxp > 1) ? ox : 0, oy1 = (w.nyp > 1) ? oy : 0;
    float *   slice = vol + first;
    for (int i = 0; i < nmid; i++, slice += dslice)
    {
      const float x = fmaf((float)i, sx, x0), y = fmaf((float)i, sy, y0);
      const int   ix = min(max((int)floorf(x), 0), xmax), iy = min(max((int)floorf(y), 0), ymax);
      const float lx = x - ix, ly = y - iy;
      float *     q = slice + ((Off)ix * ox + (Off)iy * oy);
      const float cy0 = cf * (1.f - ly), cy1 = cf * ly;
      red_add(q, cy0 * (1.f - lx));
      red_add(q + ox1, cy0 * lx);
      red_add(q + oy1, cy1 * (1.f - lx));
      red_add(q + ox1 + oy1, cy1 * lx);
    }
  }
}

// T[x][y][z] = V[z][y][x] (32x32 shared-memory tiles in the x-z plane)
__global__ void __launch_bounds__(256)
transpose_zx_kernel(const float * __restrict__ V, float * __restrict__ T, int nx, int ny, int nz)
{
  __shared__ float tile[32][33];
  const int        y = blockIdx.y;
  const int        x0 = (blockIdx.x % ((nx + 31) / 32)) * 32, z0 = (blockIdx.x / ((nx + 31) / 32)) * 32;
  const int        tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int k = ty; k < 32; k += 8)
  {
    const int z = z0 + k, x = x0 + tx;
    if (z < nz && x < nx)
      tile[k][tx] = V[((long long)z * ny + y) * nx + x];
  }
  __syncthreads();
  for (int k = ty; k < 32; k += 8)
  {
    const int x = x0 + k, z = z0 + tx;
    if (x < nx && z < nz)
      T[((long long)x * ny + y) * nz + z] = tile[tx][k];
  }
}

// out[z][y][x] = in[z][y][x] + A[z][y][x] + At[x][y][z] (+ tau * x[z][y][x]);
// in and x may be null.
template <typename TV, typename TX>
__global__ void __launch_bounds__(256)
fold_transposed_kernel(const TV * in, const float * __restrict__ A, const float * __restrict__ At,
                       const float4 * __restrict__ QAN, const float4 * __restrict__ QAT, TV * out, int nx, int ny,
                       int nz, const TX * __restrict__ xv, float tau)
{
  __shared__ float tile[32][33];
  const int        y = blockIdx.y;
  const int        x0 = (blockIdx.x % ((nx + 31) / 32)) * 32, z0 = (blockIdx.x / ((nx + 31) / 32)) * 32;
  const int        tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int k = ty; k < 32; k += 8)
  {
    const int x = x0 + k, z = z0 + tx;
    if (x < nx && z < nz)
    {
      // transposed quads: a = y (stride nz), b = z (stride 1)
      const long long t = ((long long)x * ny + y) * nz + z;
      float           r = At[t] + QAT[t].x;
      if (z > 0)
        r += QAT[t - 1].y;
      if (y > 0)
      {
        r += QAT[t - nz].z;
        if (z > 0)
          r += QAT[t - nz - 1].w;
      }
      tile[k][tx] = r;
    }
  }
  __syncthreads();
  for (int k = ty; k < 32; k += 8)
  {
    const int z = z0 + k, x = x0 + tx;
    if (z < nz && x < nx)
    {
      // natural quads: a = x (stride 1), b = y (stride nx)
      const long long o = ((long long)z * ny + y) * nx + x;
      float           r = A[o] + QAN[o].x;
      if (y > 0)
        r += QAN[o - nx].y;
      if (x > 0)
      {
        r += QAN[o - 1].z;
        if (y > 0)
          r += QAN[o - nx - 1].w;
      }
      r += tile[tx][k];
      if (in)
        r += ld_elem(in, o);
      if (xv)
        r = fmaf(tau, ld_elem(xv, o), r);
      st_elem(out, o, r);
    }
  }
}

// Number of bilinear samples the forward projector takes per launch: one per
// main-direction slice between the rounded entry and exit slices (|fs-ns|+1),
// one for rays that enter and leave within one slice.
__global__ void __launch_bounds__(256)
joseph_count_kernel(JosephArgs a, unsigned long long * total)
{
  const int          u = blockIdx.x * 32 + (threadIdx.x & 31);
  const int          v = blockIdx.y * 8 + (threadIdx.x >> 5);
  const int          s = blockIdx.z;
  unsigned long long c = 0;
  Ray                r;
  if (u < a.nu && v < a.nv && setup_ray(a, a.P[s], u, v, s, true, r))
    c = (unsigned long long)(abs(r.fs - r.ns) + 1);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c)
    atomicAdd(total, c);
}

} // namespace

namespace rtkb
{

// Per-projection ray set-up tables (ProjectionsRegionConstIteratorRayBasedWithFlatPanel::NewProjection,
// include/rtkProjectionsRegionConstIteratorRayBasedWithFlatPanel.hxx:39-71).
int
joseph_tables(const Geometry & g, const rtkb_image_desc & vol, const rtkb_image_desc & proj, std::vector<RayProj> & out,
              std::vector<CylProj> * cyl)
{
  double vpp2i[16], pi2pp[16];
  if (!physical_to_index(vol, vpp2i))
    return fail(RTKB_ERR_INVALID_ARGUMENT, "singular volume direction");
  index_to_physical(proj, pi2pp);
  out.resize(proj.size[2]);
  for (int s = 0; s < proj.size[2]; s++)
  {
    const int k = proj.index[2] + s;
    double    p2f[16], t[16], m[16], s4[4], sv[4];
    g.proj_coords_to_fixed(k, p2f);
    mat_mul(vpp2i, p2f, t, 4, 4, 4);
    mat_mul(t, pi2pp, m, 4, 4, 4);
    g.source_position(k, s4);
    mat_mul(vpp2i, s4, sv, 4, 4, 1);
    RayProj & r = out[s];
    std::memcpy(r.pix2vol, m, 12 * sizeof(double));
    r.src[0] = sv[0];
    r.src[1] = sv[1];
    r.src[2] = sv[2];
    r.parallel = 0.;
    double s2p[3];
    if (g.parallel_source_to_pixel(k, s2p))
    {
      // ...Parallel::NewProjection maps SourceToPixel by the 3x3 part of the
      // volume's physical-to-index matrix
      for (int a = 0; a < 3; a++)
        r.src[a] = vpp2i[a * 4 + 0] * s2p[0] + vpp2i[a * 4 + 1] * s2p[1] + vpp2i[a * 4 + 2] * s2p[2];
      r.parallel = 1.;
    }
  }
  if (cyl)
  {
    cyl->clear();
    if (g.radius_cylindrical != 0.)
    {
      // ...WithCylindricalPanel::NewProjection: index -> detector system
      // (GetProjectionCoordinatesToDetectorSystemMatrix x the stack's
      // index-to-physical matrix), detector -> volume index (the volume's
      // physical-to-index matrix x the inverse rotation)
      cyl->resize(proj.size[2]);
      for (int s = 0; s < proj.size[2]; s++)
      {
        const int k = proj.index[2] + s;
        double    det[16], inv[16], i2d[16], d2v[16];
        g.proj_coords_to_detector(k, det);
        g.inverse_rotation(k, inv);
        mat_mul(det, pi2pp, i2d, 4, 4, 4);
        mat_mul(vpp2i, inv, d2v, 4, 4, 4);
        std::memcpy((*cyl)[s].idx2det, i2d, 12 * sizeof(double));
        std::memcpy((*cyl)[s].det2vol, d2v, 12 * sizeof(double));
      }
    }
  }
  return RTKB_OK;
}

size_t
joseph_table_bytes(const std::vector<RayProj> & tab, const std::vector<CylProj> & cyl)
{
  auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
  return up(tab.size() * sizeof(RayProj)) + up(cyl.size() * sizeof(CylProj));
}

cudaError_t
joseph_upload_tables(const std::vector<RayProj> & tab, const std::vector<CylProj> & cyl, double radius, void * d_mem,
                     JosephArgs & a, cudaStream_t st)
{
  const size_t tb = (tab.size() * sizeof(RayProj) + 255) & ~size_t(255);
  RayProj *    d_tab = static_cast<RayProj *>(d_mem);
  CylProj *    d_cyl = cyl.empty() ? nullptr : reinterpret_cast<CylProj *>(static_cast<char *>(d_mem) + tb);
  cudaError_t  e = cudaMemcpyAsync(d_tab, tab.data(), tab.size() * sizeof(RayProj), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && d_cyl)
    e = cudaMemcpyAsync(d_cyl, cyl.data(), cyl.size() * sizeof(CylProj), cudaMemcpyHostToDevice, st);
  a.P = d_tab;
  a.C = d_cyl;
  a.radius = d_cyl ? radius : 0.;
  return e;
}

void
joseph_args(JosephArgs & a, const rtkb_image_desc & vol, const rtkb_image_desc & proj, const RayProj * d_tab)
{
  a.P = d_tab;
  a.C = nullptr;
  a.radius = 0.;
  a.nu = proj.size[0];
  a.nv = proj.size[1];
  a.np = proj.size[2];
  a.pidx0 = proj.index[0];
  a.pidx1 = proj.index[1];
  a.pidx2 = proj.index[2];
  for (int q = 0; q < 3; q++)
  {
    a.n[q] = vol.size[q];
    a.vidx[q] = vol.index[q];
    a.spacing[q] = vol.spacing[q];
    a.bmin[q] = vol.index[q];
    a.bmax[q] = (double)(vol.index[q] + vol.size[q] - 1) * (1. - DBL_EPSILON);
  }
}

// Scratch of both projectors (one buffer serves both): two volume-sized
// float regions and two quad regions.  Forward: z<->x transposed copy, FP32
// copy of a BF16 volume, natural and transposed quad copies.  Back: natural
// and transposed scalar accumulators, natural and transposed quad
// accumulators.
size_t
joseph_forward_scratch_bytes(long long nvox)
{
  return 2 * (((size_t)nvox * sizeof(float) + 255) / 256 * 256) + 2 * (size_t)nvox * sizeof(float4);
}

size_t
joseph_back_scratch_bytes(long long nvox)
{
  return joseph_forward_scratch_bytes(nvox);
}

namespace
{
__global__ void __launch_bounds__(256)
widen_kernel(const __nv_bfloat16 * __restrict__ in, float * __restrict__ out, long long n)
{
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = __bfloat162float(in[i]);
}

// The quad copies cost two passes over 5x the volume's bytes: they pay off
// over a stack, not for one or two projections (SART's subsets), which take
// the four-tap loop directly.
constexpr int kQuadMinProjections = 4;

// Detector rows per band of the projectors' grids (rtkb_joseph_set_band_rows):
// [0] forward, [1] back; multiples of 8 (one CTA covers 32 x 8 pixels).
int g_joseph_band_rows[2] = { 8, 8 };

// Grid of one projector launch: x = the band's 32 x 8-pixel blocks (detector
// columns fastest), y = projection, z = band, so every projection of a band
// runs before the next band.
dim3
band_grid(const JosephArgs & a, int rb)
{
  const unsigned nub = (unsigned)((a.nu + 31) / 32);
  const unsigned nrb = (unsigned)((a.nv + 7) / 8);
  const unsigned rbu = (unsigned)std::max(1, std::min(rb, (int)nrb));
  return dim3(nub * rbu, (unsigned)a.np, (nrb + rbu - 1) / rbu);
}

template <typename TP>
cudaError_t
forward_launch(const JosephArgs & a, const float * V, float * Vt, float4 * QN, float4 * QT, const TP * pin, TP * pout,
               const float * w, cudaStream_t st)
{
  const int       nx = a.n[0], ny = a.n[1], nz = a.n[2];
  const long long nvox = (long long)nx * ny * nz;
  const bool      quads = a.np >= kQuadMinProjections;
  const dim3      tg((unsigned)(((nx + 31) / 32) * ((nz + 31) / 32)), (unsigned)ny);
  transpose_zx_kernel<<<tg, 256, 0, st>>>(V, Vt, nx, ny, nz);
  if (quads)
  {
    const dim3 qn((unsigned)((nx + 127) / 128), (unsigned)std::min(ny, 65535), (unsigned)std::min(nz, 65535));
    const dim3 qt((unsigned)((nz + 127) / 128), (unsigned)std::min(ny, 65535), (unsigned)std::min(nx, 65535));
    quad_kernel<<<qn, 128, 0, st>>>(V, QN, nx, ny, nz, true);  // a = x, b = y
    quad_kernel<<<qt, 128, 0, st>>>(Vt, QT, nz, ny, nx, false); // a = y, b = z
  }
  const int  rb = g_joseph_band_rows[0] / 8;
  const dim3 grid(band_grid(a, rb));
  const bool small = nvox < (1ll << 31);
  if (quads && small)
    joseph_forward_kernel<int, TP, true><<<grid, 256, 0, st>>>(a, V, Vt, QN, QT, pin, pout, w, rb);
  else if (quads)
    joseph_forward_kernel<long long, TP, true><<<grid, 256, 0, st>>>(a, V, Vt, QN, QT, pin, pout, w, rb);
  else if (small)
    joseph_forward_kernel<int, TP, false><<<grid, 256, 0, st>>>(a, V, Vt, QN, QT, pin, pout, w, rb);
  else
    joseph_forward_kernel<long long, TP, false><<<grid, 256, 0, st>>>(a, V, Vt, QN, QT, pin, pout, w, rb);
  return cudaGetLastError();
}

template <typename TP, typename TV, typename TX>
cudaError_t
back_launch(const JosephArgs & a, const TP * proj, void * scratch, const TV * vin, TV * vout, const TX * x, float tau,
            cudaStream_t st)
{
  const int       nx = a.n[0], ny = a.n[1], nz = a.n[2];
  const long long nvox = (long long)nx * ny * nz;
  const size_t    vb = ((size_t)nvox * sizeof(float) + 255) / 256 * 256;
  char *          m = static_cast<char *>(scratch);
  float *         A = reinterpret_cast<float *>(m);
  float *         At = reinterpret_cast<float *>(m + vb);
  float4 *        QAN = reinterpret_cast<float4 *>(m + 2 * vb);
  float4 *        QAT = QAN + nvox;
  cudaError_t     e = cudaMemsetAsync(scratch, 0, joseph_back_scratch_bytes(nvox), st);
  if (e != cudaSuccess)
    return e;
  const int  rb = g_joseph_band_rows[1] / 8;
  const dim3 grid(band_grid(a, rb));
  if (nvox < (1ll << 31))
    joseph_back_kernel<int, TP><<<grid, 256, 0, st>>>(a, proj, A, At, QAN, QAT, rb);
  else
    joseph_back_kernel<long long, TP><<<grid, 256, 0, st>>>(a, proj, A, At, QAN, QAT, rb);
  const dim3 tg((unsigned)(((nx + 31) / 32) * ((nz + 31) / 32)), (unsigned)ny);
  fold_transposed_kernel<TV, TX><<<tg, 256, 0, st>>>(vin, A, At, QAN, QAT, vout, nx, ny, nz, x, tau);
  return cudaGetLastError();
}
} // namespace

cudaError_t
joseph_forward_launch(const JosephArgs & a, const void * V, Elem ve, void * scratch, const void * pin, void * pout,
                      Elem pe, const float * w, cudaStream_t st)
{
  const long long nvox = (long long)a.n[0] * a.n[1] * a.n[2];
  const size_t    vb = ((size_t)nvox * sizeof(float) + 255) / 256 * 256;
  char *          m = static_cast<char *>(scratch);
  float *         Vt = reinterpret_cast<float *>(m);
  float4 *        QN = reinterpret_cast<float4 *>(m + 2 * vb);
  float4 *        QT = QN + nvox;
  const float *   V32 = static_cast<const float *>(V);
  if (ve == Elem::BF16)
  {
    float * w32 = reinterpret_cast<float *>(m + vb);
    widen_kernel<<<(unsigned)std::min<long long>((nvox + 255) / 256, 148LL * 32), 256, 0, st>>>(
      static_cast<const __nv_bfloat16 *>(V), w32, nvox);
    V32 = w32;
  }
  if (pe == Elem::BF16)
    return forward_launch(a, V32, Vt, QN, QT, static_cast<const __nv_bfloat16 *>(pin),
                          static_cast<__nv_bfloat16 *>(pout), w, st);
  return forward_launch(a, V32, Vt, QN, QT, static_cast<const float *>(pin), static_cast<float *>(pout), w, st);
}

namespace
{
template <typename TP, typename TV>
cudaError_t
back_x(const JosephArgs & a, const TP * proj, void * scratch, const void * vin, void * vout, const void * x, Elem xe,
       float tau, cudaStream_t st)
{
  const TV * vi = static_cast<const TV *>(vin);
  TV *       vo = static_cast<TV *>(vout);
  if (xe == Elem::BF16)
    return back_launch(a, proj, scratch, vi, vo, static_cast<const __nv_bfloat16 *>(x), tau, st);
  return back_launch(a, proj, scratch, vi, vo, static_cast<const float *>(x), tau, st);
}

template <typename TP>
cudaError_t
back_v(const JosephArgs & a, const void * proj, void * scratch, const void * vin, void * vout, Elem ve, const void * x,
       Elem xe, float tau, cudaStream_t st)
{
  const TP * p = static_cast<const TP *>(proj);
  if (ve == Elem::BF16)
    return back_x<TP, __nv_bfloat16>(a, p, scratch, vin, vout, x, xe, tau, st);
  return back_x<TP, float>(a, p, scratch, vin, vout, x, xe, tau, st);
}
} // namespace

cudaError_t
joseph_back_launch(const JosephArgs & a, const void * proj, Elem pe, void * scratch, const void * vin, void * vout,
                   Elem ve, const void * x, Elem xe, float tau, cudaStream_t st)
{
  if (pe == Elem::BF16)
    return back_v<__nv_bfloat16>(a, proj, scratch, vin, vout, ve, x, xe, tau, st);
  return back_v<float>(a, proj, scratch, vin, vout, ve, x, xe, tau, st);
}

int
joseph_check(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj)
{
  std::string why;
  if (!g)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "Geometry has not been set.");
  if (!desc_valid(vol, why) || !desc_valid(proj, why))
    return fail(RTKB_ERR_INVALID_ARGUMENT, why);
  if (proj->index[2] < 0 || (long long)proj->index[2] + proj->size[2] > (long long)g->g.p.size())
    return fail(RTKB_ERR_INVALID_ARGUMENT, "Mismatch between the number of projections and the geometry entries.");
  if (proj->size[1] > 65535 * 8 || proj->size[2] > 65535 || vol->size[1] > 65535)
    return fail(RTKB_ERR_UNSUPPORTED, "image too large for one launch");
  // ProjectionsRegionConstIteratorRayBased::New (include/rtkProjectionsRegionConstIteratorRayBased.hxx:90-95)
  if (!g->g.p.empty() && g->g.p[0].sdd == 0. && g->g.radius_cylindrical != 0.)
    return fail(RTKB_ERR_UNSUPPORTED, "Parallel geometry assumes a flat panel detector.");
  return RTKB_OK;
}

} // namespace rtkb

extern "C" int
rtkb_joseph_forward_project(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                            const float * d_vol, const float * d_proj_in, float * d_proj_out, void * stream)
{
  RTKB_TRACE();
  using namespace rtkb;
  try
  {
    int rc = joseph_check(g, vol, proj);
    if (rc != RTKB_OK)
      return rc;
    if (!d_vol || !d_proj_in || !d_proj_out)
      return fail(RTKB_ERR_INVALID_ARGUMENT, "null buffer");
    std::vector<RayProj> tab;
    std::vector<CylProj> cyl;
    rc = joseph_tables(g->g, *vol, *proj, tab, &cyl);
    if (rc != RTKB_OK)
      return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t tbytes = joseph_table_bytes(tab, cyl);
    void *       scratch = nullptr;
    RTKB_CUDA_TRY(rtkb::scratch_malloc(&scratch, tbytes + joseph_forward_scratch_bytes(num_pixels(*vol)), st));
    void *     d_vt = static_cast<char *>(scratch) + tbytes;
    JosephArgs a;
    joseph_args(a, *vol, *proj, nullptr);
    cudaError_t e = joseph_upload_tables(tab, cyl, g->g.radius_cylindrical, scratch, a, st);
    if (e == cudaSuccess)
      e = joseph_forward_launch(a, d_vol, d_vt, d_proj_in, d_proj_out, nullptr, st);
    rc = (e == cudaSuccess) ? RTKB_OK : cuda_fail(e, "joseph forward");
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

extern "C" int
rtkb_joseph_back_project(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                         const float * d_proj, const float * d_vol_in, float * d_vol_out, void * stream)
{
  RTKB_TRACE();
  using namespace rtkb;
  try
  {
    int rc = joseph_check(g, vol, proj);
    if (rc != RTKB_OK)
      return rc;
    if (!d_proj || !d_vol_in || !d_vol_out)
      return fail(RTKB_ERR_INVALID_ARGUMENT, "null buffer");
    std::vector<RayProj> tab;
    std::vector<CylProj> cyl;
    rc = joseph_tables(g->g, *vol, *proj, tab, &cyl);
    if (rc != RTKB_OK)
      return rc;
    cudaStream_t    st = static_cast<cudaStream_t>(stream);
    const long long nvox = num_pixels(*vol);
    const size_t    tbytes = joseph_table_bytes(tab, cyl);
    void *          scratch = nullptr;
    RTKB_CUDA_TRY(rtkb::scratch_malloc(&scratch, tbytes + joseph_back_scratch_bytes(nvox), st));
    void *     d_a = static_cast<char *>(scratch) + tbytes;
    JosephArgs a;
    joseph_args(a, *vol, *proj, nullptr);
    cudaError_t e = joseph_upload_tables(tab, cyl, g->g.radius_cylindrical, scratch, a, st);
    if (e == cudaSuccess)
      e = joseph_back_launch(a, d_proj, d_a, d_vol_in, d_vol_out, nullptr, 0.f, st);
    rc = (e == cudaSuccess) ? RTKB_OK : cuda_fail(e, "joseph back projection");
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

extern "C" int
rtkb_joseph_sample_count(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                         double * count, void * stream)
{
  RTKB_TRACE();
  using namespace rtkb;
  try
  {
    int rc = joseph_check(g, vol, proj);
    if (rc != RTKB_OK)
      return rc;
    if (!count)
      return fail(RTKB_ERR_INVALID_ARGUMENT, "null count");
    std::vector<RayProj> tab;
    std::vector<CylProj> cyl;
    rc = joseph_tables(g->g, *vol, *proj, tab, &cyl);
    if (rc != RTKB_OK)
      return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t tbytes = joseph_table_bytes(tab, cyl);
    void *       scratch = nullptr;
    RTKB_CUDA_TRY(rtkb::scratch_malloc(&scratch, tbytes + sizeof(unsigned long long), st));
    unsigned long long * d_n = reinterpret_cast<unsigned long long *>(static_cast<char *>(scratch) + tbytes);
    unsigned long long   h = 0;
    JosephArgs           a;
    joseph_args(a, *vol, *proj, nullptr);
    cudaError_t e = joseph_upload_tables(tab, cyl, g->g.radius_cylindrical, scratch, a, st);
    if (e == cudaSuccess)
      e = cudaMemsetAsync(d_n, 0, sizeof(unsigned long long), st);
    if (e == cudaSuccess)
    {
      const dim3 grid((unsigned)((a.nu + 31) / 32), (unsigned)((a.nv + 7) / 8), (unsigned)a.np);
      joseph_count_kernel<<<grid, 256, 0, st>>>(a, d_n);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(&h, d_n, sizeof(h), cudaMemcpyDeviceToHost, st);
    rc = (e == cudaSuccess) ? RTKB_OK : cuda_fail(e, "joseph sample count");
    cudaError_t fe = rtkb::scratch_free(scratch, st);
    if (fe == cudaSuccess)
      fe = cudaStreamSynchronize(st);
    if (rc == RTKB_OK && fe != cudaSuccess)
      rc = cuda_fail(fe, "joseph sample count");
    *count = (double)h;
    return rc;
  }
  catch (...)
  {
    return fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

extern "C" int
rtkb_joseph_set_band_rows(int forward_rows, int back_rows)
{
  auto ok = [](int r) { return r == 8 || r == 16 || r == 32 || r == 64; };
  if (!ok(forward_rows) || !ok(back_rows))
    return rtkb::fail(RTKB_ERR_INVALID_ARGUMENT, "band rows must be 8, 16, 32 or 64");
  rtkb::g_joseph_band_rows[0] = forward_rows;
  rtkb::g_joseph_band_rows[1] = back_rows;
  return RTKB_OK;
}

extern "C" int
rtkb_joseph_get_band_rows(int * forward_rows, int * back_rows)
{
  if (forward_rows)
    *forward_rows = rtkb::g_joseph_band_rows[0];
  if (back_rows)
    *back_rows = rtkb::g_joseph_band_rows[1];
  return RTKB_OK;
}

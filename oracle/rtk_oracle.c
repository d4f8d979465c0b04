/*
 * rtk_oracle.c -- FP64 CPU restatement of RTK's hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA product, never part of
 * it.  Every function restates the RTK 2.7.0 source cited in its comment
 * (paths relative to the RTK repository).  All arithmetic is FP64, including
 * image data, except orc_fdk_backproject_f32_rtk, which reproduces RTK's own
 * CPU data types (FP32 data, FP64 coordinates) and is the timed CPU baseline.
 *
 * Parity status: partially pinned (see rtk_oracle.h).
 */
#include "rtk_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#  include <omp.h>
#endif

#define ORC_PI 3.14159265358979323846

/* ------------------------------------------------------------------------ */
/* small matrix helpers (row-major)                                         */
/* ------------------------------------------------------------------------ */
static void
mat_mul(const double * a, const double * b, double * c, int n, int k, int m)
{
  /* c (n x m) = a (n x k) * b (k x m) */
  double t[64];
  for (int i = 0; i < n; i++)
    for (int j = 0; j < m; j++)
    {
      double s = 0.;
      for (int l = 0; l < k; l++)
        s += a[i * k + l] * b[l * m + j];
      t[i * m + j] = s;
    }
  memcpy(c, t, sizeof(double) * n * m);
}

static void
mat4_identity(double * m)
{
  memset(m, 0, 16 * sizeof(double));
  m[0] = m[5] = m[10] = m[15] = 1.;
}

/* inverse of a 4x4 homogeneous affine matrix (last row 0 0 0 1) */
static void
affine4_inverse(const double * m, double * r)
{
  const double a = m[0], b = m[1], c = m[2], d = m[4], e = m[5], f = m[6], g = m[8], h = m[9], i = m[10];
  const double A = e * i - f * h, B = -(d * i - f * g), C = d * h - e * g;
  const double det = a * A + b * B + c * C;
  const double id = 1. / det;
  double       inv[9];
  inv[0] = A * id;
  inv[1] = -(b * i - c * h) * id;
  inv[2] = (b * f - c * e) * id;
  inv[3] = B * id;
  inv[4] = (a * i - c * g) * id;
  inv[5] = -(a * f - c * d) * id;
  inv[6] = C * id;
  inv[7] = -(a * h - b * g) * id;
  inv[8] = (a * e - b * d) * id;
  mat4_identity(r);
  for (int row = 0; row < 3; row++)
  {
    for (int col = 0; col < 3; col++)
      r[row * 4 + col] = inv[row * 3 + col];
    r[row * 4 + 3] = -(inv[row * 3 + 0] * m[3] + inv[row * 3 + 1] * m[7] + inv[row * 3 + 2] * m[11]);
  }
}

static double
convert_0_2pi(double a)
{
  /* ThreeDCircularProjectionGeometry::ConvertAngleBetween0And2PIRadians,
   * src/rtkThreeDCircularProjectionGeometry.cxx:40-44 */
  return a - 2 * ORC_PI * floor(a / (2 * ORC_PI));
}

/* ------------------------------------------------------------------------ */
/* geometry                                                                 */
/* ------------------------------------------------------------------------ */
struct orc_geometry
{
  double   radius_cyl; /* SetRadiusCylindricalDetector; 0: flat panel */
  int      n, cap;
  double * par; /* 10 per projection: sid sdd ga pox poy oop ip sox soy srcangle */
  double * rot; /* 16 */
  double * mag; /* 12 */
  double * srt; /* 16 */
  double * prt; /* 9 */
  double * mat; /* 12 */
};

enum
{
  P_SID,
  P_SDD,
  P_GA,
  P_POX,
  P_POY,
  P_OOP,
  P_IP,
  P_SOX,
  P_SOY,
  P_SANG
};

orc_geometry *
orc_geometry_new(void)
{
  orc_geometry * g = (orc_geometry *)calloc(1, sizeof(orc_geometry));
  return g;
}

void
orc_geometry_set_radius_cylindrical(orc_geometry * g, double radius)
{
  g->radius_cyl = radius;
}

void
orc_geometry_free(orc_geometry * g)
{
  if (!g)
    return;
  free(g->par);
  free(g->rot);
  free(g->mag);
  free(g->srt);
  free(g->prt);
  free(g->mat);
  free(g);
}

static void
geometry_grow(orc_geometry * g)
{
  if (g->n < g->cap)
    return;
  g->cap = g->cap ? 2 * g->cap : 64;
  g->par = (double *)realloc(g->par, sizeof(double) * 10 * g->cap);
  g->rot = (double *)realloc(g->rot, sizeof(double) * 16 * g->cap);
  g->mag = (double *)realloc(g->mag, sizeof(double) * 12 * g->cap);
  g->srt = (double *)realloc(g->srt, sizeof(double) * 16 * g->cap);
  g->prt = (double *)realloc(g->prt, sizeof(double) * 9 * g->cap);
  g->mat = (double *)realloc(g->mat, sizeof(double) * 12 * g->cap);
}

/* ComputeRotationHomogeneousMatrix(angleX, angleY, angleZ):
 * itk::CenteredEuler3DTransform in ZXY order, R = Rz * Rx * Ry
 * (src/rtkThreeDCircularProjectionGeometry.cxx:536-549,
 *  documentation/docs/Geometry.md:60-88) */
static void
rotation_zxy(double ax, double ay, double az, double * m)
{
  const double cx = cos(ax), sx = sin(ax), cy = cos(ay), sy = sin(ay), cz = cos(az), sz = sin(az);
  const double Rx[9] = { 1, 0, 0, 0, cx, -sx, 0, sx, cx };
  const double Ry[9] = { cy, 0, sy, 0, 1, 0, -sy, 0, cy };
  const double Rz[9] = { cz, -sz, 0, sz, cz, 0, 0, 0, 1 };
  double       t[9], r[9];
  mat_mul(Rz, Rx, t, 3, 3, 3);
  mat_mul(t, Ry, r, 3, 3, 3);
  mat4_identity(m);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      m[i * 4 + j] = r[i * 3 + j];
}

static void
rotation_inverse(const double * rot, double * inv)
{
  /* GetRotationMatrices()[i].GetInverse(): the 3x3 block is orthonormal */
  mat4_identity(inv);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      inv[i * 4 + j] = rot[j * 4 + i];
}

int
orc_geometry_add_projection_rad(orc_geometry * g, double sid, double sdd, double gantry, double pox, double poy,
                                double oop, double ip, double sox, double soy)
{
  /* AddProjectionInRadians, src/rtkThreeDCircularProjectionGeometry.cxx:79-153 */
  if (g->n > 0)
  {
    const double sdd0 = g->par[P_SDD];
    if ((sdd == 0.) != (sdd0 == 0.))
      return -1;
  }
  geometry_grow(g);
  const int i = g->n;
  double *  p = g->par + 10 * i;
  p[P_SID] = sid;
  p[P_SDD] = sdd;
  p[P_GA] = convert_0_2pi(gantry);
  p[P_POX] = pox;
  p[P_POY] = poy;
  p[P_OOP] = convert_0_2pi(oop);
  p[P_IP] = convert_0_2pi(ip);
  p[P_SOX] = sox;
  p[P_SOY] = soy;

  double * prt = g->prt + 9 * i;
  memset(prt, 0, 9 * sizeof(double));
  prt[0] = prt[4] = prt[8] = 1.;
  prt[2] = sox - pox;
  prt[5] = soy - poy;

  /* ComputeProjectionMagnificationMatrix(-sdd, -sid), :573-582 */
  double *     mag = g->mag + 12 * i;
  const double msdd = -sdd, msid = -sid;
  memset(mag, 0, 12 * sizeof(double));
  mag[0] = mag[5] = (msdd == 0.) ? 1. : msdd;
  mag[10] = (msdd == 0.) ? 0. : 1.;
  mag[11] = (msdd == 0.) ? 1. : msid;

  rotation_zxy(-oop, -gantry, -ip, g->rot + 16 * i);

  double * srt = g->srt + 16 * i;
  mat4_identity(srt);
  srt[3] = -sox;
  srt[7] = -soy;

  double t1[12], t2[12];
  mat_mul(prt, mag, t1, 3, 3, 4);
  mat_mul(t1, srt, t2, 3, 4, 4);
  mat_mul(t2, g->rot + 16 * i, g->mat + 12 * i, 3, 4, 4);
  g->n++;

  /* source angle, :133-144 */
  double sph[4];
  orc_geometry_source_position(g, i, sph);
  sph[1] = 0.;
  const double nrm = sqrt(sph[0] * sph[0] + sph[1] * sph[1] + sph[2] * sph[2]);
  double       sp[3] = { sph[0] / nrm, sph[1] / nrm, sph[2] / nrm };
  double       a = acos(sp[2]);
  if (sp[0] > 0.)
    a = 2. * ORC_PI - a;
  p[P_SANG] = convert_0_2pi(a);
  return 0;
}

int
orc_geometry_add_projection(orc_geometry * g, double sid, double sdd, double ga, double pox, double poy, double oop,
                            double ip, double sox, double soy)
{
  /* AddProjection, :56-77 */
  const double d2r = atan(1.0) / 45.0;
  return orc_geometry_add_projection_rad(g, sid, sdd, d2r * ga, pox, poy, d2r * oop, d2r * ip, sox, soy);
}

int
orc_geometry_size(const orc_geometry * g)
{
  return g->n;
}

void
orc_geometry_matrix(const orc_geometry * g, int i, double m[12])
{
  memcpy(m, g->mat + 12 * i, 12 * sizeof(double));
}

void
orc_geometry_parameters(const orc_geometry * g, int i, double p[10])
{
  memcpy(p, g->par + 10 * i, 10 * sizeof(double));
}

void
orc_geometry_source_position(const orc_geometry * g, int i, double s[4])
{
  /* GetSourcePosition, :597-608 */
  const double * p = g->par + 10 * i;
  double         inv[16];
  rotation_inverse(g->rot + 16 * i, inv);
  const double v[4] = { p[P_SOX], p[P_SOY], p[P_SID], 1. };
  mat_mul(inv, v, s, 4, 4, 1);
}

void
orc_geometry_proj_coords_to_fixed(const orc_geometry * g, int i, double m[16])
{
  /* GetProjectionCoordinatesToDetectorSystemMatrix + ...ToFixedSystemMatrix, :611-637 */
  const double * p = g->par + 10 * i;
  double         d[16], inv[16];
  mat4_identity(d);
  d[3] = p[P_POX];
  d[7] = p[P_POY];
  d[11] = (p[P_SDD] == 0.) ? -p[P_SID] : p[P_SID] - p[P_SDD];
  d[10] = 0.;
  rotation_inverse(g->rot + 16 * i, inv);
  mat_mul(inv, d, m, 4, 4, 4);
}

/* Cylindrical panel (ProjectionsRegionConstIteratorRayBasedWithCylindricalPanel,
 * include/rtkProjectionsRegionConstIteratorRayBasedWithCylindricalPanel.hxx):
 * idx2det = GetProjectionCoordinatesToDetectorSystemMatrix(i) x the stack's
 * index-to-physical matrix; inv = the inverse rotation (detector -> fixed). */
static void
cyl_matrices(const orc_geometry * g, int i, const double * pi2pp, double * idx2det, double * inv)
{
  const double * p = g->par + 10 * i;
  double         d[16];
  mat4_identity(d);
  d[3] = p[P_POX];
  d[7] = p[P_POY];
  d[11] = (p[P_SDD] == 0.) ? -p[P_SID] : p[P_SID] - p[P_SDD];
  d[10] = 0.;
  mat_mul(d, pi2pp, idx2det, 4, 4, 4);
  rotation_inverse(g->rot + 16 * i, inv);
}

/* NewPixel of the same iterator: the flat-panel u is an arc length on the
 * cylinder of radius R; its angle a = u / R gives u' = R sin a and
 * w' = w + R (1 - cos a); out = M x (u', v, w', 1) */
static void
cyl_pixel(const double * idx2det, const double * M, double radius, double iu, double iv, double ik, double * out)
{
  double pos[3];
  for (int a = 0; a < 3; a++)
    pos[a] = idx2det[a * 4 + 0] * iu + idx2det[a * 4 + 1] * iv + idx2det[a * 4 + 2] * ik + idx2det[a * 4 + 3];
  const double ang = pos[0] / radius;
  pos[0] = sin(ang) * radius;
  pos[2] += (1. - cos(ang)) * radius;
  for (int a = 0; a < 3; a++)
    out[a] = M[a * 4 + 3] + M[a * 4 + 0] * pos[0] + M[a * 4 + 1] * pos[1] + M[a * 4 + 2] * pos[2];
}

/* Parallel beam (SDD 0): ProjectionsRegionConstIteratorRayBasedParallel
 * (include/rtkProjectionsRegionConstIteratorRayBasedParallel.hxx:40-75) with
 * the identity post-matrix (RayConvexIntersectionImageFilter): pixel - source
 * = -2 SID x row 2 of the rotation matrix, in mm.  Returns 1 for a parallel
 * projection, 0 (s2p untouched) otherwise. */
static int
parallel_source_to_pixel(const orc_geometry * g, int i, double s2p[3])
{
  if (g->par[10 * i + P_SDD] != 0.)
    return 0;
  const double * R = g->rot + 16 * i + 8;
  for (int a = 0; a < 3; a++)
    s2p[a] = -2. * g->par[10 * i + P_SID] * R[a];
  return 1;
}

void
orc_geometry_source_angles(const orc_geometry * g, double * out)
{
  for (int i = 0; i < g->n; i++)
    out[i] = g->par[10 * i + P_SANG];
}

void
orc_geometry_gantry_angles(const orc_geometry * g, double * out)
{
  for (int i = 0; i < g->n; i++)
    out[i] = g->par[10 * i + P_GA];
}

void
orc_geometry_tilt_angles(const orc_geometry * g, double * out)
{
  /* GetTiltAngles, :407-418 */
  for (int i = 0; i < g->n; i++)
    out[i] = convert_0_2pi(-1. * g->par[10 * i + P_GA] - g->par[10 * i + P_SANG]);
}

typedef struct
{
  double a;
  int    i;
} angle_idx;

static int
cmp_angle(const void * x, const void * y)
{
  const angle_idx * p = (const angle_idx *)x;
  const angle_idx * q = (const angle_idx *)y;
  if (p->a < q->a)
    return -1;
  if (p->a > q->a)
    return 1;
  /* std::multimap keeps insertion order for equal keys */
  return p->i - q->i;
}

static angle_idx *
sorted_angles(const double * angles, int n)
{
  angle_idx * s = (angle_idx *)malloc(sizeof(angle_idx) * (n > 0 ? n : 1));
  for (int i = 0; i < n; i++)
  {
    s[i].a = angles[i];
    s[i].i = i;
  }
  qsort(s, n, sizeof(angle_idx), cmp_angle);
  return s;
}

void
orc_geometry_angular_gaps(const orc_geometry * g, const double * angles, double * out)
{
  /* GetAngularGaps, :478-533 */
  const int n = g->n;
  if (n == 1)
    out[0] = 2 * ORC_PI;
  if (n < 2)
    return;
  angle_idx * s = sorted_angles(angles, n);
  out[s[0].i] = 0.5 * (s[1].a - s[n - 1].a + 2 * ORC_PI);
  for (int k = 1; k < n - 1; k++)
    out[s[k].i] = 0.5 * (s[k + 1].a - s[k - 1].a);
  out[s[n - 1].i] = 0.5 * (s[0].a + 2 * ORC_PI - s[n - 2].a);
  if (g->par[P_SDD] == 0.)
  {
    double mx = out[0];
    for (int k = 1; k < n; k++)
      if (out[k] > mx)
        mx = out[k];
    if (mx > ORC_PI / 2)
      for (int k = 0; k < n; k++)
      {
        if (out[k] > ORC_PI / 2)
          out[k] -= ORC_PI / 2;
        out[k] *= 2.;
      }
  }
  free(s);
}

void
orc_geometry_angular_gaps_with_next(const orc_geometry * g, const double * angles, double * out)
{
  /* GetAngularGapsWithNext, :447-476 */
  const int n = g->n;
  if (n == 1)
    out[0] = 2 * ORC_PI;
  if (n < 2)
    return;
  angle_idx * s = sorted_angles(angles, n);
  for (int k = 0; k < n - 1; k++)
    out[s[k].i] = s[k + 1].a - s[k].a;
  out[s[n - 1].i] = s[0].a + 2 * ORC_PI - s[n - 1].a;
  free(s);
}

double
orc_geometry_to_untilted(const orc_geometry * g, int i, double tilted)
{
  /* ToUntiltedCoordinateAtIsocenter, :641-663 */
  const double * p = g->par + 10 * i;
  const double   sid = p[P_SID], sdd = p[P_SDD], sx = p[P_SOX], px = p[P_POX];
  const double   sidu = sqrt(sid * sid + sx * sx);
  const double   l = (tilted + px - sx) * sid / sdd + sx;
  const double   cosa = sx / sidu;
  return l * fabs(sid) / (sidu - l * cosa);
}

/* ------------------------------------------------------------------------ */
/* image matrices (include/rtkHomogeneousMatrix.h:38-81)                     */
/* ------------------------------------------------------------------------ */
void
orc_index_to_physical(const orc_image * im, double m[16])
{
  mat4_identity(m);
  for (int i = 0; i < 3; i++)
  {
    for (int j = 0; j < 3; j++)
      m[i * 4 + j] = im->direction[i * 3 + j] * im->spacing[j];
    m[i * 4 + 3] = im->origin[i];
  }
}

void
orc_physical_to_index(const orc_image * im, double m[16])
{
  double a[16];
  orc_index_to_physical(im, a);
  affine4_inverse(a, m);
}

static long
npix(const orc_image * im)
{
  return (long)im->size[0] * im->size[1] * im->size[2];
}

/* ------------------------------------------------------------------------ */
/* voxel-based and FDK backprojection                                       */
/* ------------------------------------------------------------------------ */
typedef struct
{
  double S[3], O[3], eu[3], ev[3], n[3];
  double a[3], b[3];     /* stack physical (u, v, 1) -> absolute index */
  double h, c0, su, sv;  /* (O - S).n, (0 - S).n, (S - O).eu, (S - O).ev */
  int    parallel, fdk, mode;
} bp_frame_t;
int
orc_bp_matrix(const orc_geometry * g, const orc_image * vol, const orc_image * proj, int i, int fdk, double m[12])
{
  /* GetIndexToIndexProjectionMatrix, include/rtkBackProjectionImageFilter.hxx:535-595
   * (untransposed: the transposition of :480-531 only changes memory layout) */
  double vi2pp[16], t[12], volidx_to_projpp[12];
  orc_index_to_physical(vol, vi2pp);
  mat_mul(g->mag + 12 * i, g->srt + 16 * i, t, 3, 4, 4);
  mat_mul(t, g->rot + 16 * i, t, 3, 4, 4);
  mat_mul(t, vi2pp, volidx_to_projpp, 3, 4, 4);

  double spp2i[16], mp[9], pp2pi[9];
  orc_physical_to_index(proj, spp2i);
  memset(mp, 0, sizeof(mp));
  for (int r = 0; r < 2; r++)
  {
    mp[r * 3 + 2] = spp2i[r * 4 + 3];
    for (int c = 0; c < 2; c++)
      mp[r * 3 + c] = spp2i[r * 4 + c];
  }
  mp[8] = 1.;
  mat_mul(mp, g->prt + 9 * i, pp2pi, 3, 3, 3);
  mat_mul(pp2pi, volidx_to_projpp, m, 3, 3, 4);

  if (fdk)
  {
    /* normalisation at the rotation centre,
     * include/rtkFDKBackProjectionImageFilter.hxx:80-104 */
    double vpp2i[16];
    orc_physical_to_index(vol, vpp2i);
    const double rc[3] = { vpp2i[3], vpp2i[7], vpp2i[11] };
    double       persp = m[11];
    for (int j = 0; j < 3; j++)
      persp += m[8 + j] * rc[j];
    for (int j = 0; j < 12; j++)
      m[j] /= persp;
  }
  /* path selection on the transposed matrix, :106-116: transposed row 1 is
   * the untransposed row 0 */
  if (fabs(m[0]) < 1e-10 && fabs(m[8]) < 1e-10)
    return 1;
  if (fabs(m[1]) < 1e-10 && fabs(m[9]) < 1e-10)
    return 2;
  return 0;
}

/* The detector frame of one projection in the fixed (physical) system:
 * source S (GetSourcePosition, src/rtkThreeDCircularProjectionGeometry.cxx:597-608),
 * detector origin O and unit axes eu, ev (the columns of
 * GetProjectionCoordinatesToFixedSystemMatrix, :611-637), normal n = eu x ev
 * (pointing at the source), and the stack's physical -> index map restricted
 * to u, v (ci = a . (pu, pv, 1), cj = b . (pu, pv, 1)), as RTK restricts it. */
static void
bp_frame(const orc_geometry * g, const orc_image * vol, const orc_image * proj, int k, int fdk, bp_frame_t * f)
{
  double m[16], s4[4], p2i[16];
  orc_geometry_proj_coords_to_fixed(g, k, m);
  orc_geometry_source_position(g, k, s4);
  orc_physical_to_index(proj, p2i);
  for (int a = 0; a < 3; a++)
  {
    f->S[a] = s4[a];
    f->eu[a] = m[a * 4 + 0];
    f->ev[a] = m[a * 4 + 1];
    f->O[a] = m[a * 4 + 3];
  }
  f->n[0] = f->eu[1] * f->ev[2] - f->eu[2] * f->ev[1];
  f->n[1] = f->eu[2] * f->ev[0] - f->eu[0] * f->ev[2];
  f->n[2] = f->eu[0] * f->ev[1] - f->eu[1] * f->ev[0];
  f->a[0] = p2i[0];
  f->a[1] = p2i[1];
  f->a[2] = p2i[3];
  f->b[0] = p2i[4];
  f->b[1] = p2i[5];
  f->b[2] = p2i[7];
  f->parallel = g->par[10 * k + P_SDD] == 0.;
  f->fdk = fdk;
  double SO[3], Sn = 0., h = 0.;
  for (int a = 0; a < 3; a++)
  {
    SO[a] = f->S[a] - f->O[a];
    Sn += f->S[a] * f->n[a];
    h -= SO[a] * f->n[a];
  }
  f->h = h;         /* (O - S) . n */
  f->c0 = -Sn;      /* (X - S) . n at the physical origin (RTK's rotation centre) */
  f->su = SO[0] * f->eu[0] + SO[1] * f->eu[1] + SO[2] * f->eu[2];
  f->sv = SO[0] * f->ev[0] + SO[1] * f->ev[1] + SO[2] * f->ev[2];
  /* RTK's choice between its optimised and generic paths
   * (include/rtkFDKBackProjectionImageFilter.hxx:106-116,
   * include/rtkBackProjectionImageFilter.hxx:220-230): the optimised Y (X)
   * path when the homogeneous u numerator and w do not change along the
   * volume's y (x) index, both below 1e-10 in RTK's scaling (w = (X - S).n,
   * divided by its value at the rotation centre for FDK; w = 1 for a
   * parallel beam).  Their rates along an index axis with physical step
   * delta: du = K (delta.n) + h (a0 delta.eu + a1 delta.ev), dw = delta.n, K the
   * u index of the point where the detector plane is met by the ray through
   * S parallel to it (a0 su + a1 sv + a2); parallel beam: du = a0 delta.eu +
   * a1 delta.ev, dw = 0. */
  double rate_u[2], rate_w[2];
  for (int ax = 0; ax < 2; ax++)
  {
    double d[3], dn = 0., de = 0., dv = 0.;
    for (int a = 0; a < 3; a++)
    {
      d[a] = vol->direction[a * 3 + ax] * vol->spacing[ax];
      dn += d[a] * f->n[a];
      de += d[a] * f->eu[a];
      dv += d[a] * f->ev[a];
    }
    if (f->parallel)
    {
      rate_u[ax] = f->a[0] * de + f->a[1] * dv;
      rate_w[ax] = 0.;
    }
    else
    {
      const double K = f->a[0] * f->su + f->a[1] * f->sv + f->a[2];
      rate_u[ax] = K * dn + h * (f->a[0] * de + f->a[1] * dv);
      rate_w[ax] = dn;
      if (fdk)
      {
        rate_u[ax] /= f->c0;
        rate_w[ax] /= f->c0;
      }
    }
  }
  if (fabs(rate_u[0]) < 1e-10 && fabs(rate_w[0]) < 1e-10)
    f->mode = 1;
  else if (fabs(rate_u[1]) < 1e-10 && fabs(rate_w[1]) < 1e-10)
    f->mode = 2;
  else
    f->mode = 0;
}

/* Continuous projection index (absolute) of the physical point X and the FDK
 * weight: cone beam, the detector-plane point P = S + t (X - S) with
 * t = ((O - S).n) / ((X - S).n), (pu, pv) = ((P - O).eu, (P - O).ev), weight
 * (w0 / w)^2 with w = (X - S).n, w0 its value at the rotation centre (the
 * distance ratio along the normal; 1 without FDK); parallel beam, P the
 * orthogonal projection of X, weight 1. */
static void
bp_frame_map(const bp_frame_t * f, const double * X, double * u, double * v, double * wt)
{
  double pu, pv;
  *wt = 1.;
  if (f->parallel)
  {
    double XO[3];
    for (int a = 0; a < 3; a++)
      XO[a] = X[a] - f->O[a];
    pu = XO[0] * f->eu[0] + XO[1] * f->eu[1] + XO[2] * f->eu[2];
    pv = XO[0] * f->ev[0] + XO[1] * f->ev[1] + XO[2] * f->ev[2];
  }
  else
  {
    double d[3];
    for (int a = 0; a < 3; a++)
      d[a] = X[a] - f->S[a];
    const double dn = d[0] * f->n[0] + d[1] * f->n[1] + d[2] * f->n[2];
    const double t = f->h / dn;
    pu = f->su + t * (d[0] * f->eu[0] + d[1] * f->eu[1] + d[2] * f->eu[2]);
    pv = f->sv + t * (d[0] * f->ev[0] + d[1] * f->ev[1] + d[2] * f->ev[2]);
    if (f->fdk)
    {
      const double r = f->c0 / dn;
      *wt = r * r;
    }
  }
  *u = f->a[0] * pu + f->a[1] * pv + f->a[2];
  *v = f->b[0] * pu + f->b[1] * pv + f->b[2];
}

int
orc_bp_project(const orc_geometry * g, const orc_image * vol, const orc_image * proj, int k, int fdk,
               const double * physical, double out[3])
{
  bp_frame_t f;
  bp_frame(g, vol, proj, k, fdk, &f);
  bp_frame_map(&f, physical, out, out + 1, out + 2);
  return f.mode;
}

static double
interp_clamped(const double * p, int nu, int nv, double u, double v)
{
  /* itk::LinearInterpolateImageFunction on a 2-D image: clamp-to-edge bilinear */
  double uc = u < 0. ? 0. : (u > nu - 1 ? nu - 1 : u);
  double vc = v < 0. ? 0. : (v > nv - 1 ? nv - 1 : v);
  int    iu = (int)floor(uc), iv = (int)floor(vc);
  int    iu1 = iu + 1 < nu ? iu + 1 : nu - 1;
  int    iv1 = iv + 1 < nv ? iv + 1 : nv - 1;
  double fu = uc - iu, fv = vc - iv;
  double a = p[(long)iv * nu + iu] + fu * (p[(long)iv * nu + iu1] - p[(long)iv * nu + iu]);
  double b = p[(long)iv1 * nu + iu] + fu * (p[(long)iv1 * nu + iu1] - p[(long)iv1 * nu + iu]);
  return a + fv * (b - a);
}

void
orc_backproject(const orc_geometry * g, const orc_image * vol, const orc_image * proj, const double * proj_data,
                const double * vol_in, double * vol_out, int fdk, int nthreads)
{
  /* BackProjectionImageFilter::DynamicThreadedGenerateData
   * (include/rtkBackProjectionImageFilter.hxx:185-279) and
   * FDKBackProjectionImageFilter::DynamicThreadedGenerateData
   * (include/rtkFDKBackProjectionImageFilter.hxx:52-148) with their optimised
   * paths (:152-306 and :352-475): RTK's u = (M0.x)/(M2.x), v = (M1.x)/(M2.x)
   * and weight (1/(M2.x))^2 after normalisation at the rotation centre are
   * computed here by bp_frame_map (the same quantities, derived from the
   * source and the detector frame instead of RTK's composed matrix);
   * optimised paths accept 0 <= floor(u) < Nu-1 and 0 <= floor(v) < Nv-1,
   * the generic path accepts [-0.5, N-0.5) with clamp-to-edge interpolation. */
  const int  nx = vol->size[0], ny = vol->size[1], nz = vol->size[2];
  const int  nu = proj->size[0], nv = proj->size[1], np = proj->size[2];
  const long nvox = npix(vol);
  if (vol_out != vol_in)
    memcpy(vol_out, vol_in, sizeof(double) * nvox);
  if (!fdk && g->radius_cyl != 0.)
  {
    /* CylindricalDetectorCenteredOnSourceBackprojection
     * (include/rtkBackProjectionImageFilter.hxx:283-345) with the matrices of
     * :551-595: (a, b, c) = Mag Src Rot I2P_vol x, u = a/c, v = b/c,
     * u' = R atan2(u, R), v' = v R / sqrt(R^2 + u^2), index = P2I_proj ProjT (u', v'),
     * clamp-to-edge bilinear inside [-0.5, N - 0.5) */
    const double R = g->radius_cyl;
    double       i2p[16], p2i[16];
    orc_index_to_physical(vol, i2p);
    orc_physical_to_index(proj, p2i);
    for (int s = 0; s < np; s++)
    {
      const int      k = proj->index[2] + s;
      double         t1[12], t2[12], A[12], B[9];
      const double   m[9] = { p2i[0], p2i[1], p2i[3], p2i[4], p2i[5], p2i[7], 0., 0., 1. };
      const double * p = proj_data + (long)s * nu * nv;
      mat_mul(g->mag + 12 * k, g->srt + 16 * k, t1, 3, 4, 4);
      mat_mul(t1, g->rot + 16 * k, t2, 3, 4, 4);
      mat_mul(t2, i2p, A, 3, 4, 4);
      mat_mul(m, g->prt + 9 * k, B, 3, 3, 3);
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
      for (int kz = 0; kz < nz; kz++)
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < nx; i++)
          {
            const double x = i + vol->index[0], y = j + vol->index[1], z = kz + vol->index[2];
            const double c = A[8] * x + A[9] * y + A[10] * z + A[11];
            const double u = (A[0] * x + A[1] * y + A[2] * z + A[3]) / c;
            const double v = (A[4] * x + A[5] * y + A[6] * z + A[7]) / c;
            const double u2 = R * atan2(u, R), v2 = v * R / sqrt(R * R + u * u);
            const double ci = B[0] * u2 + B[1] * v2 + B[2] - proj->index[0];
            const double cj = B[3] * u2 + B[4] * v2 + B[5] - proj->index[1];
            if (ci >= -0.5 && ci < nu - 0.5 && cj >= -0.5 && cj < nv - 0.5)
              vol_out[((long)kz * ny + j) * nx + i] += interp_clamped(p, nu, nv, ci, cj);
          }
    }
    return;
  }
  /* Flat panels.  The voxel -> pixel map is derived here from the geometry's
   * frame, not from RTK's composed index-to-index matrix (orc_bp_matrix, kept
   * as a separate restatement and checked against this derivation): the ray
   * from the source through the voxel centre meets the detector plane. */
  bp_frame_t * fr = (bp_frame_t *)malloc(sizeof(bp_frame_t) * (np > 0 ? np : 1));
  for (int s = 0; s < np; s++)
    bp_frame(g, vol, proj, proj->index[2] + s, fdk, fr + s);
  double i2p[16];
  orc_index_to_physical(vol, i2p);
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
  for (int k = 0; k < nz; k++)
  {
    for (int s = 0; s < np; s++)
    {
      const bp_frame_t * f = fr + s;
      const double *     p = proj_data + (long)s * nu * nv;
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++)
        {
          const double idx[3] = { i + vol->index[0], j + vol->index[1], k + vol->index[2] };
          double       X[3], u, v, wt;
          for (int a = 0; a < 3; a++)
            X[a] = i2p[a * 4 + 0] * idx[0] + i2p[a * 4 + 1] * idx[1] + i2p[a * 4 + 2] * idx[2] + i2p[a * 4 + 3];
          bp_frame_map(f, X, &u, &v, &wt);
          u -= proj->index[0];
          v -= proj->index[1];
          const long o = ((long)k * ny + j) * nx + i;
          if (f->mode)
          {
            const int iu = (int)floor(u), iv = (int)floor(v);
            if (iu >= 0 && iu < nu - 1 && iv >= 0 && iv < nv - 1)
            {
              const double fu = u - iu, fv = v - iv;
              const double * q = p + (long)iv * nu + iu;
              vol_out[o] += wt * ((1 - fv) * ((1 - fu) * q[0] + fu * q[1]) + fv * ((1 - fu) * q[nu] + fu * q[nu + 1]));
            }
          }
          else if (u >= -0.5 && u < nu - 0.5 && v >= -0.5 && v < nv - 0.5)
            vol_out[o] += wt * interp_clamped(p, nu, nv, u, v);
        }
    }
  }
  free(fr);
}

/* ------------------------------------------------------------------------ */
/* Joseph projector pair                                                    */
/* ------------------------------------------------------------------------ */
typedef struct
{
  double pix[3], dir[3];
} ray_t;

/* BoxShape::IsIntersectedByRay with identity direction, src/rtkBoxShape.cxx:47-97 */
static int
box_intersect(const double * bmin, const double * bmax, const double * org, const double * dir, double * tin,
              double * tout)
{
  double inf = -DBL_MAX, sup = DBL_MAX;
  for (int i = 0; i < 3; i++)
  {
    double mn = bmin[i], mx = bmax[i];
    if (mn > mx)
    {
      double t = mn;
      mn = mx;
      mx = t;
    }
    if (dir[i] == 0. && (org[i] < mn || org[i] > mx))
      return 0;
    const double inv = 1 / dir[i];
    double       t1 = (mn - org[i]) * inv, t2 = (mx - org[i]) * inv;
    if (t1 > t2)
    {
      double t = t1;
      t1 = t2;
      t2 = t;
    }
    if (t1 > inf)
      inf = t1;
    if (t2 < sup)
      sup = t2;
    if (inf > sup)
      return 0;
    if (sup < 0.)
      return 0;
  }
  *tin = inf;
  *tout = sup;
  return 1;
}

typedef struct
{
  double pix2vol[16]; /* projection index -> volume index (homogeneous) */
  double src[3];      /* source in volume index coordinates */
  int    parallel;    /* parallel beam: every pixel has its own source */
  double s2p[3];      /* parallel beam: pixel - source, volume index coordinates */
  double radius;      /* cylindrical panel radius, 0: flat */
  double idx2det[16]; /* cylindrical: projection index -> flat detector coordinates */
  double det2vol[16]; /* cylindrical: detector coordinates -> volume index */
} joseph_proj_t;

static void
joseph_setup(const orc_geometry * g, const orc_image * vol, const orc_image * proj, int i, joseph_proj_t * jp)
{
  /* ProjectionsRegionConstIteratorRayBasedWithFlatPanel::NewProjection,
   * include/rtkProjectionsRegionConstIteratorRayBasedWithFlatPanel.hxx:39-71 */
  double vpp2i[16], p2f[16], pi2pp[16], t[16], s4[4], sv[4];
  orc_physical_to_index(vol, vpp2i);
  orc_geometry_proj_coords_to_fixed(g, i, p2f);
  orc_index_to_physical(proj, pi2pp);
  mat_mul(vpp2i, p2f, t, 4, 4, 4);
  mat_mul(t, pi2pp, jp->pix2vol, 4, 4, 4);
  orc_geometry_source_position(g, i, s4);
  mat_mul(vpp2i, s4, sv, 4, 4, 1);
  jp->src[0] = sv[0];
  jp->src[1] = sv[1];
  jp->src[2] = sv[2];
  /* ProjectionsRegionConstIteratorRayBased::New picks the parallel iterator
   * when the SDD is 0 (include/rtkProjectionsRegionConstIteratorRayBased.hxx:86-98).
   * ...Parallel::NewProjection (include/rtkProjectionsRegionConstIteratorRayBasedParallel.hxx:40-60):
   * SourceToPixel = -2 SID x (row 2 of the rotation matrix), mapped by the
   * 3x3 part of the volume's physical-to-index matrix; NewPixel puts the
   * source at pixel - SourceToPixel, so every ray is parallel to that row. */
  jp->parallel = g->par[10 * i + P_SDD] == 0.;
  if (jp->parallel)
  {
    const double * R = g->rot + 16 * i + 8;
    const double   sid = g->par[10 * i + P_SID];
    for (int a = 0; a < 3; a++)
      jp->s2p[a] = -2. * sid * (vpp2i[a * 4 + 0] * R[0] + vpp2i[a * 4 + 1] * R[1] + vpp2i[a * 4 + 2] * R[2]);
  }
  /* ProjectionsRegionConstIteratorRayBasedWithCylindricalPanel::NewProjection
   * (include/rtkProjectionsRegionConstIteratorRayBasedWithCylindricalPanel.hxx):
   * index -> detector system (GetProjectionCoordinatesToDetectorSystemMatrix x
   * the stack's index-to-physical matrix), detector -> volume index (the
   * volume's physical-to-index matrix x the inverse rotation) */
  jp->radius = g->radius_cyl;
  if (jp->radius != 0.)
  {
    double inv[16];
    cyl_matrices(g, i, pi2pp, jp->idx2det, inv);
    mat_mul(vpp2i, inv, jp->det2vol, 4, 4, 4);
  }
}

typedef struct
{
  int    main, dinf, dsup;
  int    ns, fs;
  double np_main, fp_main;
  double residualB, residualE, stepx, stepy, curx, cury;
  double stepmm_norm;
  double minx, miny, maxx, maxy;
  long   ox, oy, oz;
} joseph_ray_t;

/* Ray set-up shared by the forward and back projectors,
 * include/rtkJosephForwardProjectionImageFilter.hxx:244-335 and
 * include/rtkJosephBackProjectionImageFilter.hxx:127-201.
 * forward != 0 selects the forward acceptance test.  Returns 1 if the ray is
 * cast. */
static int
joseph_ray(const orc_image * vol, const joseph_proj_t * jp, double iu, double iv, double ik, int forward,
           joseph_ray_t * r)
{
  double pix[3], dir[3], bmin[3], bmax[3];
  if (jp->radius != 0.)
    cyl_pixel(jp->idx2det, jp->det2vol, jp->radius, iu, iv, ik, pix);
  else
    for (int a = 0; a < 3; a++)
      pix[a] = jp->pix2vol[a * 4 + 0] * iu + jp->pix2vol[a * 4 + 1] * iv + jp->pix2vol[a * 4 + 2] * ik +
               jp->pix2vol[a * 4 + 3];
  for (int a = 0; a < 3; a++) /* dirVox = -SourceToPixel */
    dir[a] = jp->parallel ? -jp->s2p[a] : -(pix[a] - jp->src[a]);
  int mainDir = 0;
  for (int a = 0; a < 3; a++)
    if (fabs(dir[a]) > fabs(dir[mainDir]))
      mainDir = a;
  for (int a = 0; a < 3; a++)
  {
    bmin[a] = vol->index[a];
    bmax[a] = vol->index[a] + vol->size[a] - 1;
    bmax[a] *= 1. - DBL_EPSILON;
  }
  double infd = 0., supd = 0.;
  int    hit = box_intersect(bmin, bmax, pix, dir, &infd, &supd);
  if (forward)
  {
    if (infd < 0.)
      infd = 0.;
    if (supd > 1.)
      supd = 1.;
    if (!(hit && supd > 0. && infd <= 1. && supd > infd))
      return 0;
  }
  else
  {
    if (!(hit && supd >= 0. && infd <= 1.))
      return 0;
    if (infd < 0.)
      infd = 0.;
    if (supd > 1.)
      supd = 1.;
  }
  double np[3], fp[3];
  for (int a = 0; a < 3; a++)
  {
    np[a] = pix[a] + infd * dir[a];
    fp[a] = pix[a] + supd * dir[a];
  }
  r->main = mainDir;
  r->ns = (int)rint(np[mainDir]);
  r->fs = (int)rint(fp[mainDir]);
  int dinf = (mainDir + 1) % 3, dsup = (mainDir + 2) % 3;
  if (dinf > dsup)
  {
    int t = dinf;
    dinf = dsup;
    dsup = t;
  }
  r->dinf = dinf;
  r->dsup = dsup;
  r->minx = bmin[dinf];
  r->miny = bmin[dsup];
  r->maxx = bmax[dinf];
  r->maxy = bmax[dsup];
  const long offsets[3] = { 1, vol->size[0], (long)vol->size[0] * vol->size[1] };
  r->ox = offsets[dinf];
  r->oy = offsets[dsup];
  r->oz = offsets[mainDir];
  r->np_main = np[mainDir];
  r->fp_main = fp[mainDir];
  r->residualB = r->ns - np[mainDir];
  r->residualE = fp[mainDir] - r->fs;
  const double nrm = 1. / dir[mainDir];
  r->stepx = dir[dinf] * nrm;
  r->stepy = dir[dsup] * nrm;
  if (np[mainDir] > fp[mainDir])
  {
    r->residualB *= -1;
    r->residualE *= -1;
    r->oz *= -1;
    r->stepx *= -1;
    r->stepy *= -1;
  }
  r->curx = np[dinf] + r->residualB * r->stepx;
  r->cury = np[dsup] + r->residualB * r->stepy;
  double smm[3];
  smm[dinf] = vol->spacing[dinf] * r->stepx;
  smm[dsup] = vol->spacing[dsup] * r->stepy;
  smm[mainDir] = vol->spacing[mainDir];
  r->stepmm_norm = sqrt(smm[0] * smm[0] + smm[1] * smm[1] + smm[2] * smm[2]);
  return 1;
}

/* buffer offset of the absolute voxel index along one axis */
static long
clampl(long v, long lo, long hi)
{
  return v < lo ? lo : (v > hi ? hi : v);
}

/* Joseph bilinear (BilinearInterpolation / ...OnBorders, FP :443-543; BP
 * :335-413).  Returns the four buffer offsets and weights of a sample at
 * (x, y) in slice sl.  Indices are clamped into the buffer to guard rounding
 * at the box faces (a no-op for the in-box samples RTK takes). */
static void
joseph_taps(const orc_image * vol, const joseph_ray_t * r, int sl, double x, double y, int border, long o[4],
            double wgt[4])
{
  const int    ix = (int)floor(x), iy = (int)floor(y);
  const double lx = x - ix, ly = y - iy, lxc = 1. - lx, lyc = 1. - ly;
  const int    szx = vol->size[r->dinf], szy = vol->size[r->dsup];
  const int    bx = vol->index[r->dinf], by = vol->index[r->dsup], bz = vol->index[r->main];
  long         xi = ix, xs = ix + 1, yi = iy, ys = iy + 1;
  if (border)
  {
    if (ix < r->minx)
      xi = ix + 1;
    if (iy < r->miny)
      yi = iy + 1;
    if (ix >= r->maxx)
      xs = ix;
    if (iy >= r->maxy)
      ys = iy;
  }
  xi = clampl(xi - bx, 0, szx - 1);
  xs = clampl(xs - bx, 0, szx - 1);
  yi = clampl(yi - by, 0, szy - 1);
  ys = clampl(ys - by, 0, szy - 1);
  const long zo = (long)(sl - bz);
  const long oz = labs(r->oz);
  o[0] = zo * oz + xi * r->ox + yi * r->oy;
  o[1] = zo * oz + xs * r->ox + yi * r->oy;
  o[2] = zo * oz + xi * r->ox + ys * r->oy;
  o[3] = zo * oz + xs * r->ox + ys * r->oy;
  wgt[0] = lxc * lyc;
  wgt[1] = lx * lyc;
  wgt[2] = lxc * ly;
  wgt[3] = lx * ly;
}

void
orc_joseph_forward(const orc_geometry * g, const orc_image * vol, const double * vol_data, const orc_image * proj,
                   const double * proj_in, double * proj_out, int nthreads)
{
  /* JosephForwardProjectionImageFilter::ThreadedGenerateData,
   * include/rtkJosephForwardProjectionImageFilter.hxx:182-427 */
  const int nu = proj->size[0], nv = proj->size[1], np = proj->size[2];
  for (int s = 0; s < np; s++)
  {
    joseph_proj_t jp;
    joseph_setup(g, vol, proj, proj->index[2] + s, &jp);
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 4)
    for (int j = 0; j < nv; j++)
      for (int i = 0; i < nu; i++)
      {
        const long   po = ((long)s * nv + j) * nu + i;
        joseph_ray_t r;
        if (!joseph_ray(vol, &jp, i + proj->index[0], j + proj->index[1], proj->index[2] + s, 1, &r))
        {
          proj_out[po] = proj_in[po];
          continue;
        }
        const int dz = (r.np_main > r.fp_main) ? -1 : 1;
        double    sum = 0.;
        long      o[4];
        double    w[4];
        int       sl = r.ns;
        double    x = r.curx, y = r.cury;
        if (r.fs == r.ns)
        {
          joseph_taps(vol, &r, sl, x, y, 1, o, w);
          sum += fabs(r.fp_main - r.np_main) *
                 (w[0] * vol_data[o[0]] + w[2] * vol_data[o[2]] + w[1] * vol_data[o[1]] + w[3] * vol_data[o[3]]);
        }
        else
        {
          joseph_taps(vol, &r, sl, x, y, 1, o, w);
          sum += (r.residualB + 0.5) *
                 (w[0] * vol_data[o[0]] + w[2] * vol_data[o[2]] + w[1] * vol_data[o[1]] + w[3] * vol_data[o[3]]);
          sl += dz;
          x += r.stepx;
          y += r.stepy;
          const int nmid = abs(r.fs - r.ns) - 1;
          for (int t = 0; t < nmid; t++)
          {
            joseph_taps(vol, &r, sl, x, y, 0, o, w);
            sum += w[0] * vol_data[o[0]] + w[1] * vol_data[o[1]] + w[2] * vol_data[o[2]] + w[3] * vol_data[o[3]];
            sl += dz;
            x += r.stepx;
            y += r.stepy;
          }
          joseph_taps(vol, &r, sl, x, y, 1, o, w);
          sum += (r.residualE + 0.5) *
                 (w[0] * vol_data[o[0]] + w[2] * vol_data[o[2]] + w[1] * vol_data[o[1]] + w[3] * vol_data[o[3]]);
        }
        proj_out[po] = proj_in[po] + sum * r.stepmm_norm;
      }
  }
}

/* Joseph back projection of stack slices [s0, s1) added into vol_out. */
static void
joseph_back_slices(const orc_geometry * g, const orc_image * vol, double * vol_out, const orc_image * proj,
                   const double * proj_data, int s0, int s1)
{
  const int nu = proj->size[0], nv = proj->size[1];
  for (int s = s0; s < s1; s++)
  {
    joseph_proj_t jp;
    joseph_setup(g, vol, proj, proj->index[2] + s, &jp);
    for (int j = 0; j < nv; j++)
      for (int i = 0; i < nu; i++)
      {
        const double val = proj_data[((long)s * nv + j) * nu + i];
        joseph_ray_t r;
        if (!joseph_ray(vol, &jp, i + proj->index[0], j + proj->index[1], proj->index[2] + s, 0, &r))
          continue;
        const int    dz = (r.np_main > r.fp_main) ? -1 : 1;
        long         o[4];
        double       w[4];
        int          sl = r.ns;
        double       x = r.curx, y = r.cury;
        const double c = val * r.stepmm_norm;
        if (r.fs == r.ns)
        {
          joseph_taps(vol, &r, sl, x, y, 1, o, w);
          const double f = c * fabs(r.fp_main - r.np_main);
          for (int q = 0; q < 4; q++)
            vol_out[o[q]] += f * w[q];
        }
        else
        {
          joseph_taps(vol, &r, sl, x, y, 1, o, w);
          double f = c * (r.residualB + 0.5);
          for (int q = 0; q < 4; q++)
            vol_out[o[q]] += f * w[q];
          sl += dz;
          x += r.stepx;
          y += r.stepy;
          const int nmid = abs(r.fs - r.ns) - 1;
          for (int t = 0; t < nmid; t++)
          {
            joseph_taps(vol, &r, sl, x, y, 0, o, w);
            for (int q = 0; q < 4; q++)
              vol_out[o[q]] += c * w[q];
            sl += dz;
            x += r.stepx;
            y += r.stepy;
          }
          joseph_taps(vol, &r, sl, x, y, 1, o, w);
          f = c * (r.residualE + 0.5);
          for (int q = 0; q < 4; q++)
            vol_out[o[q]] += f * w[q];
        }
      }
  }
}

void
orc_joseph_back(const orc_geometry * g, const orc_image * vol, const double * vol_in, double * vol_out,
                const orc_image * proj, const double * proj_data)
{
  /* JosephBackProjectionImageFilter::GenerateData,
   * include/rtkJosephBackProjectionImageFilter.hxx:57-323 (single-threaded) */
  if (vol_out != vol_in)
    memcpy(vol_out, vol_in, sizeof(double) * npix(vol));
  joseph_back_slices(g, vol, vol_out, proj, proj_data, 0, proj->size[2]);
}

void
orc_joseph_back_mt(const orc_geometry * g, const orc_image * vol, const double * vol_in, double * vol_out,
                   const orc_image * proj, const double * proj_data, int nthreads)
{
  /* the same sum split over threads by projection, each into its own FP64
   * volume, added together at the end (RTK's filter is single-threaded; only
   * the FP64 summation order differs) */
  const long nvx = npix(vol);
  const int  np = proj->size[2];
  if (vol_out != vol_in)
    memcpy(vol_out, vol_in, sizeof(double) * nvx);
  if (nthreads > np)
    nthreads = np;
  if (nthreads <= 1)
  {
    joseph_back_slices(g, vol, vol_out, proj, proj_data, 0, np);
    return;
  }
  double ** part = (double **)calloc(nthreads, sizeof(double *));
#pragma omp parallel num_threads(nthreads)
  {
#ifdef _OPENMP
    const int t = omp_get_thread_num(), nt = omp_get_num_threads();
#else
    const int t = 0, nt = 1;
#endif
    double * acc = (double *)calloc(nvx, sizeof(double));
    part[t] = acc;
    joseph_back_slices(g, vol, acc, proj, proj_data, (int)((long)np * t / nt), (int)((long)np * (t + 1) / nt));
  }
#pragma omp parallel for num_threads(nthreads) schedule(static)
  for (long q = 0; q < nvx; q++)
  {
    double v = vol_out[q];
    for (int t = 0; t < nthreads; t++)
      if (part[t])
        v += part[t][q];
    vol_out[q] = v;
  }
  for (int t = 0; t < nthreads; t++)
    free(part[t]);
  free(part);
}

double
orc_joseph_sample_count(const orc_geometry * g, const orc_image * vol, const orc_image * proj, int nthreads)
{
  const int nu = proj->size[0], nv = proj->size[1], np = proj->size[2];
  double    total = 0.;
  for (int s = 0; s < np; s++)
  {
    joseph_proj_t jp;
    joseph_setup(g, vol, proj, proj->index[2] + s, &jp);
    double acc = 0.;
#pragma omp parallel for num_threads(nthreads) reduction(+ : acc) schedule(dynamic, 4)
    for (int j = 0; j < nv; j++)
      for (int i = 0; i < nu; i++)
      {
        joseph_ray_t r;
        if (joseph_ray(vol, &jp, i + proj->index[0], j + proj->index[1], proj->index[2] + s, 1, &r))
          acc += (r.fs == r.ns) ? 1. : (double)(abs(r.fs - r.ns) + 1);
      }
    total += acc;
  }
  return total;
}

/* ------------------------------------------------------------------------ */
/* FDK weighting (include/rtkFDKWeightProjectionFilter.hxx:40-128)            */
/* ------------------------------------------------------------------------ */
void
orc_fdk_weight(const orc_geometry * g, const orc_image * proj, const double * in, double * out)
{
  const int n = g->n;
  double *  sang = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
  double *  fac = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
  double *  tilt = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
  orc_geometry_source_angles(g, sang);
  orc_geometry_angular_gaps(g, sang, fac);
  orc_geometry_tilt_angles(g, tilt);
  for (int k = 0; k < n; k++)
  {
    const double sdd = g->par[10 * k + P_SDD];
    if (sdd == 0.)
      fac[k] *= 0.5;
    else
    {
      double sp[4];
      orc_geometry_source_position(g, k, sp);
      const double sid = g->par[10 * k + P_SID];
      fac[k] *= fabs(sdd) / (2. * sid * sid);
      fac[k] *= sqrt(sp[0] * sp[0] + sp[1] * sp[1] + sp[2] * sp[2]);
    }
  }
  /* point base and increment from TransformIndexToPhysicalPoint */
  double i2p[16], base[3], inc[3];
  orc_index_to_physical(proj, i2p);
  for (int a = 0; a < 3; a++)
  {
    base[a] = i2p[a * 4 + 3] + i2p[a * 4 + 0] * proj->index[0] + i2p[a * 4 + 1] * proj->index[1] +
              i2p[a * 4 + 2] * proj->index[2];
    inc[a] = i2p[a * 4 + 0] + i2p[a * 4 + 1] + i2p[a * 4 + 2];
  }
  const int nu = proj->size[0], nv = proj->size[1], np = proj->size[2];
  for (int s = 0; s < np; s++)
  {
    const int      k = proj->index[2] + s;
    const double * p = g->par + 10 * k;
    const double   sdd = p[P_SDD];
    const long     off = (long)s * nu * nv;
    if (sdd != 0.)
    {
      double       py = base[1] + p[P_POY] - p[P_SOY];
      const double cosa = cos(tilt[k]), sina = sin(tilt[k]), tana = tan(tilt[k]);
      const double sid = p[P_SID], sdd2 = sdd * sdd, RD = sdd - sid;
      const double numpart1 = sdd * (cosa + tana * sina);
      const double sddtana = sdd * tana;
      for (int j = 0; j < nv; j++, py += inc[1])
      {
        double       px = base[0] + p[P_POX] + tana * RD;
        const double sdd2y2 = sdd2 + py * py;
        for (int i = 0; i < nu; i++, px += inc[0])
        {
          const double denom = sqrt(sdd2y2 + pow(px - sddtana, 2.));
          const double cosGamma = (numpart1 - px * sina) / denom;
          out[off + (long)j * nu + i] = in[off + (long)j * nu + i] * fac[k] * cosGamma;
        }
      }
    }
    else
      for (long q = 0; q < (long)nu * nv; q++)
        out[off + q] = in[off + q] * fac[k];
  }
  free(sang);
  free(fac);
  free(tilt);
}

/* ------------------------------------------------------------------------ */
/* Parker short scan (include/rtkParkerShortScanImageFilter.hxx:41-209)      */
/* ------------------------------------------------------------------------ */

/* ParkerShortScanImageFilter::GenerateInputRequestedRegion's short-scan
 * detection and angles (include/rtkParkerShortScanImageFilter.hxx:41-110):
 * returns 1 for a short scan (largest gap between consecutive gantry angles
 * above threshold, divergent geometry) with delta and the first angle. */
int
orc_parker_params(const orc_geometry * g, double threshold, double * delta_out, double * first_out)
{
  const int n = g->n;
  double *  ga = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
  double *  gaps = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
  orc_geometry_gantry_angles(g, ga);
  orc_geometry_angular_gaps_with_next(g, ga, gaps);
  int maxpos = 0;
  for (int k = 1; k < n; k++)
    if (gaps[k] > gaps[maxpos])
      maxpos = k;
  if (n < 1 || g->par[P_SDD] == 0. || gaps[maxpos] < threshold)
  {
    free(ga);
    free(gaps);
    return 0;
  }
  angle_idx * s = sorted_angles(ga, n);
  int         nu_ = 0;
  for (int k = 0; k < n; k++)
    if (nu_ == 0 || s[k].a != s[nu_ - 1].a)
      s[nu_++] = s[k];
  int last = 0;
  for (int k = 0; k < nu_; k++)
    if (s[k].a == ga[maxpos])
      last = k;
  const int first = (last + 1 == nu_) ? 0 : last + 1;
  double    firstAngle = s[first].a, lastAngle = s[last].a;
  if (lastAngle < firstAngle)
    lastAngle += 2 * ORC_PI;
  double delta = 0.5 * (lastAngle - firstAngle - ORC_PI);
  delta = delta - 2 * ORC_PI * floor(delta / (2 * ORC_PI));
  free(s);
  free(ga);
  free(gaps);
  *delta_out = delta;
  *first_out = firstAngle;
  return 1;
}

int
orc_parker_weight(const orc_geometry * g, const orc_image * proj, double threshold, const double * in, double * out)
{
  const int  n = g->n;
  const int  nu = proj->size[0], nv = proj->size[1], np = proj->size[2];
  const long tot = npix(proj);
  double *   ga = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
  double *   gaps = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
  orc_geometry_gantry_angles(g, ga);
  orc_geometry_angular_gaps_with_next(g, ga, gaps);
  int maxpos = 0;
  for (int k = 1; k < n; k++)
    if (gaps[k] > gaps[maxpos])
      maxpos = k;
  if (n < 1 || g->par[P_SDD] == 0. || gaps[maxpos] < threshold)
  {
    if (out != in)
      memcpy(out, in, sizeof(double) * tot);
    free(ga);
    free(gaps);
    return 0;
  }
  /* unique sorted angles (std::map keeps the first inserted index) */
  angle_idx * s = sorted_angles(ga, n);
  int         nu_ = 0;
  for (int k = 0; k < n; k++)
    if (nu_ == 0 || s[k].a != s[nu_ - 1].a)
      s[nu_++] = s[k];
  int last = 0;
  for (int k = 0; k < nu_; k++)
    if (s[k].a == ga[maxpos])
      last = k;
  const int first = (last + 1 == nu_) ? 0 : last + 1;
  double    firstAngle = s[first].a, lastAngle = s[last].a;
  if (lastAngle < firstAngle)
    lastAngle += 2 * ORC_PI;
  double delta = 0.5 * (lastAngle - firstAngle - ORC_PI);
  delta = delta - 2 * ORC_PI * floor(delta / (2 * ORC_PI));
  free(s);

  for (int sl = 0; sl < np; sl++)
  {
    const int      k = proj->index[2] + sl;
    const double * p = g->par + 10 * k;
    const double   sox = p[P_SOX], sid = p[P_SID];
    const double   invsid = 1. / sqrt(sid * sid + sox * sox);
    double         beta = ga[k] - firstAngle;
    if (beta < 0)
      beta += 2 * ORC_PI;
    for (int i = 0; i < nu; i++)
    {
      const double x = proj->origin[0] + proj->spacing[0] * (proj->index[0] + i);
      const double l = orc_geometry_to_untilted(g, k, x);
      const double alpha = atan(-1 * l * invsid);
      double       w;
      if (beta <= 2 * delta - 2 * alpha)
        w = 2. * pow(sin((ORC_PI * beta) / (4 * (delta - alpha))), 2.);
      else if (beta <= ORC_PI - 2 * alpha)
        w = 2.;
      else if (beta <= ORC_PI + 2 * delta)
        w = 2. * pow(sin((ORC_PI * (ORC_PI + 2 * delta - beta)) / (4 * (delta + alpha))), 2.);
      else
        w = 0.;
      for (int j = 0; j < nv; j++)
      {
        const long o = ((long)sl * nv + j) * nu + i;
        out[o] = in[o] * w;
      }
    }
  }
  free(ga);
  free(gaps);
  return 1;
}

/* ------------------------------------------------------------------------ */
/* displaced detector (include/rtkDisplacedDetectorImageFilter.hxx:83-323)   */
/* ------------------------------------------------------------------------ */
int
orc_displaced_detector_region(const orc_geometry * g, const orc_image * proj, int pad, int * out_index0,
                              int * out_size0, double * inf_corner, double * sup_corner)
{
  double i2p[16];
  orc_index_to_physical(proj, i2p);
  double inf = i2p[3] + i2p[0] * proj->index[0] + i2p[1] * proj->index[1] + i2p[2] * proj->index[2];
  double sup = inf;
  if (proj->spacing[0] < 0.)
    inf += proj->spacing[0] * (proj->size[0] - 1);
  else
    sup += proj->spacing[0] * (proj->size[0] - 1);
  double maxInf = -DBL_MAX, minSup = DBL_MAX;
  for (int i = 0; i < g->n; i++)
  {
    const double a = orc_geometry_to_untilted(g, i, inf), b = orc_geometry_to_untilted(g, i, sup);
    if (a > maxInf)
      maxInf = a;
    if (b < minSup)
      minSup = b;
  }
  inf = maxInf;
  sup = minSup;
  *inf_corner = inf;
  *sup_corner = sup;
  *out_index0 = proj->index[0];
  *out_size0 = proj->size[0];
  if (inf > 0. || sup < 0.)
    return -1;
  if (fabs(inf + sup) < 0.1 * fabs(sup - inf))
    return 0;
  if (!pad)
    return 1;
  if (sup + inf > 0.)
    *out_index0 = proj->index[0] - proj->size[0];
  *out_size0 = 2 * proj->size[0];
  return 1;
}

int
orc_displaced_detector(const orc_geometry * g, const orc_image * proj, int pad, const double * in, double * out)
{
  int    oi0, os0;
  double inf, sup;
  int    st = orc_displaced_detector_region(g, proj, pad, &oi0, &os0, &inf, &sup);
  if (st < 0)
    return st;
  const int nu = proj->size[0], nv = proj->size[1], np = proj->size[2];
  if (st == 0)
  {
    memcpy(out, in, sizeof(double) * npix(proj));
    return 0;
  }
  const double theta = (-inf < sup) ? -inf : sup;
  const int    shift = proj->index[0] - oi0;
  double *     w = (double *)malloc(sizeof(double) * nu);
  for (int sl = 0; sl < np; sl++)
  {
    const int      k = proj->index[2] + sl;
    const double * p = g->par + 10 * k;
    const double   sx = p[P_SOX];
    double         sid = p[P_SID];
    sid = sqrt(sid * sid + sx * sx);
    double invsid = 0., invden = 0.;
    if (sid != 0.)
    {
      invsid = 1. / sid;
      invden = 1. / (2. * atan(theta * invsid));
    }
    for (int i = 0; i < nu; i++)
    {
      const double x = proj->origin[0] + proj->spacing[0] * (proj->index[0] + i);
      const double l = orc_geometry_to_untilted(g, k, x);
      if (sup + inf > 0.)
        w[i] = (l <= -theta) ? 0. : (l >= theta ? 2. : sin(ORC_PI * atan(l * invsid) * invden) + 1);
      else
        w[i] = (l <= -theta) ? 2. : (l >= theta ? 0. : 1 - sin(ORC_PI * atan(l * invsid) * invden));
    }
    for (int j = 0; j < nv; j++)
    {
      double *       orow = out + ((long)sl * nv + j) * os0;
      const double * irow = in + ((long)sl * nv + j) * nu;
      for (int i = 0; i < os0; i++)
        orow[i] = 0.;
      for (int i = 0; i < nu; i++)
        orow[shift + i] = irow[i] * w[i];
    }
  }
  free(w);
  return 1;
}

/* ------------------------------------------------------------------------ */
/* ramp filter                                                              */
/* ------------------------------------------------------------------------ */
static int
is_prime(int n)
{
  int last = (int)sqrt((double)n);
  for (int x = 2; x <= last; x++)
    if (n % x == 0)
      return 0;
  return 1;
}

static int
greatest_prime_factor(int n)
{
  /* FFTProjectionsConvolutionImageFilter::GreatestPrimeFactor, :322-333 */
  int v = 2;
  while (v <= n)
    if (n % v == 0 && is_prime(v))
      n /= v;
    else
      v += 1;
  return v;
}

int
orc_ramp_padded_size(int nu, const orc_ramp_params * p)
{
  /* GetPaddedImageRegion, include/rtkFFTProjectionsConvolutionImageFilter.hxx:280-306 */
  int x = p->zero_pad_factor * nu;
  while (greatest_prime_factor(x) > p->greatest_prime_factor)
    x++;
  return x;
}

int
orc_ramp_padded_size_y(int nv, const orc_ramp_params * p)
{
  /* GetPaddedImageRegion :296-301: padding along y only with the 2-D kernel
   * (HannCutFrequencyY > 0, FFTRampImageFilter::GenerateInputRequestedRegion
   * :41); ZeroPadFactors[1] is clamped to [1, 2] (header :108-111), default 2 */
  if (!(p->hann_cut_y > 0.))
    return nv;
  int zy = p->zero_pad_factor_y <= 0 ? 2 : (p->zero_pad_factor_y > 2 ? 2 : p->zero_pad_factor_y);
  int y = zy * nv;
  while (greatest_prime_factor(y) > p->greatest_prime_factor)
    y++;
  return y;
}

void
orc_ramp_window_y(int padded_y, const orc_ramp_params * p, double * w)
{
  /* UpdateFFTProjectionsConvolutionKernel :141-177: kernel rows j < ncut and
   * padded_y - j (1 <= j < ncut) are the 1-D kernel times the Hann window
   * 0.5 (1 + cos(pi j / ncut)), ncut = round((padded_y / 2 + 1) min(1, fy));
   * the other rows are zero */
  const int half = padded_y / 2;
  for (int j = 0; j <= half; j++)
    w[j] = 0.;
  if (!(p->hann_cut_y > 0.))
    return;
  const int ncut = (int)floor((half + 1) * fmin(1.0, p->hann_cut_y) + 0.5);
  for (int j = 0; j < ncut && j <= half; j++)
    w[j] = 0.5 * (1 + cos(ORC_PI * j / ncut));
}

/* complex DFT of length n in place (radix-2 when n is a power of two,
 * direct O(n^2) otherwise); sign -1 forward, +1 inverse (unscaled) */
static void
dft(double * re, double * im, int n, int sign)
{
  if ((n & (n - 1)) == 0)
  {
    for (int i = 1, j = 0; i < n; i++)
    {
      int bit = n >> 1;
      for (; j & bit; bit >>= 1)
        j ^= bit;
      j ^= bit;
      if (i < j)
      {
        double t = re[i];
        re[i] = re[j];
        re[j] = t;
        t = im[i];
        im[i] = im[j];
        im[j] = t;
      }
    }
    for (int len = 2; len <= n; len <<= 1)
    {
      const double ang = sign * 2 * ORC_PI / len;
      for (int i = 0; i < n; i += len)
        for (int k = 0; k < len / 2; k++)
        {
          const double wr = cos(ang * k), wi = sin(ang * k);
          const int    a = i + k, b = i + k + len / 2;
          const double xr = re[b] * wr - im[b] * wi, xi = re[b] * wi + im[b] * wr;
          re[b] = re[a] - xr;
          im[b] = im[a] - xi;
          re[a] += xr;
          im[a] += xi;
        }
    }
    return;
  }
  double * tr = (double *)malloc(sizeof(double) * n);
  double * ti = (double *)malloc(sizeof(double) * n);
  for (int k = 0; k < n; k++)
  {
    double sr = 0., si = 0.;
    for (int t = 0; t < n; t++)
    {
      const double a = sign * 2 * ORC_PI * (double)(((long)k * t) % n) / n;
      sr += re[t] * cos(a) - im[t] * sin(a);
      si += re[t] * sin(a) + im[t] * cos(a);
    }
    tr[k] = sr;
    ti[k] = si;
  }
  memcpy(re, tr, sizeof(double) * n);
  memcpy(im, ti, sizeof(double) * n);
  free(tr);
  free(ti);
}

void
orc_ramp_kernel(int padded, double spacing, const orc_ramp_params * p, double * kernel)
{
  /* FFTRampImageFilter::UpdateFFTProjectionsConvolutionKernel,
   * include/rtkFFTRampImageFilter.hxx:47-178 (1-D kernel) */
  double * re = (double *)calloc(padded, sizeof(double));
  double * im = (double *)calloc(padded, sizeof(double));
  re[0] = 1. / (4. * spacing);
  for (int ix = 1, jx = padded - 1; ix < padded / 2; ix += 2, jx -= 2)
  {
    double v = ix * ORC_PI;
    v = -1. / (v * v * spacing);
    re[ix] = v;
    re[jx] = v;
  }
  dft(re, im, padded, -1);
  const int n = padded / 2 + 1;
  for (int i = 0; i < n; i++)
    kernel[i] = re[i];
  int start_zero = n; /* index from which the kernel is zeroed */
  if (p->hann_cut > 0.)
  {
    const int ncut = (int)floor(n * fmin(1.0, p->hann_cut) + 0.5);
    for (int i = 0; i < ncut; i++)
      kernel[i] *= 0.5 * (1 + cos(ORC_PI * i / ncut));
    start_zero = ncut;
  }
  else if (p->cosine_cut > 0.)
  {
    const int ncut = (int)floor(n * fmin(1.0, p->cosine_cut) + 0.5);
    for (int i = 0; i < ncut; i++)
      kernel[i] *= cos(0.5 * ORC_PI * i / ncut);
    start_zero = ncut;
  }
  else if (p->hamming > 0.)
  {
    const int ncut = (int)floor(n * fmin(1.0, p->hamming) + 0.5);
    for (int i = 0; i < ncut; i++)
      kernel[i] *= 0.54 + 0.46 * cos(ORC_PI * i / ncut);
    start_zero = ncut;
  }
  else if (p->ramlak_cut > 0.)
  {
    start_zero = (int)floor(n * fmin(1.0, p->ramlak_cut) + 0.5);
  }
  else if (p->shepplogan_cut > 0.)
  {
    const int ncut = (int)floor(n * fmin(1.0, p->shepplogan_cut) + 0.5);
    for (int i = 1; i < ncut; i++)
    {
      const double x = 0.5 * ORC_PI * i / ncut;
      kernel[i] *= sin(x) / x;
    }
    start_zero = ncut < 1 ? 1 : ncut;
  }
  for (int i = start_zero; i < n; i++)
    kernel[i] = 0.;
  free(re);
  free(im);
}

void
orc_ramp_filter(const orc_image * proj, const orc_ramp_params * p, const double * in, double * out, int nthreads)
{
  /* FFTProjectionsConvolutionImageFilter::ThreadedGenerateData and
   * PadInputImageRegion, include/rtkFFTProjectionsConvolutionImageFilter.hxx:121-276 */
  const int nu = proj->size[0], nv = proj->size[1], np = proj->size[2];
  const int padded = orc_ramp_padded_size(nu, p);
  const int zeroext = (padded - nu) / 2;
  /* the weights follow the full extent floor(t * nu)
   * (UpdateTruncationMirrorWeights :345-355, GetTruncationCorrectionExtent
   * :78-81); the mirror covers at most the zero padding (:215-216) */
  const int extent = (int)floor(p->truncation_correction * nu);
  const int next = extent < zeroext ? extent : zeroext;
  double *  mw = (double *)malloc(sizeof(double) * (extent + 1));
  for (int i = 0; i < extent + 1; i++)
    mw[i] = pow(sin((extent - i) * ORC_PI / (2 * extent - 2)), 0.75);
  double * K = (double *)malloc(sizeof(double) * (padded / 2 + 1));
  orc_ramp_kernel(padded, proj->spacing[0], p, K);
  if (p->hann_cut_y > 0.)
  {
    /* 2-D kernel: per projection, the padded image (rows 0..nv-1 at their own
     * index, x as for the 1-D kernel, zero rows up to the padded height)
     * through a 2-D DFT, times K2[j][f] = wy[min(j, H - j)] K[min(f, N - f)],
     * the inverse 2-D DFT and the crop (ThreadedGenerateData :121-198 with
     * one projection per region, GetPaddedImageRegion :280-306) */
    const int H = orc_ramp_padded_size_y(nv, p);
    double *  wy = (double *)malloc(sizeof(double) * (H / 2 + 1));
    orc_ramp_window_y(H, p, wy);
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
    for (int s = 0; s < np; s++)
    {
      double * re = (double *)calloc((size_t)H * padded, sizeof(double));
      double * im = (double *)calloc((size_t)H * padded, sizeof(double));
      double * cr = (double *)malloc(sizeof(double) * H);
      double * ci = (double *)malloc(sizeof(double) * H);
      for (int r = 0; r < nv; r++)
      {
        const double * x = in + ((long)s * nv + r) * nu;
        double *       rr = re + (size_t)r * padded;
        for (int i = 0; i < nu; i++)
          rr[zeroext + i] = x[i];
        if (next)
        {
          const double SA = x[1], SE = x[nu - 1];
          for (int b = 1; b <= next; b++)
          {
            rr[zeroext - b] = mw[b] * (2.0 * SA - x[b]);
            rr[zeroext + nu - 1 + b] = mw[b] * (2.0 * SE - x[nu - 1 - b]);
          }
        }
        dft(rr, im + (size_t)r * padded, padded, -1);
      }
      for (int f = 0; f < padded; f++)
      {
        const double kf = K[f <= padded / 2 ? f : padded - f];
        for (int j = 0; j < H; j++)
        {
          cr[j] = re[(size_t)j * padded + f];
          ci[j] = im[(size_t)j * padded + f];
        }
        dft(cr, ci, H, -1);
        for (int j = 0; j < H; j++)
        {
          const double k = kf * wy[j <= H / 2 ? j : H - j];
          cr[j] *= k;
          ci[j] *= k;
        }
        dft(cr, ci, H, +1);
        for (int j = 0; j < H; j++)
        {
          re[(size_t)j * padded + f] = cr[j];
          im[(size_t)j * padded + f] = ci[j];
        }
      }
      for (int r = 0; r < nv; r++)
      {
        double * rr = re + (size_t)r * padded;
        dft(rr, im + (size_t)r * padded, padded, +1);
        for (int i = 0; i < nu; i++)
          out[((long)s * nv + r) * nu + i] = rr[zeroext + i] / ((double)padded * H);
      }
      free(re);
      free(im);
      free(cr);
      free(ci);
    }
    free(wy);
    free(K);
    free(mw);
    return;
  }
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 8)
  for (long row = 0; row < (long)nv * np; row++)
  {
    double *       re = (double *)calloc(padded, sizeof(double));
    double *       im = (double *)calloc(padded, sizeof(double));
    const double * r = in + row * nu;
    /* padded buffer position q corresponds to input column q - zeroext */
    for (int i = 0; i < nu; i++)
      re[zeroext + i] = r[i];
    if (next)
    {
      const double SA = r[1];
      for (int b = 1; b <= next; b++)
        re[zeroext - b] = mw[b] * (2.0 * SA - r[b]);
      const double SE = r[nu - 1];
      for (int b = 1; b <= next; b++)
        re[zeroext + nu - 1 + b] = mw[b] * (2.0 * SE - r[nu - 1 - b]);
    }
    dft(re, im, padded, -1);
    for (int f = 0; f < padded; f++)
    {
      const int    ff = f <= padded / 2 ? f : padded - f;
      const double k = K[ff];
      re[f] *= k;
      im[f] *= k;
    }
    dft(re, im, padded, +1);
    for (int i = 0; i < nu; i++)
      out[row * nu + i] = re[zeroext + i] / padded;
    free(re);
    free(im);
  }
  free(K);
  free(mw);
}

/* ------------------------------------------------------------------------ */
/* conjugate gradient                                                       */
/* ------------------------------------------------------------------------ */
void
orc_laplacian(const orc_image * vol, const double * x, double * out)
{
  /* LaplacianImageFilter (include/rtkLaplacianImageFilter.hxx): the
   * backward-difference divergence (include/rtkBackwardDifferenceDivergenceImageFilter.hxx,
   * zero before the first index, the last gradient subtracted at the last
   * index) of the forward-difference gradient
   * (include/rtkForwardDifferenceGradientImageFilter.hxx, zero-flux Neumann
   * boundary), both scaled by 1/spacing: per axis, the sum over the existing
   * neighbours of (x_nb - x_i) / spacing^2. */
  const int nx = vol->size[0], ny = vol->size[1], nz = vol->size[2];
  const double w[3] = { 1. / (vol->spacing[0] * vol->spacing[0]), 1. / (vol->spacing[1] * vol->spacing[1]),
                        1. / (vol->spacing[2] * vol->spacing[2]) };
  const long st[3] = { 1, nx, (long)nx * ny };
  const int  n[3] = { nx, ny, nz };
  for (int z = 0; z < nz; z++)
    for (int y = 0; y < ny; y++)
      for (int xx = 0; xx < nx; xx++)
      {
        const long i = ((long)z * ny + y) * nx + xx;
        const int  c[3] = { xx, y, z };
        double     l = 0.;
        for (int a = 0; a < 3; a++)
        {
          if (c[a] + 1 < n[a])
            l += (x[i + st[a]] - x[i]) * w[a];
          if (c[a] > 0)
            l += (x[i - st[a]] - x[i]) * w[a];
        }
        out[i] = l;
      }
}

/* The CG's back projector (IterativeConeBeamReconstructionFilter's
 * InstantiateBackProjectionFilter, include/rtkIterativeConeBeamReconstructionFilter.hxx:33-103):
 * 0 Joseph (BP_JOSEPH), 1 voxel-based (BP_VOXELBASED, rtkconjugategradient's
 * default); out += BP(p). */
static void
cg_backproject(const orc_geometry * g, const orc_image * vol, const orc_image * proj, const double * p, double * out,
               int backprojector, int nthreads)
{
  if (backprojector == 1)
    orc_backproject(g, vol, proj, p, out, out, 0, nthreads);
  else
    orc_joseph_back_mt(g, vol, out, out, proj, p, nthreads);
}

static void
cg_apply_A(const orc_geometry * g, const orc_image * vol, const orc_image * proj, const double * weights,
           const double * mask, double tikhonov, double gamma, const double * x_in, double * out, double * ptmp,
           int backprojector, int nthreads)
{
  /* ReconstructionConjugateGradientOperator::GenerateData,
   * include/rtkReconstructionConjugateGradientOperator.hxx:192-311:
   * BP(W .* FP(x)), then + gamma * (-Laplacian(x)), then + tikhonov * x; with a
   * support mask M, x is M .* x_in and the result is multiplied by M */
  const long np = npix(proj), nvx = npix(vol);
  double *   xm = NULL;
  const double * x = x_in;
  if (mask)
  {
    xm = (double *)malloc(sizeof(double) * nvx);
    for (long q = 0; q < nvx; q++)
      xm[q] = mask[q] * x_in[q];
    x = xm;
  }
  memset(ptmp, 0, sizeof(double) * np);
  orc_joseph_forward(g, vol, x, proj, ptmp, ptmp, nthreads);
  if (weights)
    for (long q = 0; q < np; q++)
      ptmp[q] *= weights[q];
  memset(out, 0, sizeof(double) * nvx);
  cg_backproject(g, vol, proj, ptmp, out, backprojector, nthreads);
  if (gamma != 0.)
  {
    double * lap = (double *)malloc(sizeof(double) * nvx);
    orc_laplacian(vol, x, lap);
    for (long q = 0; q < nvx; q++)
      out[q] += -gamma * lap[q];
    free(lap);
  }
  if (tikhonov != 0.)
    for (long q = 0; q < nvx; q++)
      out[q] += tikhonov * x[q];
  if (mask)
  {
    for (long q = 0; q < nvx; q++)
      out[q] *= mask[q];
    free(xm);
  }
}

void
orc_cg(const orc_geometry * g, const orc_image * vol, const orc_image * proj, const double * proj_data,
       const double * weights, const double * mask, double tikhonov, double gamma, int niter, double * x,
       double * residuals, int backprojector, int nthreads)
{
  /* with a support mask M (ConjugateGradientConeBeamReconstructionFilter,
   * include/rtkConjugateGradientConeBeamReconstructionFilter.hxx:246-258): b is
   * multiplied by M, the operator masks its input and output, and the result
   * x is multiplied by M at the end */
  /* ConjugateGradientImageFilter::GenerateData,
   * include/rtkConjugateGradientImageFilter.hxx:108-258, with FP64
   * accumulators; b from ConjugateGradientConeBeamReconstructionFilter
   * (include/rtkConjugateGradientConeBeamReconstructionFilter.hxx:223-244) */
  const long np = npix(proj), nvx = npix(vol);
  double *   ptmp = (double *)malloc(sizeof(double) * np);
  double *   b = (double *)calloc(nvx, sizeof(double));
  double *   R = (double *)malloc(sizeof(double) * nvx);
  double *   P = (double *)malloc(sizeof(double) * nvx);
  double *   AP = (double *)malloc(sizeof(double) * nvx);
  for (long q = 0; q < np; q++)
    ptmp[q] = proj_data[q] * (weights ? weights[q] : 1.);
  cg_backproject(g, vol, proj, ptmp, b, backprojector, nthreads);
  if (mask)
    for (long q = 0; q < nvx; q++)
      b[q] *= mask[q];
  cg_apply_A(g, vol, proj, weights, mask, tikhonov, gamma, x, AP, ptmp, backprojector, nthreads);
  for (long q = 0; q < nvx; q++)
  {
    R[q] = b[q] - AP[q];
    P[q] = R[q];
  }
  const double eps = DBL_MIN;
  double       rr = 0.;
  for (long q = 0; q < nvx; q++)
    rr += R[q] * R[q];
  if (residuals)
    residuals[0] = rr;
  for (int it = 0; it < niter; it++)
  {
    cg_apply_A(g, vol, proj, weights, mask, tikhonov, gamma, P, AP, ptmp, backprojector, nthreads);
    double num = 0., den = 0.;
    for (long q = 0; q < nvx; q++)
    {
      num += R[q] * R[q];
      den += P[q] * AP[q];
    }
    const double alpha = num / (den + eps);
    for (long q = 0; q < nvx; q++)
      x[q] += alpha * P[q];
    den = num;
    num = 0.;
    for (long q = 0; q < nvx; q++)
    {
      R[q] -= alpha * AP[q];
      num += R[q] * R[q];
    }
    const double beta = num / (den + eps);
    for (long q = 0; q < nvx; q++)
      P[q] = R[q] + beta * P[q];
    if (residuals)
      residuals[it + 1] = num;
  }
  if (mask)
    for (long q = 0; q < nvx; q++)
      x[q] *= mask[q];
  free(ptmp);
  free(b);
  free(R);
  free(P);
  free(AP);
}

void
orc_cg_joseph(const orc_geometry * g, const orc_image * vol, const orc_image * proj, const double * proj_data,
              const double * weights, const double * mask, double tikhonov, double gamma, int niter, double * x,
              double * residuals, int nthreads)
{
  orc_cg(g, vol, proj, proj_data, weights, mask, tikhonov, gamma, niter, x, residuals, 0, nthreads);
}

/* ------------------------------------------------------------------------ */
/* phantoms                                                                 */
/* ------------------------------------------------------------------------ */
void
orc_project_ellipsoids(const orc_geometry * g, const orc_image * proj, int n_ell, const double * ell,
                       double * proj_out, int nthreads)
{
  /* analytic line integrals (RayConvexIntersectionImageFilter semantics,
   * include/rtkRayConvexIntersectionImageFilter.hxx:57-84): for every pixel,
   * sum over ellipsoids of density x chord length between source and pixel. */
  const int nu = proj->size[0], nv = proj->size[1], np = proj->size[2];
  double    pi2pp[16];
  orc_index_to_physical(proj, pi2pp);
  for (int s = 0; s < np; s++)
  {
    const int k = proj->index[2] + s;
    double    p2f[16], T[16], src[4], idx2det[16], inv[16];
    orc_geometry_proj_coords_to_fixed(g, k, p2f);
    mat_mul(p2f, pi2pp, T, 4, 4, 4);
    orc_geometry_source_position(g, k, src);
    if (g->radius_cyl != 0.)
      cyl_matrices(g, k, pi2pp, idx2det, inv);
    double s2p[3];
    const int parallel = parallel_source_to_pixel(g, k, s2p);
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 4)
    for (int j = 0; j < nv; j++)
      for (int i = 0; i < nu; i++)
      {
        const double ii = i + proj->index[0], jj = j + proj->index[1], kk = k;
        double       pix[3], d[3], srcp[3];
        if (g->radius_cyl != 0.)
          cyl_pixel(idx2det, inv, g->radius_cyl, ii, jj, kk, pix);
        else
          for (int a = 0; a < 3; a++)
            pix[a] = T[a * 4 + 0] * ii + T[a * 4 + 1] * jj + T[a * 4 + 2] * kk + T[a * 4 + 3];
        for (int a = 0; a < 3; a++)
        {
          srcp[a] = parallel ? pix[a] - s2p[a] : src[a];
          d[a] = pix[a] - srcp[a];
        }
        const double len = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        double       acc = 0.;
        for (int e = 0; e < n_ell; e++)
        {
          const double * E = ell + 16 * e;
          const double * R = E + 6;
          double         o[3], dd[3], rel[3] = { srcp[0] - E[0], srcp[1] - E[1], srcp[2] - E[2] };
          for (int a = 0; a < 3; a++)
          {
            /* local = R^T (world - c), scaled by 1/axis */
            o[a] = (R[0 * 3 + a] * rel[0] + R[1 * 3 + a] * rel[1] + R[2 * 3 + a] * rel[2]) / E[3 + a];
            dd[a] = (R[0 * 3 + a] * d[0] + R[1 * 3 + a] * d[1] + R[2 * 3 + a] * d[2]) / E[3 + a];
          }
          const double A = dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2];
          const double B = 2 * (o[0] * dd[0] + o[1] * dd[1] + o[2] * dd[2]);
          const double C = o[0] * o[0] + o[1] * o[1] + o[2] * o[2] - 1.;
          const double disc = B * B - 4 * A * C;
          if (disc <= 0.)
            continue;
          const double sq = sqrt(disc);
          double       t1 = (-B - sq) / (2 * A), t2 = (-B + sq) / (2 * A);
          if (t1 < 0.)
            t1 = 0.;
          if (t2 > 1.)
            t2 = 1.;
          if (t2 > t1)
            acc += E[15] * (t2 - t1) * len;
        }
        proj_out[((long)s * nv + j) * nu + i] = acc;
      }
  }
}

void
orc_draw_ellipsoids(const orc_image * vol, int n_ell, const double * ell, double * vol_out, int nthreads)
{
  /* voxelised reference (DrawConvexImageFilter semantics,
   * include/rtkDrawConvexImageFilter.hxx:54-57): density added where the voxel
   * centre is inside */
  const int nx = vol->size[0], ny = vol->size[1], nz = vol->size[2];
  double    i2p[16];
  orc_index_to_physical(vol, i2p);
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
      {
        const double x[3] = { i + vol->index[0], j + vol->index[1], k + vol->index[2] };
        double       w[3];
        for (int a = 0; a < 3; a++)
          w[a] = i2p[a * 4 + 0] * x[0] + i2p[a * 4 + 1] * x[1] + i2p[a * 4 + 2] * x[2] + i2p[a * 4 + 3];
        double acc = 0.;
        for (int e = 0; e < n_ell; e++)
        {
          const double * E = ell + 16 * e;
          const double * R = E + 6;
          const double   rel[3] = { w[0] - E[0], w[1] - E[1], w[2] - E[2] };
          double         q = 0.;
          for (int a = 0; a < 3; a++)
          {
            const double l = (R[0 * 3 + a] * rel[0] + R[1 * 3 + a] * rel[1] + R[2 * 3 + a] * rel[2]) / E[3 + a];
            q += l * l;
          }
          if (q <= 1.)
            acc += E[15];
        }
        vol_out[((long)k * ny + j) * nx + i] = acc;
      }
}

/* ------------------------------------------------------------------------ */
/* timed CPU baseline: RTK's CPU FDK backprojector with RTK's data types     */
/* ------------------------------------------------------------------------ */
int
orc_fdk_backproject_f32_rtk(const orc_geometry * g, const orc_image * vol, const orc_image * proj,
                            const float * proj_data, float * vol_inout, int nthreads)
{
  /* FDKBackProjectionImageFilter::DynamicThreadedGenerateData with
   * OptimizedBackprojectionY (include/rtkFDKBackProjectionImageFilter.hxx:52-148,
   * 232-306), BackProjectionImageFilter::GetProjection transposing each
   * projection per thread (include/rtkBackProjectionImageFilter.hxx:480-531).
   * Returns -1 when a projection would take another path. */
  const int nx = vol->size[0], ny = vol->size[1], nz = vol->size[2];
  const int nu = proj->size[0], nv = proj->size[1], np = proj->size[2];
  double *  mats = (double *)malloc(sizeof(double) * 12 * (np > 0 ? np : 1));
  for (int s = 0; s < np; s++)
    if (orc_bp_matrix(g, vol, proj, proj->index[2] + s, 1, mats + 12 * s) != 2)
    {
      free(mats);
      return -1;
    }
  int bad = 0;
#pragma omp parallel num_threads(nthreads)
  {
    int tid = 0, nt = 1;
#ifdef _OPENMP
    tid = omp_get_thread_num();
    nt = omp_get_num_threads();
#endif
    const int k0 = (int)((long)nz * tid / nt), k1 = (int)((long)nz * (tid + 1) / nt);
    float *   tp = (float *)malloc(sizeof(float) * (long)nu * nv);
    if (!tp)
    {
#pragma omp atomic write
      bad = 1;
    }
    else
    {
      for (int s = 0; s < np; s++)
      {
        /* transposed copy: tp[u][v] */
        const float * pin = proj_data + (long)s * nu * nv;
        for (int v = 0; v < nv; v++)
          for (int u = 0; u < nu; u++)
            tp[(long)u * nv + v] = pin[(long)v * nu + u];
        /* transposed matrix: row0 = v-row, row1 = u-row */
        const double * m = mats + 12 * s;
        const double   t00 = m[4], t01 = m[5], t02 = m[6], t03 = m[7];
        const double   t10 = m[0], t12 = m[2], t13 = m[3];
        const double   t20 = m[8], t22 = m[10], t23 = m[11];
        const int      psz0 = nv, psz1 = nu; /* transposed sizes */
        const double   pidx0 = proj->index[1], pidx1 = proj->index[0];
        for (int k = k0; k < k1; k++)
        {
          const int kk = k + vol->index[2];
          for (int i = 0; i < nx; i++)
          {
            const int ii = i + vol->index[0];
            int       jj = vol->index[1];
            double    u = t00 * ii + t01 * jj + t02 * kk + t03;
            double    v = t10 * ii + t12 * kk + t13;
            double    w = t20 * ii + t22 * kk + t23;
            w = 1 / w;
            u = u * w - pidx0;
            v = v * w - pidx1;
            const double du = w * t01;
            w *= w;
            const int vi = (int)floor(v);
            if (vi >= 0 && vi < psz1 - 1)
            {
              float * pv = vol_inout + ((long)k * ny) * nx + i;
              for (int j = 0; j < ny; j++, pv += nx, u += du)
              {
                const int ui = (int)floor(u);
                if (ui >= 0 && ui < psz0 - 1)
                {
                  const float * pp = tp + (long)vi * psz0 + ui;
                  const double  v1 = v - vi, v2 = 1.0 - v1, u1 = u - ui, u2 = 1.0 - u1;
                  *pv += w * (v2 * (u2 * pp[0] + u1 * pp[1]) + v1 * (u2 * pp[psz0] + u1 * pp[psz0 + 1]));
                }
              }
            }
          }
        }
      }
      free(tp);
    }
  }
  free(mats);
  return bad ? -2 : 0;
}

/* ------------------------------------------------------------------------ */
/* SART: SARTConeBeamReconstructionFilter (include/rtkSARTConeBeamReconstructionFilter.hxx) */

static void
ray_box_impl(const orc_geometry * g, const orc_image * proj, const double * D, const double * mn, const double * mx,
             double * out, int nthreads)
{
  const int nu = proj->size[0], nv = proj->size[1], np = proj->size[2];
  double pi2pp[16];
  orc_index_to_physical(proj, pi2pp);
  for (int s = 0; s < np; s++)
  {
    const int k = proj->index[2] + s;
    double    p2f[16], T[16], src[4];
    orc_geometry_proj_coords_to_fixed(g, k, p2f);
    mat_mul(p2f, pi2pp, T, 4, 4, 4);
    orc_geometry_source_position(g, k, src);
    double    s2p[3];
    const int parallel = parallel_source_to_pixel(g, k, s2p);
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 4)
    for (int j = 0; j < nv; j++)
      for (int i = 0; i < nu; i++)
      {
        const double ii = i + proj->index[0], jj = j + proj->index[1], kk = k;
        double       d[3], srcp[3];
        for (int a = 0; a < 3; a++)
        {
          const double pix = T[a * 4 + 0] * ii + T[a * 4 + 1] * jj + T[a * 4 + 2] * kk + T[a * 4 + 3];
          srcp[a] = parallel ? pix - s2p[a] : src[a];
          d[a] = pix - srcp[a];
        }
        const double len = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        double       org[3], dir[3];
        for (int a = 0; a < 3; a++)
        {
          org[a] = D[0 * 3 + a] * srcp[0] + D[1 * 3 + a] * srcp[1] + D[2 * 3 + a] * srcp[2];
          dir[a] = (D[0 * 3 + a] * d[0] + D[1 * 3 + a] * d[1] + D[2 * 3 + a] * d[2]) / len;
        }
        double inf = -DBL_MAX, sup = DBL_MAX;
        int    hit = 1;
        for (int a = 0; a < 3 && hit; a++)
        {
          if (dir[a] == 0. && (org[a] < mn[a] || org[a] > mx[a]))
          {
            hit = 0;
            break;
          }
          const double inv = 1. / dir[a];
          double       t1 = (mn[a] - org[a]) * inv, t2 = (mx[a] - org[a]) * inv;
          if (t1 > t2)
          {
            const double t = t1;
            t1 = t2;
            t2 = t;
          }
          inf = fmax(t1, inf);
          sup = fmin(t2, sup);
          if (inf > sup || sup < 0.)
            hit = 0;
        }
        out[((long)s * nv + j) * nu + i] = hit ? sup - inf : 0.;
      }
  }
}

void
orc_ray_box(const orc_geometry * g, const orc_image * vol, const orc_image * proj, double * out, int nthreads)
{
  /* RayBoxIntersectionImageFilter: RayConvexIntersectionImageFilter
   * (include/rtkRayConvexIntersectionImageFilter.hxx:57-84) with density 1
   * and the BoxShape of BoxShape::SetBoxFromImage(volume, false)
   * (src/rtkBoxShape.cxx:141-160: from the origin to origin + D (spacing x
   * (size - 1))), intersected as BoxShape::IsIntersectedByRay
   * (src/rtkBoxShape.cxx:47-97) along the normalised source-to-pixel
   * direction: out = supDist - infDist in mm, 0 without intersection. */
  const double * D = vol->direction;
  double         bmin[3], bmax[3], ext[3];
  for (int a = 0; a < 3; a++)
    ext[a] = vol->spacing[a] * (vol->size[a] - 1);
  for (int r = 0; r < 3; r++)
  {
    bmin[r] = vol->origin[r];
    bmax[r] = vol->origin[r] + D[3 * r + 0] * ext[0] + D[3 * r + 1] * ext[1] + D[3 * r + 2] * ext[2];
  }
  double mn[3], mx[3];
  for (int a = 0; a < 3; a++) /* D^T applied to the corners */
  {
    mn[a] = D[0 * 3 + a] * bmin[0] + D[1 * 3 + a] * bmin[1] + D[2 * 3 + a] * bmin[2];
    mx[a] = D[0 * 3 + a] * bmax[0] + D[1 * 3 + a] * bmax[1] + D[2 * 3 + a] * bmax[2];
    if (mn[a] > mx[a])
    {
      const double t = mn[a];
      mn[a] = mx[a];
      mx[a] = t;
    }
  }
  ray_box_impl(g, proj, D, mn, mx, out, nthreads);
}

void
orc_ray_box_corners(const orc_geometry * g, const orc_image * proj, const double * bmin, const double * bmax,
                    double * out, int nthreads)
{
  /* RayBoxIntersectionImageFilter with SetBoxMin / SetBoxMax (identity direction) */
  static const double I[9] = { 1., 0., 0., 0., 1., 0., 0., 0., 1. };
  double              mn[3], mx[3];
  for (int a = 0; a < 3; a++)
  {
    mn[a] = bmin[a] < bmax[a] ? bmin[a] : bmax[a];
    mx[a] = bmin[a] < bmax[a] ? bmax[a] : bmin[a];
  }
  ray_box_impl(g, proj, I, mn, mx, out, nthreads);
}

void
orc_sart(const orc_geometry * g, const orc_image * vol, const orc_image * proj, const double * proj_data, double * x,
         int niter, double lambda, int positivity, int projections_per_subset, int displaced_detector,
         double threshold, const int * order, int nthreads)
{
  /* SARTConeBeamReconstructionFilter::GenerateData (include/rtkSARTConeBeamReconstructionFilter.hxx):
   * for each projection s in `order`: e = lambda (p_s - JosephFP_s(x)),
   * divided (or zeroed below threshold) by the ray-box length, displaced-
   * detector weighted (no padding), voxel-based back projected into B, and
   * ones back projected into N; after every `projections_per_subset`
   * projections (and after the last one) x += B / N (or 0 below threshold),
   * then x = max(x, 0) with positivity. */
  const long per = (long)proj->size[0] * proj->size[1], nvx = npix(vol);
  const int  np = proj->size[2];
  double *   rb = (double *)malloc(sizeof(double) * per * np);
  double *   fp = (double *)malloc(sizeof(double) * per);
  double *   e = (double *)malloc(sizeof(double) * per);
  double *   e2 = (double *)malloc(sizeof(double) * per);
  double *   ones = (double *)malloc(sizeof(double) * per);
  double *   B = (double *)calloc(nvx, sizeof(double));
  double *   N = (double *)calloc(nvx, sizeof(double));
  orc_ray_box(g, vol, proj, rb, nthreads);
  for (long q = 0; q < per; q++)
    ones[q] = 1.;
  for (int it = 0; it < niter; it++)
  {
    int count = 0;
    for (int i = 0; i < np; i++)
    {
      const int  s = order[i];
      orc_image  p1 = *proj;
      p1.size[2] = 1;
      p1.index[2] = proj->index[2] + s;
      memset(fp, 0, sizeof(double) * per);
      orc_joseph_forward(g, vol, x, &p1, fp, fp, nthreads);
      for (long q = 0; q < per; q++)
      {
        const double den = rb[(long)s * per + q];
        e[q] = den < threshold ? 0. : lambda * (proj_data[(long)s * per + q] - fp[q]) / den;
      }
      if (displaced_detector)
        orc_displaced_detector(g, &p1, 0, e, e2);
      else
        memcpy(e2, e, sizeof(double) * per);
      if (count == 0)
      {
        memset(B, 0, sizeof(double) * nvx);
        memset(N, 0, sizeof(double) * nvx);
      }
      orc_backproject(g, vol, &p1, e2, B, B, 0, nthreads);
      orc_backproject(g, vol, &p1, ones, N, N, 0, nthreads);
      if (++count == projections_per_subset || i == np - 1)
      {
        for (long v = 0; v < nvx; v++)
        {
          x[v] += N[v] < threshold ? 0. : B[v] / N[v];
          if (positivity && x[v] < 0.)
            x[v] = 0.;
        }
        count = 0;
      }
    }
  }
  free(rb);
  free(fp);
  free(e);
  free(e2);
  free(ones);
  free(B);
  free(N);
}

void
orc_de_pierro(const orc_image * vol, const double * xk, const double * update, const double * norm, double beta,
              double * out)
{
  /* DePierroRegularizationImageFilter (include/rtkDePierroRegularizationImageFilter.hxx:26-131):
   * K = 3x3x3 neighbourhood inner product with weight 3^3 - 1 = 26 at the
   * centre and 1 elsewhere, zero outside the image (ConstantBoundaryCondition);
   * A = norm - beta K(xk) (norm = 1 when absent); B = 4 * 2 * beta * 26 * update;
   * out = (A + sqrt(A^2 + B)) / 2. */
  const long nx = vol->size[0], ny = vol->size[1], nz = vol->size[2];
  for (long z = 0; z < nz; z++)
    for (long y = 0; y < ny; y++)
      for (long x = 0; x < nx; x++)
      {
        const long i = (z * ny + y) * nx + x;
        double     k = 0.;
        for (long dz = -1; dz <= 1; dz++)
          for (long dy = -1; dy <= 1; dy++)
            for (long dx = -1; dx <= 1; dx++)
            {
              const long zz = z + dz, yy = y + dy, xx = x + dx;
              if (zz < 0 || zz >= nz || yy < 0 || yy >= ny || xx < 0 || xx >= nx)
                continue;
              k += ((dx | dy | dz) == 0 ? 26. : 1.) * xk[(zz * ny + yy) * nx + xx];
            }
        const double a = (norm ? norm[i] : 1.) - beta * k;
        const double b = 4. * 2. * beta * 26. * update[i];
        out[i] = (a + sqrt(a * a + b)) / 2.;
      }
}

void
orc_osem(const orc_geometry * g, const orc_image * vol, const orc_image * proj, const double * proj_data, double * x,
         int niter, int projections_per_subset, double beta, int joseph_bp, const int * order, int nthreads)
{
  /* OSEMConeBeamReconstructionFilter::GenerateData
   * (include/rtkOSEMConeBeamReconstructionFilter.hxx:161-273): for each
   * projection s in `order`, r = p_s / JosephFP_s(x) (1 where
   * |FP| < 1e-5: DivideOrZeroOutImageFilter with constant 1), back projected
   * (voxel-based, or Joseph with joseph_bp) into B, ones back projected into N;
   * after every `projections_per_subset` projections (and after the last one)
   * M = B x, R = DePierro(x, M, N) and x = M / R (0 where |R| < 1e-5).  The
   * normalisation images are recomputed every iteration; storing them, as RTK
   * does by default, gives the same values. */
  const long per = (long)proj->size[0] * proj->size[1], nvx = npix(vol);
  const int  np = proj->size[2];
  double *   fp = (double *)malloc(sizeof(double) * per);
  double *   ones = (double *)malloc(sizeof(double) * per);
  double *   B = (double *)calloc(nvx, sizeof(double));
  double *   N = (double *)calloc(nvx, sizeof(double));
  double *   M = (double *)malloc(sizeof(double) * nvx);
  double *   R = (double *)malloc(sizeof(double) * nvx);
  for (long q = 0; q < per; q++)
    ones[q] = 1.;
  for (int it = 0; it < niter; it++)
  {
    int count = 0;
    for (int i = 0; i < np; i++)
    {
      const int s = order[i];
      orc_image p1 = *proj;
      p1.size[2] = 1;
      p1.index[2] = proj->index[2] + s;
      memset(fp, 0, sizeof(double) * per);
      orc_joseph_forward(g, vol, x, &p1, fp, fp, nthreads);
      for (long q = 0; q < per; q++)
        fp[q] = fabs(fp[q]) < 1e-5 ? 1. : proj_data[(long)s * per + q] / fp[q];
      if (count == 0)
      {
        memset(B, 0, sizeof(double) * nvx);
        memset(N, 0, sizeof(double) * nvx);
      }
      if (joseph_bp)
      {
        orc_joseph_back(g, vol, B, B, &p1, fp);
        orc_joseph_back(g, vol, N, N, &p1, ones);
      }
      else
      {
        orc_backproject(g, vol, &p1, fp, B, B, 0, nthreads);
        orc_backproject(g, vol, &p1, ones, N, N, 0, nthreads);
      }
      if (++count == projections_per_subset || i == np - 1)
      {
        for (long v = 0; v < nvx; v++)
          M[v] = B[v] * x[v];
        orc_de_pierro(vol, x, M, N, beta, R);
        for (long v = 0; v < nvx; v++)
          x[v] = fabs(R[v]) < 1e-5 ? 0. : M[v] / R[v];
        count = 0;
      }
    }
  }
  free(fp);
  free(ones);
  free(B);
  free(N);
  free(M);
  free(R);
}

/* ------------------------------------------------------------------------ */
/* total variation and the regularised conjugate gradient                   */
/* ------------------------------------------------------------------------ */
static double
tv_div(const orc_image * vol, const double * z, const int * dk, int nd, long x, long y, long zz)
{
  /* BackwardDifferenceDivergenceImageFilter::DynamicThreadedGenerateData
   * (include/rtkBackwardDifferenceDivergenceImageFilter.hxx): per processed
   * dimension (packed component j, dimension dk[j]), (z_j(i) - z_j(i - e))/s
   * with zero outside (ConstantBoundaryCondition); AfterThreadedGenerateData
   * then subtracts z_j(i)/s on the last slice along dk[j] -- for the single
   * voxel at which its iterators start (all other coordinates 0), as coded. */
  const long n[3] = { vol->size[0], vol->size[1], vol->size[2] }, c[3] = { x, y, zz };
  const long nvx = n[0] * n[1] * n[2], i = (zz * n[1] + y) * n[0] + x;
  const long stride[3] = { 1, n[0], n[0] * n[1] };
  double     div = 0.;
  for (int j = 0; j < nd; j++)
  {
    const int    k = dk[j];
    const double inv = 1. / vol->spacing[k];
    const double here = z[(long)j * nvx + i];
    const double prev = c[k] > 0 ? z[(long)j * nvx + i - stride[k]] : 0.;
    div += (here - prev) * inv;
  }
  for (int j = 0; j < nd; j++)
  {
    const int k = dk[j];
    int       first = 1;
    for (int d = 0; d < 3; d++)
      if (d != k && c[d] != 0)
        first = 0;
    if (first && c[k] == n[k] - 1)
      div -= z[(long)j * nvx + i] / vol->spacing[k];
  }
  return div;
}

static void
tv_grad_threshold(const orc_image * vol, const double * w, double * z, const int * dk, int nd, double gamma,
                  int subtract)
{
  /* z_j = P_gamma(z_j - grad_j w) (subtract) or P_gamma(grad_j w): the
   * forward-difference gradient with a zero-flux Neumann boundary
   * (ForwardDifferenceGradientImageFilter, spacing-scaled) and
   * MagnitudeThresholdImageFilter (vectors longer than gamma scaled back to
   * gamma, others unchanged) */
  const long n[3] = { vol->size[0], vol->size[1], vol->size[2] };
  const long nvx = n[0] * n[1] * n[2], stride[3] = { 1, n[0], n[0] * n[1] };
  for (long zz = 0; zz < n[2]; zz++)
    for (long y = 0; y < n[1]; y++)
      for (long x = 0; x < n[0]; x++)
      {
        const long c[3] = { x, y, zz }, i = (zz * n[1] + y) * n[0] + x;
        double     v[3] = { 0., 0., 0. }, nn = 0.;
        for (int j = 0; j < nd; j++)
        {
          const int    k = dk[j];
          const double g = c[k] < n[k] - 1 ? (w[i + stride[k]] - w[i]) / vol->spacing[k] : 0.;
          v[j] = subtract ? z[(long)j * nvx + i] - g : g;
          nn += v[j] * v[j];
        }
        nn = sqrt(nn);
        for (int j = 0; j < nd; j++)
          z[(long)j * nvx + i] = nn > gamma ? gamma * v[j] / nn : v[j];
      }
}

void
orc_tv_denoising_bpdq(const orc_image * vol, const double * f, double * out, double gamma, int niter,
                      const int dims[3])
{
  /* TotalVariationDenoisingBPDQImageFilter / DenoisingBPDQImageFilter
   * (include/rtkDenoisingBPDQImageFilter.hxx:60-148): beta = 0.9 minSpacing
   * / 2^d (d processed dimensions; minSpacing starts from spacing[0], then the
   * minimum over the processed ones); iteration 0: z = P(grad(beta f));
   * iterations 1..niter-1: z = P(z - grad(beta minSpacing (f - div z)));
   * out = f - div z. */
  const long nvx = npix(vol);
  int        dk[3], nd = 0;
  double     minsp = vol->spacing[0];
  for (int d = 0; d < 3; d++)
    if (dims[d])
    {
      dk[nd++] = d;
      if (vol->spacing[d] < minsp)
        minsp = vol->spacing[d];
    }
  const double beta = 1. / pow(2., nd) * 0.9 * minsp;
  double *     z = (double *)calloc((size_t)(nd > 0 ? nd : 1) * nvx, sizeof(double));
  double *     w = (double *)malloc(sizeof(double) * nvx);
  for (long i = 0; i < nvx; i++)
    w[i] = beta * f[i];
  tv_grad_threshold(vol, w, z, dk, nd, gamma, 0);
  const long n0 = vol->size[0], n1 = vol->size[1], n2 = vol->size[2];
  for (int it = 1; it < niter; it++)
  {
    for (long zz = 0; zz < n2; zz++)
      for (long y = 0; y < n1; y++)
        for (long x = 0; x < n0; x++)
        {
          const long i = (zz * n1 + y) * n0 + x;
          w[i] = beta * minsp * (f[i] - tv_div(vol, z, dk, nd, x, y, zz));
        }
    tv_grad_threshold(vol, w, z, dk, nd, gamma, 1);
  }
  for (long zz = 0; zz < n2; zz++)
    for (long y = 0; y < n1; y++)
      for (long x = 0; x < n0; x++)
      {
        const long i = (zz * n1 + y) * n0 + x;
        w[i] = f[i] - tv_div(vol, z, dk, nd, x, y, zz);
      }
  memcpy(out, w, sizeof(double) * nvx);
  free(z);
  free(w);
}

double
orc_total_variation(const orc_image * vol, const double * x)
{
  /* TotalVariationImageFilter::ThreadedGenerateData
   * (include/rtkTotalVariationImageFilter.hxx): sum over voxels of the norm of
   * the forward-difference gradient (zero-flux Neumann, spacing-scaled) */
  const long n[3] = { vol->size[0], vol->size[1], vol->size[2] }, stride[3] = { 1, n[0], n[0] * n[1] };
  double     tv = 0.;
  for (long zz = 0; zz < n[2]; zz++)
    for (long y = 0; y < n[1]; y++)
      for (long xx = 0; xx < n[0]; xx++)
      {
        const long c[3] = { xx, y, zz }, i = (zz * n[1] + y) * n[0] + xx;
        double     s = 0.;
        for (int d = 0; d < 3; d++)
        {
          const double g = c[d] < n[d] - 1 ? (x[i + stride[d]] - x[i]) / vol->spacing[d] : 0.;
          s += g * g;
        }
        tv += sqrt(s);
      }
  return tv;
}

void
orc_regularized_cg(const orc_geometry * g, const orc_image * vol, const orc_image * proj, const double * proj_data,
                   const double * weights, const double * mask, double * x, int main_iterations, int cg_iterations, double tikhonov,
                   double gamma, int positivity, int tv, double gamma_tv, int tv_iterations, const int tv_dims[3],
                   int soft_threshold, double soft_threshold_value, int nthreads)
{
  /* RegularizedConjugateGradientConeBeamReconstructionFilter::GenerateData
   * (include/rtkRegularizedConjugateGradientConeBeamReconstructionFilter.hxx:
   * 250-296): main_iterations x (CG restarted from the current volume for
   * cg_iterations iterations, then ThresholdBelow(0) -> 0, TV denoising (BPDQ),
   * soft thresholding sgn(x) max(|x| - t, 0)).  weights: the CG's W (the
   * displaced-detector weighting already applied), NULL for ones. */
  const long nvx = npix(vol);
  double *   t = (double *)malloc(sizeof(double) * nvx);
  for (int m = 0; m < main_iterations; m++)
  {
    orc_cg_joseph(g, vol, proj, proj_data, weights, mask, tikhonov, gamma, cg_iterations, x, NULL, nthreads);
    if (positivity)
      for (long i = 0; i < nvx; i++)
        if (x[i] < 0.)
          x[i] = 0.;
    if (tv)
    {
      orc_tv_denoising_bpdq(vol, x, t, gamma_tv, tv_iterations, tv_dims);
      memcpy(x, t, sizeof(double) * nvx);
    }
    if (soft_threshold)
      for (long i = 0; i < nvx; i++)
      {
        const double a = fabs(x[i]) - soft_threshold_value;
        x[i] = a > 0. ? (x[i] > 0. ? a : (x[i] < 0. ? -a : 0.)) : 0.;
      }
  }
  free(t);
}

/* ------------------------------------------------------------------------ */
/* raw projections to line integrals                                        */
/* ------------------------------------------------------------------------ */
void
orc_i0_estimation(const unsigned short * raw, long n, int shift, unsigned int dyn_threshold, double out[6])
{
  /* I0EstimationProjectionFilter (include/rtkI0EstimationProjectionFilter.hxx):
   * histogram of raw >> shift over 65536 >> shift bins; Imax = the last bin
   * holding more than dyn_threshold counts (then back to a non-empty bin), Imin
   * the first such bin below it (then back to a non-empty bin); I0 = the last
   * highest bin in [3 Imax / 4, Imax) of pixel values; the FWHM bounds walk out
   * from it while a bin holds more than half the mode's count.  Imin, Imax, I0,
   * the mode's count and the half count have the 16-bit pixel type, as the
   * filter declares them. */
  const long      nbins = 65536L >> shift;
  unsigned int *  h = (unsigned int *)calloc((size_t)nbins, sizeof(unsigned int));
  for (long i = 0; i < n; i++)
    h[raw[i] >> shift]++;
  long imax = nbins - 1;
  while (h[imax] <= dyn_threshold && imax > 0)
    imax--;
  while (h[imax] == 0 && imax < nbins - 1)
    imax++;
  long imin = 0;
  while (h[imin] <= dyn_threshold && imin < imax)
    imin++;
  while (h[imin] == 0 && imin > 0)
    imin--;
  const unsigned short Imin = (unsigned short)(imin << shift), Imax = (unsigned short)(imax << shift);
  const unsigned int   start = (3u * (unsigned int)(Imax >> 2)) >> shift;
  unsigned int         id = start, maxid = start;
  unsigned short       maxval = (unsigned short)h[start];
  for (; id < (unsigned int)(Imax >> shift); id++)
    if (h[id] >= maxval)
    {
      maxval = (unsigned short)h[id];
      maxid = id;
    }
  const unsigned short half = (unsigned short)(float)(maxval >> 1);
  unsigned int         lo = maxid, hi = maxid;
  while (h[lo] > half && lo > 0)
    lo--;
  while (h[hi] > half && hi < Imax && hi < (unsigned int)nbins - 1)
    hi++;
  out[0] = (unsigned short)(maxid << shift);
  out[1] = (unsigned short)((hi - lo) << shift);
  out[2] = Imin;
  out[3] = Imax;
  out[4] = lo << shift;
  out[5] = hi << shift;
  free(h);
}

void
orc_raw_to_attenuation(const unsigned short * raw, long n, double i0, double idark, float * out)
{
  /* LUTbasedVariableI0RawToAttenuationImageFilter
   * (include/rtkLUTbasedVariableI0RawToAttenuationImageFilter.hxx): the float
   * ramp 0..65535 minus float(IDark), values below 1 set to 1 (ThresholdBelow),
   * log in double rounded to float (itk::LogImageFilter), subtracted from
   * float(log(max(I0 - IDark, 1))); out = lut[raw] */
  float *     lut = (float *)malloc(sizeof(float) * 65536);
  const float c = (float)log(i0 - idark > 1. ? i0 - idark : 1.);
  for (long r = 0; r < 65536; r++)
  {
    float v = (float)r - (float)idark;
    if (v < 1.f)
      v = 1.f;
    lut[r] = c - (float)log((double)v);
  }
  for (long i = 0; i < n; i++)
    out[i] = lut[raw[i]];
  free(lut);
}

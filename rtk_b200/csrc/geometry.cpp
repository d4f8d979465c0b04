// geometry.cpp -- FP64 host geometry of librtkb200: the product-side
// restatement of rtk::ThreeDCircularProjectionGeometry
// (src/rtkThreeDCircularProjectionGeometry.cxx) and of the matrices that RTK's
// backprojection filters derive from it (include/rtkBackProjectionImageFilter.hxx:535-595,
// include/rtkHomogeneousMatrix.h:38-81).
#include "rtkb_internal.h"

#include <algorithm>
#include <cfloat>
#include <cstring>
#include <map>
#include <mutex>

#include <cudaTypedefs.h>

namespace rtkb
{

static thread_local std::string g_last_error;

const char *
g_last_error_cstr()
{
  return g_last_error.c_str();
}

void
set_error(const std::string & msg)
{
  g_last_error = msg;
}
void
clear_error()
{
  g_last_error.clear();
}
int
fail(int code, const std::string & msg)
{
  g_last_error = msg;
  return code;
}
int
cuda_fail(cudaError_t err, const char * what)
{
  g_last_error = std::string(what) + ": " + cudaGetErrorName(err) + " (" + cudaGetErrorString(err) + ")";
  return (err == cudaErrorMemoryAllocation) ? RTKB_ERR_OUT_OF_MEMORY : RTKB_ERR_CUDA;
}

static const double kPi = 3.14159265358979323846;

void
mat_mul(const double * a, const double * b, double * c, int n, int k, int m)
{
  double t[64];
  for (int i = 0; i < n; i++)
    for (int j = 0; j < m; j++)
    {
      double s = 0.;
      for (int l = 0; l < k; l++)
        s += a[i * k + l] * b[l * m + j];
      t[i * m + j] = s;
    }
  std::memcpy(c, t, sizeof(double) * n * m);
}

void
mat4_identity(double * m)
{
  std::memset(m, 0, 16 * sizeof(double));
  m[0] = m[5] = m[10] = m[15] = 1.;
}

bool
affine4_inverse(const double * m, double * r)
{
  const double a = m[0], b = m[1], c = m[2], d = m[4], e = m[5], f = m[6], g = m[8], h = m[9], i = m[10];
  const double A = e * i - f * h, B = -(d * i - f * g), C = d * h - e * g;
  const double det = a * A + b * B + c * C;
  if (det == 0. || !std::isfinite(det))
    return false;
  const double id = 1. / det;
  double       inv[9] = { A * id,
                          -(b * i - c * h) * id,
                          (b * f - c * e) * id,
                          B * id,
                          (a * i - c * g) * id,
                          -(a * f - c * d) * id,
                          C * id,
                          -(a * h - b * g) * id,
                          (a * e - b * d) * id };
  mat4_identity(r);
  for (int row = 0; row < 3; row++)
  {
    for (int col = 0; col < 3; col++)
      r[row * 4 + col] = inv[row * 3 + col];
    r[row * 4 + 3] = -(inv[row * 3 + 0] * m[3] + inv[row * 3 + 1] * m[7] + inv[row * 3 + 2] * m[11]);
  }
  return true;
}

void
index_to_physical(const rtkb_image_desc & im, double m[16])
{
  // GetIndexToPhysicalPointMatrix, include/rtkHomogeneousMatrix.h:38-63
  mat4_identity(m);
  for (int i = 0; i < 3; i++)
  {
    for (int j = 0; j < 3; j++)
      m[i * 4 + j] = im.direction[i * 3 + j] * im.spacing[j];
    m[i * 4 + 3] = im.origin[i];
  }
}

bool
physical_to_index(const rtkb_image_desc & im, double m[16])
{
  // GetPhysicalPointToIndexMatrix, include/rtkHomogeneousMatrix.h:73-79
  double a[16];
  index_to_physical(im, a);
  return affine4_inverse(a, m);
}

bool
desc_valid(const rtkb_image_desc * d, std::string & why)
{
  if (!d)
  {
    why = "null image description";
    return false;
  }
  for (int a = 0; a < 3; a++)
  {
    if (d->size[a] <= 0)
    {
      why = "image size must be positive";
      return false;
    }
    if (!std::isfinite(d->origin[a]) || !std::isfinite(d->spacing[a]) || d->spacing[a] == 0.)
    {
      why = "image origin/spacing must be finite and spacing non-zero";
      return false;
    }
  }
  for (int q = 0; q < 9; q++)
    if (!std::isfinite(d->direction[q]))
    {
      why = "image direction must be finite";
      return false;
    }
  if ((long long)d->size[0] * d->size[1] * d->size[2] >= (1LL << 40))
  {
    why = "image too large";
    return false;
  }
  double m[16];
  if (!physical_to_index(*d, m))
  {
    why = "image direction is singular";
    return false;
  }
  return true;
}

// ---- geometry ---------------------------------------------------------------
static double
convert_0_2pi(double a)
{
  // ConvertAngleBetween0And2PIRadians, src/rtkThreeDCircularProjectionGeometry.cxx:40-44
  return a - 2 * kPi * std::floor(a / (2 * kPi));
}

static void
rotation_zxy(double ax, double ay, double az, double * m)
{
  // ComputeRotationHomogeneousMatrix (:536-549): Euler ZXY, R = Rz * Rx * Ry
  const double cx = std::cos(ax), sx = std::sin(ax), cy = std::cos(ay), sy = std::sin(ay), cz = std::cos(az),
               sz = std::sin(az);
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
  mat4_identity(inv);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      inv[i * 4 + j] = rot[j * 4 + i];
}

int
Geometry::add_projection_rad(double sid, double sdd, double ga, double pox, double poy, double oop, double ip,
                             double sox, double soy)
{
  // AddProjectionInRadians, src/rtkThreeDCircularProjectionGeometry.cxx:79-153
  const double vals[9] = { sid, sdd, ga, pox, poy, oop, ip, sox, soy };
  for (double v : vals)
    if (!std::isfinite(v))
      return fail(RTKB_ERR_INVALID_ARGUMENT, "geometry parameters must be finite");
  if (!p.empty())
  {
    if (sdd == 0. && p[0].sdd != 0.)
      return fail(RTKB_ERR_INVALID_ARGUMENT,
                  "Cannot add a parallel projection in a 3D geometry object containing divergent projections");
    if (sdd != 0. && p[0].sdd == 0.)
      return fail(RTKB_ERR_INVALID_ARGUMENT,
                  "Cannot add a divergent projection in a 3D geometry object containing parallel projections");
  }
  Proj q;
  q.sid = sid;
  q.sdd = sdd;
  q.gantry = convert_0_2pi(ga);
  q.pox = pox;
  q.poy = poy;
  q.oop = convert_0_2pi(oop);
  q.ip = convert_0_2pi(ip);
  q.sox = sox;
  q.soy = soy;
  q.coll_uinf = q.coll_usup = q.coll_vinf = q.coll_vsup = DBL_MAX; // RTK's default: no collimation

  std::memset(q.projt, 0, sizeof(q.projt));
  q.projt[0] = q.projt[4] = q.projt[8] = 1.;
  q.projt[2] = sox - pox;
  q.projt[5] = soy - poy;

  // ComputeProjectionMagnificationMatrix(-sdd, -sid), :573-582
  const double msdd = -sdd, msid = -sid;
  std::memset(q.mag, 0, sizeof(q.mag));
  q.mag[0] = q.mag[5] = (msdd == 0.) ? 1. : msdd;
  q.mag[10] = (msdd == 0.) ? 0. : 1.;
  q.mag[11] = (msdd == 0.) ? 1. : msid;

  rotation_zxy(-oop, -ga, -ip, q.rot);
  mat4_identity(q.srct);
  q.srct[3] = -sox;
  q.srct[7] = -soy;

  double t1[12], t2[12];
  mat_mul(q.projt, q.mag, t1, 3, 3, 4);
  mat_mul(t1, q.srct, t2, 3, 4, 4);
  mat_mul(t2, q.rot, q.mat, 3, 4, 4);
  p.push_back(q);

  // source angle, :133-144
  double sph[4];
  source_position((int)p.size() - 1, sph);
  sph[1] = 0.;
  const double nrm = std::sqrt(sph[0] * sph[0] + sph[2] * sph[2]);
  double       a = std::acos(sph[2] / nrm);
  if (sph[0] / nrm > 0.)
    a = 2. * kPi - a;
  p.back().source_angle = convert_0_2pi(a);
  return RTKB_OK;
}

void
Geometry::source_position(int i, double out[4]) const
{
  // GetSourcePosition, :597-608
  double inv[16];
  rotation_inverse(p[i].rot, inv);
  const double v[4] = { p[i].sox, p[i].soy, p[i].sid, 1. };
  mat_mul(inv, v, out, 4, 4, 1);
}

void
Geometry::proj_coords_to_detector(int i, double out[16]) const
{
  // GetProjectionCoordinatesToDetectorSystemMatrix, :611-625
  mat4_identity(out);
  out[3] = p[i].pox;
  out[7] = p[i].poy;
  out[11] = (p[i].sdd == 0.) ? -p[i].sid : p[i].sid - p[i].sdd;
  out[10] = 0.;
}

void
Geometry::inverse_rotation(int i, double out[16]) const
{
  rotation_inverse(p[i].rot, out);
}

// ProjectionsRegionConstIteratorRayBasedParallel::NewProjection
// (include/rtkProjectionsRegionConstIteratorRayBasedParallel.hxx:40-60): with
// no source-to-detector distance every pixel gets its own source, 2 SID along
// the detector normal, so all rays of a projection are parallel.
bool
Geometry::parallel_source_to_pixel(int i, double out[3]) const
{
  const Proj & q = p[i];
  if (q.sdd != 0.)
    return false;
  for (int a = 0; a < 3; a++)
    out[a] = -2. * q.sid * q.rot[8 + a];
  return true;
}

void
Geometry::proj_coords_to_fixed(int i, double out[16]) const
{
  // GetProjectionCoordinatesToFixedSystemMatrix, :627-637
  double d[16], inv[16];
  proj_coords_to_detector(i, d);
  rotation_inverse(p[i].rot, inv);
  mat_mul(inv, d, out, 4, 4, 4);
}

void
Geometry::source_angles(std::vector<double> & out) const
{
  out.resize(p.size());
  for (size_t i = 0; i < p.size(); i++)
    out[i] = p[i].source_angle;
}

void
Geometry::gantry_angles(std::vector<double> & out) const
{
  out.resize(p.size());
  for (size_t i = 0; i < p.size(); i++)
    out[i] = p[i].gantry;
}

void
Geometry::tilt_angles(std::vector<double> & out) const
{
  // GetTiltAngles, :407-418
  out.resize(p.size());
  for (size_t i = 0; i < p.size(); i++)
    out[i] = convert_0_2pi(-1. * p[i].gantry - p[i].source_angle);
}

void
Geometry::angular_gaps(const std::vector<double> & angles, std::vector<double> & out) const
{
  // GetAngularGaps, :478-533 (multimap order: by angle, then insertion)
  const size_t n = angles.size();
  out.assign(n, 0.);
  if (n == 1)
    out[0] = 2 * kPi;
  if (n < 2)
    return;
  std::multimap<double, unsigned> s;
  for (unsigned i = 0; i < n; i++)
    s.insert(std::make_pair(angles[i], i));
  std::vector<std::pair<double, unsigned>> v(s.begin(), s.end());
  out[v[0].second] = 0.5 * (v[1].first - v[n - 1].first + 2 * kPi);
  for (size_t k = 1; k + 1 < n; k++)
    out[v[k].second] = 0.5 * (v[k + 1].first - v[k - 1].first);
  out[v[n - 1].second] = 0.5 * (v[0].first + 2 * kPi - v[n - 2].first);
  if (!p.empty() && p[0].sdd == 0.)
  {
    const double mx = *std::max_element(out.begin(), out.end());
    if (mx > kPi / 2)
      for (double & gap : out)
      {
        if (gap > kPi / 2)
          gap -= kPi / 2;
        gap *= 2.;
      }
  }
}

void
Geometry::angular_gaps_with_next(const std::vector<double> & angles, std::vector<double> & out) const
{
  // GetAngularGapsWithNext, :447-476
  const size_t n = angles.size();
  out.assign(n, 0.);
  if (n == 1)
    out[0] = 2 * kPi;
  if (n < 2)
    return;
  std::multimap<double, unsigned> s;
  for (unsigned i = 0; i < n; i++)
    s.insert(std::make_pair(angles[i], i));
  std::vector<std::pair<double, unsigned>> v(s.begin(), s.end());
  for (size_t k = 0; k + 1 < n; k++)
    out[v[k].second] = v[k + 1].first - v[k].first;
  out[v[n - 1].second] = v[0].first + 2 * kPi - v[n - 1].first;
}

double
Geometry::to_untilted(int i, double tilted) const
{
  // ToUntiltedCoordinateAtIsocenter, :641-663
  const double sid = p[i].sid, sdd = p[i].sdd, sx = p[i].sox, px = p[i].pox;
  const double sidu = std::sqrt(sid * sid + sx * sx);
  const double l = (tilted + px - sx) * sid / sdd + sx;
  const double cosa = sx / sidu;
  return l * std::abs(sid) / (sidu - l * cosa);
}

int
bp_matrix(const Geometry & g, const rtkb_image_desc & vol, const rtkb_image_desc & proj, int i, bool fdk,
          double m[12])
{
  // BackProjectionImageFilter::GetIndexToIndexProjectionMatrix and its two
  // factors (include/rtkBackProjectionImageFilter.hxx:535-595).  The matrix is
  // kept untransposed: RTK's transposition (:480-531) is a memory-layout trick
  // and its bilinear bounds are symmetric in u and v.
  const Geometry::Proj & q = g.p[i];
  double                 vi2pp[16], t[12], volidx_to_projpp[12];
  index_to_physical(vol, vi2pp);
  mat_mul(q.mag, q.srct, t, 3, 4, 4);
  mat_mul(t, q.rot, t, 3, 4, 4);
  mat_mul(t, vi2pp, volidx_to_projpp, 3, 4, 4);

  double spp2i[16], mp[9], pp2pi[9];
  physical_to_index(proj, spp2i);
  std::memset(mp, 0, sizeof(mp));
  for (int r = 0; r < 2; r++)
  {
    mp[r * 3 + 2] = spp2i[r * 4 + 3];
    for (int c = 0; c < 2; c++)
      mp[r * 3 + c] = spp2i[r * 4 + c];
  }
  mp[8] = 1.;
  mat_mul(mp, q.projt, pp2pi, 3, 3, 3);
  mat_mul(pp2pi, volidx_to_projpp, m, 3, 3, 4);

  if (fdk)
  {
    // normalisation at the rotation centre, include/rtkFDKBackProjectionImageFilter.hxx:80-104
    double vpp2i[16];
    physical_to_index(vol, vpp2i);
    const double rc[3] = { vpp2i[3], vpp2i[7], vpp2i[11] };
    double       persp = m[11];
    for (int j = 0; j < 3; j++)
      persp += m[8 + j] * rc[j];
    for (int j = 0; j < 12; j++)
      m[j] /= persp;
  }
  // path selection on the transposed matrix (:106-116)
  if (std::abs(m[0]) < 1e-10 && std::abs(m[8]) < 1e-10)
    return 1;
  if (std::abs(m[1]) < 1e-10 && std::abs(m[9]) < 1e-10)
    return 2;
  return 0;
}

EncodeTiledFn
tensor_map_encoder()
{
  static std::once_flag once;
  static EncodeTiledFn  fn = nullptr;
  std::call_once(once, [] {
    void *                          ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(ptr);
    else
      cudaGetLastError();
  });
  return fn;
}

} // namespace rtkb

// ---- C ABI: geometry -----------------------------------------------------------
using rtkb::fail;

extern "C" const char *
rtkb_last_error(void)
{
  return rtkb::g_last_error_cstr();
}

extern "C" const char *
rtkb_version(void)
{
  return "rtkb200 0.1.0 (sm_100a)";
}

extern "C" rtkb_geometry *
rtkb_geometry_new(void)
{
  try
  {
    return new rtkb_geometry();
  }
  catch (...)
  {
    rtkb::set_error("out of host memory");
    return nullptr;
  }
}

extern "C" void
rtkb_geometry_free(rtkb_geometry * g)
{
  delete g;
}

extern "C" int
rtkb_geometry_add_projection_in_radians(rtkb_geometry * g, double sid, double sdd, double ga, double pox, double poy,
                                        double oop, double ip, double sox, double soy)
{
  if (!g)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null geometry");
  try
  {
    return g->g.add_projection_rad(sid, sdd, ga, pox, poy, oop, ip, sox, soy);
  }
  catch (...)
  {
    return fail(RTKB_ERR_OUT_OF_MEMORY, "out of host memory");
  }
}

extern "C" int
rtkb_geometry_add_projection(rtkb_geometry * g, double sid, double sdd, double ga, double pox, double poy, double oop,
                             double ip, double sox, double soy)
{
  // AddProjection, src/rtkThreeDCircularProjectionGeometry.cxx:56-77
  const double d2r = std::atan(1.0) / 45.0;
  return rtkb_geometry_add_projection_in_radians(g, sid, sdd, d2r * ga, pox, poy, d2r * oop, d2r * ip, sox, soy);
}

extern "C" int
rtkb_geometry_number_of_projections(const rtkb_geometry * g)
{
  return g ? (int)g->g.p.size() : 0;
}

static bool
proj_ok(const rtkb_geometry * g, int i)
{
  if (!g)
  {
    rtkb::set_error("null geometry");
    return false;
  }
  if (i < 0 || i >= (int)g->g.p.size())
  {
    rtkb::set_error("projection index out of range");
    return false;
  }
  return true;
}

extern "C" int
rtkb_geometry_get_matrix(const rtkb_geometry * g, int i, double out[12])
{
  if (!proj_ok(g, i) || !out)
    return RTKB_ERR_INVALID_ARGUMENT;
  std::memcpy(out, g->g.p[i].mat, 12 * sizeof(double));
  return RTKB_OK;
}

extern "C" int
rtkb_geometry_get_source_position(const rtkb_geometry * g, int i, double out[4])
{
  if (!proj_ok(g, i) || !out)
    return RTKB_ERR_INVALID_ARGUMENT;
  g->g.source_position(i, out);
  return RTKB_OK;
}

extern "C" int
rtkb_geometry_get_projection_coordinates_to_fixed_system_matrix(const rtkb_geometry * g, int i, double out[16])
{
  if (!proj_ok(g, i) || !out)
    return RTKB_ERR_INVALID_ARGUMENT;
  g->g.proj_coords_to_fixed(i, out);
  return RTKB_OK;
}

extern "C" int
rtkb_geometry_get_parameters(const rtkb_geometry * g, int which, double * out)
{
  if (!g || !out)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  const auto &        P = g->g.p;
  std::vector<double> v;
  switch (which)
  {
    case 0:
      g->g.gantry_angles(v);
      break;
    case 1:
      g->g.source_angles(v);
      break;
    case 2:
      g->g.tilt_angles(v);
      break;
    case 11:
    {
      std::vector<double> s;
      g->g.source_angles(s);
      g->g.angular_gaps(s, v);
      break;
    }
    default:
      if (which < 3 || which > 15 || which == 11)
        return fail(RTKB_ERR_INVALID_ARGUMENT, "unknown geometry parameter selector");
      v.resize(P.size());
      for (size_t i = 0; i < P.size(); i++)
      {
        const auto & q = P[i];
        const double vals[13] = { q.oop, q.ip,  q.sid, q.sdd,       q.pox,       q.poy,      q.sox,
                                  q.soy, 0.,    q.coll_uinf, q.coll_usup, q.coll_vinf, q.coll_vsup };
        v[i] = vals[which - 3];
      }
  }
  std::copy(v.begin(), v.end(), out);
  return RTKB_OK;
}

extern "C" double
rtkb_geometry_to_untilted_coordinate_at_isocenter(const rtkb_geometry * g, int i, double tilted)
{
  if (!proj_ok(g, i))
    return NAN;
  return g->g.to_untilted(i, tilted);
}

extern "C" int
rtkb_geometry_set_collimation_of_last_projection(rtkb_geometry * g, double uinf, double usup, double vinf,
                                                 double vsup)
{
  // SetCollimationOfLastProjection, src/rtkThreeDCircularProjectionGeometry.cxx
  if (!g || g->g.p.empty())
    return fail(RTKB_ERR_INVALID_ARGUMENT, "geometry has no projection");
  auto & q = g->g.p.back();
  q.coll_uinf = uinf;
  q.coll_usup = usup;
  q.coll_vinf = vinf;
  q.coll_vsup = vsup;
  return RTKB_OK;
}

extern "C" int
rtkb_geometry_set_radius_cylindrical_detector(rtkb_geometry * g, double radius)
{
  if (!g || !std::isfinite(radius))
    return fail(RTKB_ERR_INVALID_ARGUMENT, "invalid radius");
  g->g.radius_cylindrical = radius;
  return RTKB_OK;
}

extern "C" int
rtkb_backprojection_matrices(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                             int first, int n, int fdk, double * out, int * modes)
{
  std::string why;
  if (!g || !out)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  if (!rtkb::desc_valid(vol, why) || !rtkb::desc_valid(proj, why))
    return fail(RTKB_ERR_INVALID_ARGUMENT, why);
  if (first < 0 || n < 0 || first + n > proj->size[2] || proj->index[2] + first + n > (int)g->g.p.size() ||
      proj->index[2] + first < 0)
    return fail(RTKB_ERR_INVALID_ARGUMENT,
                "Mismatch between the number of projections and the geometry entries.");
  for (int s = 0; s < n; s++)
  {
    const int md = rtkb::bp_matrix(g->g, *vol, *proj, proj->index[2] + first + s, fdk != 0, out + 12 * s);
    if (modes)
      modes[s] = md;
  }
  return RTKB_OK;
}

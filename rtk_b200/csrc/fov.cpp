// fov.cpp -- the field of view of a projection stack and the displaced-detector
// weighting built on it (host code).
//
// rtk::FieldOfViewImageFilter::ComputeFOVRadius
// (include/rtkFieldOfViewImageFilter.hxx:41-187) finds the largest disc, in the
// rotation plane (x, z), that every projection sees: per projection the lines
// from the source through the first and last detector columns (corner pixels
// of the first and last rows) bound half-planes a x + b z <= c, and the disc
// (x, z, r) must lie r away inside each, a x + b z + |(a, b)| r <= c, r >= 0,
// r maximal.  RTK solves that linear programme with lp_solve; here its dual
// (three equality rows, one column per half-plane, min sum c_i y_i) runs through
// a revised simplex with Bland's rule, and the disc is the dual's simplex
// multipliers.  The optimum is unique for the stacks this serves (a polygon
// whose largest inscribed disc touches three sides), so any exact LP solver
// returns the same disc.
//
// rtk::DisplacedDetectorForOffsetFieldOfViewImageFilter
// (include/rtkDisplacedDetectorForOffsetFieldOfViewImageFilter.hxx) uses that
// disc instead of the detector corners to decide the padding and to weight
// the redundant columns.
#include "rtkb_filters.h"

#include <array>
#include <cfloat>
#include <cmath>
#include <vector>

namespace rtkb
{
namespace
{

constexpr double kPi = 3.14159265358979323846;

struct HalfPlane
{
  double a, b, c; // a x + b z + r <= c after normalisation by |(a, b)|
};

// Revised simplex for min cost^T y s.t. A y = rhs, y >= 0 with three rows:
// column j is (A[j][0], A[j][1], A[j][2]).  Returns the simplex multipliers
// pi = c_B B^-1 at the optimum, or false when the problem is infeasible or
// unbounded (or the iteration limit is reached).
bool
simplex3(const std::vector<std::array<double, 3>> & A, const std::vector<double> & cost, const double rhs[3],
         double pi_out[3])
{
  const int n = (int)A.size();
  // columns n, n+1, n+2 are the artificials of phase I
  auto col = [&](int j, int r) { return j < n ? A[j][r] : (j - n == r ? 1. : 0.); };
  int    basis[3] = { n, n + 1, n + 2 };
  double Binv[3][3] = { { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 } };
  double xb[3] = { rhs[0], rhs[1], rhs[2] };
  const double eps = 1e-11;
  auto   run = [&](bool phase1) -> int {
    // returns 0 optimal, 1 unbounded, 2 iteration limit
    for (int it = 0; it < 100000; it++)
    {
      double cb[3];
      for (int r = 0; r < 3; r++)
        cb[r] = phase1 ? (basis[r] >= n ? 1. : 0.) : (basis[r] < n ? cost[basis[r]] : 0.);
      double pi[3];
      for (int k = 0; k < 3; k++)
        pi[k] = cb[0] * Binv[0][k] + cb[1] * Binv[1][k] + cb[2] * Binv[2][k];
      // Bland: the first column with a negative reduced cost enters
      int enter = -1;
      for (int j = 0; j < n + (phase1 ? 3 : 0) && enter < 0; j++)
      {
        bool basic = false;
        for (int r = 0; r < 3; r++)
          basic = basic || basis[r] == j;
        if (basic)
          continue;
        const double cj = phase1 ? (j >= n ? 1. : 0.) : cost[j];
        const double rc = cj - (pi[0] * col(j, 0) + pi[1] * col(j, 1) + pi[2] * col(j, 2));
        if (rc < -eps)
          enter = j;
      }
      if (enter < 0)
        return 0;
      double d[3];
      for (int r = 0; r < 3; r++)
        d[r] = Binv[r][0] * col(enter, 0) + Binv[r][1] * col(enter, 1) + Binv[r][2] * col(enter, 2);
      int    leave = -1;
      double best = DBL_MAX;
      for (int r = 0; r < 3; r++)
        if (d[r] > eps)
        {
          const double ratio = xb[r] / d[r];
          if (ratio < best - 1e-14 || (std::fabs(ratio - best) <= 1e-14 && leave >= 0 && basis[r] < basis[leave]))
          {
            best = ratio;
            leave = r;
          }
        }
      if (leave < 0)
        return 1;
      const double pv = d[leave];
      for (int k = 0; k < 3; k++)
        Binv[leave][k] /= pv;
      xb[leave] /= pv;
      for (int r = 0; r < 3; r++)
        if (r != leave && d[r] != 0.)
        {
          const double f = d[r];
          for (int k = 0; k < 3; k++)
            Binv[r][k] -= f * Binv[leave][k];
          xb[r] -= f * xb[leave];
          if (xb[r] < 0. && xb[r] > -1e-12)
            xb[r] = 0.;
        }
      basis[leave] = enter;
    }
    return 2;
  };
  if (run(true) != 0)
    return false;
  double infeas = 0.;
  for (int r = 0; r < 3; r++)
    if (basis[r] >= n)
      infeas += xb[r];
  if (infeas > 1e-9)
    return false;
  // artificials left in the basis at zero: pivot them out on any column that
  // has a non-zero entry in their row (degenerate pivots)
  for (int r = 0; r < 3; r++)
  {
    if (basis[r] < n)
      continue;
    for (int j = 0; j < n; j++)
    {
      bool basic = false;
      for (int q = 0; q < 3; q++)
        basic = basic || basis[q] == j;
      if (basic)
        continue;
      double d[3];
      for (int q = 0; q < 3; q++)
        d[q] = Binv[q][0] * col(j, 0) + Binv[q][1] * col(j, 1) + Binv[q][2] * col(j, 2);
      if (std::fabs(d[r]) > 1e-9)
      {
        const double pv = d[r];
        for (int k = 0; k < 3; k++)
          Binv[r][k] /= pv;
        xb[r] /= pv;
        for (int q = 0; q < 3; q++)
          if (q != r && d[q] != 0.)
          {
            for (int k = 0; k < 3; k++)
              Binv[q][k] -= d[q] * Binv[r][k];
            xb[q] -= d[q] * xb[r];
          }
        basis[r] = j;
        break;
      }
    }
    if (basis[r] >= n)
      return false; // a redundant row: the disc is not determined
  }
  if (run(false) != 0)
    return false;
  double cb[3];
  for (int r = 0; r < 3; r++)
    cb[r] = cost[basis[r]];
  for (int k = 0; k < 3; k++)
    pi_out[k] = cb[0] * Binv[0][k] + cb[1] * Binv[1][k] + cb[2] * Binv[2][k];
  return true;
}

} // namespace

// ComputeFOVRadius (:41-187 and AddCollimationConstraints :367-452): type 0
// RADIUSINF (the first detector column's rays), 1 RADIUSSUP (the last), 2
// RADIUSBOTH.  False when the programme has no solution (lp_solve's non-zero
// return) or the detector's rotation is not handled.
int
fov_radius(const Geometry & g, const rtkb_image_desc & proj, int type, double & x, double & z, double & r)
{
  double i2p[16];
  index_to_physical(proj, i2p);
  std::vector<HalfPlane> hp;
  for (size_t k = 0; k < g.p.size(); k++)
  {
    double s4[4], p2f[16];
    g.source_position((int)k, s4);
    g.proj_coords_to_fixed((int)k, p2f);
    double a[4], b[4], c[4], d[4], cx[4], cz[4];
    for (int q = 0; q < 4; q++)
    {
      // corner q: column first / last (q / 2), row first / last (q % 2); the
      // stack coordinate does not matter (the matrix's third column is zero)
      const double iu = proj.index[0] + (q / 2) * (proj.size[0] - 1.);
      const double iv = proj.index[1] + (q % 2) * (proj.size[1] - 1.);
      double       ph[4];
      for (int r4 = 0; r4 < 4; r4++)
        ph[r4] = i2p[r4 * 4 + 0] * iu + i2p[r4 * 4 + 1] * iv + i2p[r4 * 4 + 2] * (double)k + i2p[r4 * 4 + 3];
      double pos[3];
      for (int r3 = 0; r3 < 3; r3++)
        pos[r3] = p2f[r3 * 4 + 0] * ph[0] + p2f[r3 * 4 + 1] * ph[1] + p2f[r3 * 4 + 2] * ph[2] + p2f[r3 * 4 + 3] * ph[3];
      cx[q] = pos[0];
      cz[q] = pos[2];
      a[q] = cz[q] - s4[2];
      b[q] = s4[0] - cx[q];
      c[q] = s4[0] * cz[q] - cx[q] * s4[2];
      d[q] = std::sqrt(a[q] * a[q] + b[q] * b[q]);
    }
    // orient the half-planes so that the other side's corners are inside (:110-131)
    if (a[0] * cx[2] + b[0] * cz[2] >= c[0] && a[1] * cx[3] + b[1] * cz[3] >= c[1])
      for (int q = 0; q < 2; q++)
        a[q] = -a[q], b[q] = -b[q], c[q] = -c[q];
    else if (a[2] * cx[0] + b[2] * cz[0] >= c[2] && a[3] * cx[1] + b[3] * cz[1] >= c[3])
      for (int q = 2; q < 4; q++)
        a[q] = -a[q], b[q] = -b[q], c[q] = -c[q];
    else
      return fail(RTKB_ERR_UNSUPPORTED, "Error computing the FOV, unhandled detector rotation.");
    for (int q = 0; q < 4; q++)
      if ((q < 2 && type != 1) || (q >= 2 && type != 0))
        if (d[q] > 0.)
          hp.push_back(HalfPlane{ a[q] / d[q], b[q] / d[q], c[q] / d[q] });
  }
  // collimation jaws (:367-452), when a projection sets them
  for (size_t k = 0; k < g.p.size(); k++)
  {
    const double X1 = g.p[k].coll_uinf, X2 = g.p[k].coll_usup;
    if (X1 == DBL_MAX && X2 == DBL_MAX)
      continue;
    double s4[4];
    g.source_position((int)k, s4);
    const double sx = s4[0], sz = s4[2], sn = std::sqrt(sx * sx + sz * sz);
    const double dx = sx / sn, dz = sz / sn;
    // u = (0, 1, 0) x dir = (dz, 0, -dx)
    const double ux = dz, uz = -dx;
    const double ix = -ux * X1, iz = -uz * X1, px = ux * X2, pz = uz * X2;
    double       aI = iz - sz, bI = sx - ix, cI = sx * iz - ix * sz;
    double       aS = pz - sz, bS = sx - px, cS = sx * pz - px * sz;
    const double dI = std::sqrt(aI * aI + bI * bI), dS = std::sqrt(aS * aS + bS * bS);
    if (aI * px + bI * pz >= cI)
      aI = -aI, bI = -bI, cI = -cI;
    else if (aS * ix + bS * iz >= cS)
      aS = -aS, bS = -bS, cS = -cS;
    else
      return fail(RTKB_ERR_UNSUPPORTED, "Something's wrong with the jaw handling.");
    if (type != 1 && dI > 0.)
      hp.push_back(HalfPlane{ aI / dI, bI / dI, cI / dI });
    if (type != 0 && dS > 0.)
      hp.push_back(HalfPlane{ aS / dS, bS / dS, cS / dS });
  }
  // the dual: min sum c_i y_i, sum a_i y_i = 0, sum b_i y_i = 0,
  // sum y_i - s = 1 (x, z free, r >= 0), y, s >= 0
  std::vector<std::array<double, 3>> A;
  std::vector<double>                cost;
  A.reserve(hp.size() + 1);
  for (const HalfPlane & h : hp)
  {
    A.push_back({ h.a, h.b, 1. });
    cost.push_back(h.c);
  }
  A.push_back({ 0., 0., -1. });
  cost.push_back(0.);
  const double rhs[3] = { 0., 0., 1. };
  double       pi[3];
  if (!simplex3(A, cost, rhs, pi))
    return RTKB_ERR_INVALID_ARGUMENT; // no disc: the caller decides (RTK returns false)
  x = pi[0];
  z = pi[1];
  r = pi[2];
  return RTKB_OK;
}

int
offset_fov_region(const Geometry & g, const rtkb_image_desc & proj, DisplacedInfo & info)
{
  // DisplacedDetectorForOffsetFieldOfViewImageFilter::GenerateOutputInformation
  // (include/rtkDisplacedDetectorForOffsetFieldOfViewImageFilter.hxx:36-118)
  info.out = proj;
  info.weighted = false;
  info.shift = 0;
  info.offset_fov = true;
  double cx = 0., cz = 0., cr = -1.;
  const int rcb = fov_radius(g, proj, 2, cx, cz, cr);
  if (rcb == RTKB_ERR_UNSUPPORTED)
    return rcb;
  if (rcb != RTKB_OK)
    return fail(RTKB_ERR_INVALID_ARGUMENT,
                "Cannot account for too large detector displacements, a part of space must be covered by all projections.");
  double xi = NAN, zi = NAN, ri = NAN, xs = NAN, zs = NAN, rs = NAN;
  if (fov_radius(g, proj, 0, xi, zi, ri) == RTKB_ERR_UNSUPPORTED || fov_radius(g, proj, 1, xs, zs, rs) == RTKB_ERR_UNSUPPORTED)
    return RTKB_ERR_UNSUPPORTED;
  info.fov_x = cx;
  info.fov_z = cz;
  info.fov_r = cr;
  // not displaced if the two radii differ by less than 10 % (:96-98)
  if (200. * std::fabs(ri - rs) / (ri + rs) < 10.)
    return RTKB_OK;
  info.weighted = true;
  if (rs > ri)
  {
    info.out.index[0] = proj.index[0] - proj.size[0];
    info.shift = proj.size[0];
  }
  info.out.size[0] = 2 * proj.size[0];
  return RTKB_OK;
}

void
offset_fov_weights(const Geometry & g, const rtkb_image_desc & proj, const DisplacedInfo & info, std::vector<float> & w)
{
  // DynamicThreadedGenerateData (:122-270): weights over the input columns
  const int nu = proj.size[0], np = proj.size[2];
  w.assign((size_t)np * nu, 0.f);
  const double R = info.fov_r;
  for (int s = 0; s < np; s++)
  {
    const int k = proj.index[2] + s;
    double    sp[4];
    g.source_position(k, sp);
    const double oppInvNormSource = -1. / (sp[0] * sp[0] + sp[2] * sp[2]);
    const double scx = info.fov_x - sp[0], scz = info.fov_z - sp[2];
    const double invNorm = 1. / std::sqrt(scx * scx + scz * scz);
    double       centerFOVAngle =
      std::atan2(scz * invNorm, scx * invNorm) - std::atan2(sp[2] * oppInvNormSource, sp[0] * oppInvNormSource);
    if (centerFOVAngle > kPi)
      centerFOVAngle -= 2 * kPi;
    if (centerFOVAngle < -kPi)
      centerFOVAngle += 2 * kPi;
    double theta2 = std::asin(R / std::sqrt(std::pow(info.fov_x - sp[0], 2.) + std::pow(info.fov_z - sp[2], 2.)));
    double theta1 = -1. * theta2;
    theta1 += centerFOVAngle;
    theta2 += centerFOVAngle;
    const double sx = g.p[k].sox;
    double       sid = g.p[k].sid;
    sid = std::sqrt(sid * sid + sx * sx);
    const double liml1 = std::tan(theta1) * sid, liml2 = std::tan(theta2) * sid;
    double       invsid = 0., piOverDen = 0.;
    if (sid != 0.)
    {
      invsid = 1. / sid;
      piOverDen = (kPi / 2) * std::sqrt(scx * scx + scz * scz) / R;
    }
    for (int i = 0; i < nu; i++)
    {
      const double x = proj.origin[0] + proj.spacing[0] * (proj.index[0] + i);
      const double l = g.to_untilted(k, x);
      double       v;
      if (info.shift != 0) // padded on the left: the input starts at a later output index
        v = (l <= liml1) ? 0. : (l >= liml2 ? 2. : std::sin(std::sin(std::atan(l * invsid) - centerFOVAngle) * piOverDen) + 1.);
      else
        v = (l <= liml1) ? 2. : (l >= liml2 ? 0. : 1. - std::sin(std::sin(std::atan(l * invsid) - centerFOVAngle) * piOverDen));
      w[(size_t)s * nu + i] = (float)v;
    }
  }
}

} // namespace rtkb

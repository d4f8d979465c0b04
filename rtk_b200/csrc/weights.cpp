// weights.cpp -- FP64 host-side tables of the projection weighting filters:
// rtk::FDKWeightProjectionFilter (include/rtkFDKWeightProjectionFilter.hxx:40-128),
// rtk::ParkerShortScanImageFilter (include/rtkParkerShortScanImageFilter.hxx:41-209),
// rtk::DisplacedDetectorImageFilter (include/rtkDisplacedDetectorImageFilter.hxx:83-323)
// and the ramp kernel of rtk::FFTRampImageFilter (include/rtkFFTRampImageFilter.hxx:47-178).
#include "rtkb_filters.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <complex>
#include <map>

namespace rtkb
{

static const double kPi = 3.14159265358979323846;

void
fdk_weight_params(const Geometry & g, const rtkb_image_desc & proj, std::vector<double> & out)
{
  // BeforeThreadedGenerateData: angular gaps of the source angles times the
  // ramp correction; DynamicThreadedGenerateData: cos(gamma) on the detector.
  std::vector<double> sang, fac, tilt;
  g.source_angles(sang);
  g.angular_gaps(sang, fac);
  g.tilt_angles(tilt);
  double i2p[16], base[3], inc[3];
  index_to_physical(proj, i2p);
  for (int a = 0; a < 3; a++)
  {
    base[a] = i2p[a * 4 + 3] + i2p[a * 4 + 0] * proj.index[0] + i2p[a * 4 + 1] * proj.index[1] +
              i2p[a * 4 + 2] * proj.index[2];
    inc[a] = i2p[a * 4 + 0] + i2p[a * 4 + 1] + i2p[a * 4 + 2];
  }
  const int np = proj.size[2];
  out.assign((size_t)np * kFdkWeightParams, 0.);
  for (int s = 0; s < np; s++)
  {
    const int              k = proj.index[2] + s;
    const Geometry::Proj & q = g.p[k];
    double *               o = out.data() + (size_t)s * kFdkWeightParams;
    double                 f = fac[k];
    if (q.sdd == 0.)
    {
      f *= 0.5;
      o[0] = f;
      o[7] = 1.; // parallel: constant weight
      continue;
    }
    double sp[4];
    g.source_position(k, sp);
    f *= std::abs(q.sdd) / (2. * q.sid * q.sid);
    f *= std::sqrt(sp[0] * sp[0] + sp[1] * sp[1] + sp[2] * sp[2]);
    const double cosa = std::cos(tilt[k]), sina = std::sin(tilt[k]), tana = std::tan(tilt[k]);
    const double RD = q.sdd - q.sid;
    o[0] = f;
    o[1] = q.sdd * (cosa + tana * sina); // numpart1
    o[2] = sina;
    o[3] = q.sdd * tana; // sddtana
    o[4] = q.sdd * q.sdd;
    o[5] = base[0] + q.pox + tana * RD; // x of column 0
    o[6] = base[1] + q.poy - q.soy;     // y of row 0
    o[7] = 0.;
    o[8] = inc[0];
    o[9] = inc[1];
  }
}

bool
parker_weights(const Geometry & g, const rtkb_image_desc & proj, double threshold, std::vector<float> & w)
{
  // GenerateInputRequestedRegion (short-scan detection, delta, first angle)
  // and DynamicThreadedGenerateData (per-column weights).
  const int           n = (int)g.p.size();
  std::vector<double> ga, gaps;
  g.gantry_angles(ga);
  g.angular_gaps_with_next(ga, gaps);
  if (n < 1 || g.p[0].sdd == 0.)
    return false;
  int maxpos = 0;
  for (int k = 1; k < n; k++)
    if (gaps[k] > gaps[maxpos])
      maxpos = k;
  if (gaps[maxpos] < threshold)
    return false;
  std::map<double, unsigned> sorted;
  for (int k = 0; k < n; k++)
    sorted.insert(std::make_pair(ga[k], (unsigned)k));
  auto itLast = sorted.find(ga[maxpos]);
  auto itFirst = itLast;
  ++itFirst;
  if (itFirst == sorted.end())
    itFirst = sorted.begin();
  const double firstAngle = itFirst->first;
  double       lastAngle = itLast->first;
  if (lastAngle < firstAngle)
    lastAngle += 2 * kPi;
  double delta = 0.5 * (lastAngle - firstAngle - kPi);
  delta = delta - 2 * kPi * std::floor(delta / (2 * kPi));

  const int nu = proj.size[0], np = proj.size[2];
  w.assign((size_t)np * nu, 0.f);
  for (int s = 0; s < np; s++)
  {
    const int    k = proj.index[2] + s;
    const double sox = g.p[k].sox, sid = g.p[k].sid;
    const double invsid = 1. / std::sqrt(sid * sid + sox * sox);
    double       beta = ga[k] - firstAngle;
    if (beta < 0)
      beta += 2 * kPi;
    for (int i = 0; i < nu; i++)
    {
      const double x = proj.origin[0] + proj.spacing[0] * (proj.index[0] + i);
      const double l = g.to_untilted(k, x);
      const double alpha = std::atan(-1 * l * invsid);
      double       v;
      if (beta <= 2 * delta - 2 * alpha)
        v = 2. * std::pow(std::sin((kPi * beta) / (4 * (delta - alpha))), 2.);
      else if (beta <= kPi - 2 * alpha)
        v = 2.;
      else if (beta <= kPi + 2 * delta)
        v = 2. * std::pow(std::sin((kPi * (kPi + 2 * delta - beta)) / (4 * (delta + alpha))), 2.);
      else
        v = 0.;
      w[(size_t)s * nu + i] = (float)v;
    }
  }
  return true;
}

int
displaced_region(const Geometry & g, const rtkb_image_desc & proj, bool pad, DisplacedInfo & info)
{
  // GenerateOutputInformation, include/rtkDisplacedDetectorImageFilter.hxx:83-178
  double i2p[16];
  index_to_physical(proj, i2p);
  double inf = i2p[3] + i2p[0] * proj.index[0] + i2p[1] * proj.index[1] + i2p[2] * proj.index[2];
  double sup = inf;
  if (proj.spacing[0] < 0.)
    inf += proj.spacing[0] * (proj.size[0] - 1);
  else
    sup += proj.spacing[0] * (proj.size[0] - 1);
  double maxInf = -DBL_MAX, minSup = DBL_MAX;
  for (size_t i = 0; i < g.p.size(); i++)
  {
    maxInf = std::max(maxInf, g.to_untilted((int)i, inf));
    minSup = std::min(minSup, g.to_untilted((int)i, sup));
  }
  info.inf = maxInf;
  info.sup = minSup;
  info.out = proj;
  info.weighted = false;
  info.shift = 0;
  if (maxInf > 0. || minSup < 0.)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "Cannot account for detector displacement larger than 50% of panel size.");
  if (std::abs(maxInf + minSup) < 0.1 * std::abs(minSup - maxInf))
    return RTKB_OK; // not displaced: the filter copies its input
  info.weighted = true;
  if (!pad)
    return RTKB_OK;
  if (minSup + maxInf > 0.)
  {
    info.out.index[0] = proj.index[0] - proj.size[0];
    info.shift = proj.size[0];
  }
  info.out.size[0] = 2 * proj.size[0];
  return RTKB_OK;
}

void
displaced_weights(const Geometry & g, const rtkb_image_desc & proj, const DisplacedInfo & info, std::vector<float> & w)
{
  // DynamicThreadedGenerateData, :182-323 (weights over the input columns)
  const int    nu = proj.size[0], np = proj.size[2];
  const double theta = std::min(-1 * info.inf, info.sup);
  w.assign((size_t)np * nu, 0.f);
  for (int s = 0; s < np; s++)
  {
    const int    k = proj.index[2] + s;
    const double sx = g.p[k].sox;
    double       sid = g.p[k].sid;
    sid = std::sqrt(sid * sid + sx * sx);
    double invsid = 0., invden = 0.;
    if (sid != 0.)
    {
      invsid = 1. / sid;
      invden = 1. / (2. * std::atan(theta * invsid));
    }
    for (int i = 0; i < nu; i++)
    {
      const double x = proj.origin[0] + proj.spacing[0] * (proj.index[0] + i);
      const double l = g.to_untilted(k, x);
      double       v;
      if (info.sup + info.inf > 0.)
        v = (l <= -theta) ? 0. : (l >= theta ? 2. : std::sin(kPi * std::atan(l * invsid) * invden) + 1);
      else
        v = (l <= -theta) ? 2. : (l >= theta ? 0. : 1 - std::sin(kPi * std::atan(l * invsid) * invden));
      w[(size_t)s * nu + i] = (float)v;
    }
  }
}

static int
greatest_prime_factor(int n)
{
  // FFTProjectionsConvolutionImageFilter::GreatestPrimeFactor,
  // include/rtkFFTProjectionsConvolutionImageFilter.hxx:322-333
  int v = 2;
  auto is_prime = [](int x) {
    const int last = (int)std::sqrt((double)x);
    for (int d = 2; d <= last; d++)
      if (x % d == 0)
        return false;
    return true;
  };
  while (v <= n)
    if (n % v == 0 && is_prime(v))
      n /= v;
    else
      v += 1;
  return v;
}

int
ramp_padded_size(int nu, const rtkb_ramp_params & p)
{
  // GetPaddedImageRegion, :280-306
  const int gpf = p.greatest_prime_factor > 0 ? p.greatest_prime_factor : 2;
  const int zp = p.zero_pad_factor > 0 ? p.zero_pad_factor : 2;
  long long x = (long long)zp * nu;
  while (greatest_prime_factor((int)x) > gpf)
    x++;
  return (int)x;
}

int
ramp_padded_size_y(int nv, const rtkb_ramp_params & p)
{
  // GetPaddedImageRegion, :296-301: rows are padded only for the 2-D kernel
  // (HannCutFrequencyY > 0, FFTRampImageFilter.hxx:41); ZeroPadFactors[1] is
  // clamped to [1, 2] (FFTProjectionsConvolutionImageFilter.h:108-111)
  if (!(p.hann_cut_y > 0.))
    return nv;
  const int gpf = p.greatest_prime_factor > 0 ? p.greatest_prime_factor : 2;
  const int zy = p.zero_pad_factor_y > 0 ? std::min(p.zero_pad_factor_y, 2) : 2;
  long long y = (long long)zy * nv;
  while (greatest_prime_factor((int)y) > gpf)
    y++;
  return (int)y;
}

void
ramp_window_y(int padded_y, const rtkb_ramp_params & p, std::vector<double> & w)
{
  // UpdateFFTProjectionsConvolutionKernel, include/rtkFFTRampImageFilter.hxx:141-177:
  // rows j and padded_y - j of the 2-D kernel carry the 1-D kernel times
  // 0.5 (1 + cos(pi j / ncut)) for j < ncut = round((padded_y/2 + 1) min(1, fy))
  const int half = padded_y / 2;
  w.assign((size_t)half + 1, 0.);
  if (!(p.hann_cut_y > 0.))
    return;
  const int ncut = (int)std::floor((half + 1) * std::min(1.0, p.hann_cut_y) + 0.5);
  for (int j = 0; j < ncut && j <= half; j++)
    w[j] = 0.5 * (1 + std::cos(kPi * j / ncut));
}

static void
fft_pow2(std::vector<std::complex<double>> & a)
{
  const size_t n = a.size();
  for (size_t i = 1, j = 0; i < n; i++)
  {
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1)
      j ^= bit;
    j ^= bit;
    if (i < j)
      std::swap(a[i], a[j]);
  }
  for (size_t len = 2; len <= n; len <<= 1)
  {
    const double ang = -2 * kPi / (double)len;
    for (size_t i = 0; i < n; i += len)
      for (size_t k = 0; k < len / 2; k++)
      {
        const std::complex<double> w(std::cos(ang * k), std::sin(ang * k));
        const std::complex<double> u = a[i + k], v = a[i + k + len / 2] * w;
        a[i + k] = u + v;
        a[i + k + len / 2] = u - v;
      }
  }
}

void
ramp_kernel(int padded, double spacing, const rtkb_ramp_params & p, std::vector<double> & K)
{
  // UpdateFFTProjectionsConvolutionKernel (1-D kernel): spatial ramp
  // 1/(4s), -1/((k pi)^2 s) at odd k, FFT, then windowing.
  std::vector<std::complex<double>> a((size_t)padded, 0.);
  a[0] = 1. / (4. * spacing);
  for (int ix = 1, jx = padded - 1; ix < padded / 2; ix += 2, jx -= 2)
  {
    double v = ix * kPi;
    v = -1. / (v * v * spacing);
    a[ix] = v;
    a[jx] = v;
  }
  const int n = padded / 2 + 1;
  K.resize(n);
  if ((padded & (padded - 1)) == 0)
  {
    fft_pow2(a);
    for (int i = 0; i < n; i++)
      K[i] = a[i].real();
  }
  else
  {
    // other lengths (a greatest prime factor above 2, RTK built with FFTW):
    // the transform of the real, even kernel as cosine sums
    for (int i = 0; i < n; i++)
    {
      double acc = 0.;
      for (int k = 0; k < padded; k++)
        acc += a[k].real() * std::cos(2. * kPi * (double)(((long long)i * k) % padded) / padded);
      K[i] = acc;
    }
  }
  auto ncut_of = [n](double c) { return (int)std::floor(n * std::min(1.0, c) + 0.5); };
  int  start_zero = n;
  if (p.hann_cut > 0.)
  {
    const int ncut = ncut_of(p.hann_cut);
    for (int i = 0; i < ncut; i++)
      K[i] *= 0.5 * (1 + std::cos(kPi * i / ncut));
    start_zero = ncut;
  }
  else if (p.cosine_cut > 0.)
  {
    const int ncut = ncut_of(p.cosine_cut);
    for (int i = 0; i < ncut; i++)
      K[i] *= std::cos(0.5 * kPi * i / ncut);
    start_zero = ncut;
  }
  else if (p.hamming > 0.)
  {
    const int ncut = ncut_of(p.hamming);
    for (int i = 0; i < ncut; i++)
      K[i] *= 0.54 + 0.46 * std::cos(kPi * i / ncut);
    start_zero = ncut;
  }
  else if (p.ramlak_cut > 0.)
    start_zero = ncut_of(p.ramlak_cut);
  else if (p.shepplogan_cut > 0.)
  {
    const int ncut = ncut_of(p.shepplogan_cut);
    for (int i = 1; i < ncut; i++)
    {
      const double x = 0.5 * kPi * i / ncut;
      K[i] *= std::sin(x) / x;
    }
    start_zero = std::max(ncut, 1);
  }
  for (int i = start_zero; i < n; i++)
    K[i] = 0.;
}

void
embed_spectrum(int P, int M, const std::vector<double> & K, std::vector<double> & KM)
{
  // h = the kernel's period-P spatial form (real and even: h[d] = h[P - d]);
  // on an FFT of length M >= 2P - 1 it sits at offsets -(P-1)..P-1, so the
  // length-M circular convolution of an input supported in [0, P) equals the
  // period-P one at every output sample in [0, P).
  std::vector<double> h((size_t)P);
  for (int d = 0; d < P; d++)
  {
    double acc = 0.;
    for (int f = 0; f < P; f++)
      acc += K[(size_t)std::min(f, P - f)] * std::cos(2. * kPi * (double)(((long long)f * d) % P) / P);
    h[d] = acc / P;
  }
  std::vector<std::complex<double>> a((size_t)M, 0.);
  for (int d = 0; d < P; d++)
    a[d] = h[d];
  for (int d = 1; d < P; d++)
    a[(size_t)M - d] = h[(size_t)P - d];
  fft_pow2(a);
  KM.resize((size_t)M / 2 + 1);
  for (int i = 0; i <= M / 2; i++)
    KM[i] = a[i].real();
}

int
fft_length_for_period(int P)
{
  if ((P & (P - 1)) == 0)
    return P;
  int M = 1;
  while (M < 2 * P - 1)
    M <<= 1;
  return M;
}

void
twiddles(int n, std::vector<float> & tw)
{
  // e^{-2 pi i m / n}, m in [0, n), computed in FP64
  tw.resize(2 * (size_t)n);
  for (int m = 0; m < n; m++)
  {
    const double a = -2. * kPi * (double)m / (double)n;
    tw[2 * m] = (float)std::cos(a);
    tw[2 * m + 1] = (float)std::sin(a);
  }
}

void
truncation_mirror_weights(int next, std::vector<float> & mw)
{
  // UpdateTruncationMirrorWeights, :345-355
  mw.assign((size_t)next + 1, 0.f);
  for (int i = 0; i < next + 1; i++)
    mw[i] = (float)std::pow(std::sin((next - i) * kPi / (2 * next - 2)), 0.75);
}

} // namespace rtkb

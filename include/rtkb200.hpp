/*
 * rtkb200.hpp -- header-only C++ layer over the C ABI of librtkb200, with the
 * class and setter names of the RTK filters each entry point replaces, for C++
 * callers that hold device buffers themselves (no ITK dependency).
 *
 * Conventions, as in RTK: a filter is configured with Set...() calls and runs
 * on Update(); failures throw rtkb::Exception (RTK throws itk::ExceptionObject)
 * with the library's message.  Images are rtkb_image_desc descriptions plus
 * caller-owned device pointers; Update() enqueues the work on the filter's
 * stream (SetStream, default the legacy stream) and returns without
 * synchronising, except where the C entry point it calls waits (the solvers
 * that iterate on host-side decisions say so in rtkb200.h).
 */
#ifndef RTKB200_HPP
#define RTKB200_HPP

#include "rtkb200.h"

#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace rtkb
{

class Exception : public std::runtime_error
{
public:
  explicit Exception(const std::string & what)
    : std::runtime_error(what)
  {}
};

inline void
Check(int rc, const char * where)
{
  if (rc != RTKB_OK)
    throw Exception(std::string(where) + ": " + rtkb_last_error());
}

/* An ITK-style image description: size, index, origin, spacing, direction. */
inline rtkb_image_desc
MakeImageDescription(const int size[3], const double spacing[3], const double origin[3], const int index[3] = nullptr,
                     const double direction[9] = nullptr)
{
  rtkb_image_desc d{};
  for (int a = 0; a < 3; a++)
  {
    d.size[a] = size[a];
    d.index[a] = index ? index[a] : 0;
    d.origin[a] = origin[a];
    d.spacing[a] = spacing[a];
  }
  for (int k = 0; k < 9; k++)
    d.direction[k] = direction ? direction[k] : (k % 4 == 0 ? 1. : 0.);
  return d;
}

/* rtk::ThreeDCircularProjectionGeometry (FP64), owning its handle. */
class ThreeDCircularProjectionGeometry
{
public:
  ThreeDCircularProjectionGeometry()
    : m_G(rtkb_geometry_new())
  {
    if (!m_G)
      throw Exception("rtkb_geometry_new: allocation failed");
  }
  ~ThreeDCircularProjectionGeometry() { rtkb_geometry_free(m_G); }
  ThreeDCircularProjectionGeometry(const ThreeDCircularProjectionGeometry &) = delete;
  ThreeDCircularProjectionGeometry & operator=(const ThreeDCircularProjectionGeometry &) = delete;
  ThreeDCircularProjectionGeometry(ThreeDCircularProjectionGeometry && o) noexcept
    : m_G(std::exchange(o.m_G, nullptr))
  {}

  /* angles in degrees, as RTK's AddProjection */
  void
  AddProjection(double sid, double sdd, double gantryAngle, double projOffsetX = 0., double projOffsetY = 0.,
                double outOfPlaneAngle = 0., double inPlaneAngle = 0., double sourceOffsetX = 0.,
                double sourceOffsetY = 0.)
  {
    Check(rtkb_geometry_add_projection(m_G, sid, sdd, gantryAngle, projOffsetX, projOffsetY, outOfPlaneAngle,
                                       inPlaneAngle, sourceOffsetX, sourceOffsetY),
          "AddProjection");
  }
  void
  SetRadiusCylindricalDetector(double r)
  {
    Check(rtkb_geometry_set_radius_cylindrical_detector(m_G, r), "SetRadiusCylindricalDetector");
  }
  void
  SetCollimationOfLastProjection(double uinf, double usup, double vinf, double vsup)
  {
    Check(rtkb_geometry_set_collimation_of_last_projection(m_G, uinf, usup, vinf, vsup),
          "SetCollimationOfLastProjection");
  }
  int
  GetNumberOfProjections() const
  {
    return rtkb_geometry_number_of_projections(m_G);
  }
  std::vector<double>
  GetMatrix(int i) const
  {
    std::vector<double> m(12);
    Check(rtkb_geometry_get_matrix(m_G, i, m.data()), "GetMatrix");
    return m;
  }
  /* rtk::ThreeDCircularProjectionGeometryXMLFileReader / ...Writer */
  static ThreeDCircularProjectionGeometry
  Read(const std::string & filename)
  {
    rtkb_geometry * g = nullptr;
    Check(rtkb_geometry_read_xml(filename.c_str(), &g), "ReadGeometry");
    return ThreeDCircularProjectionGeometry(g);
  }
  void
  Write(const std::string & filename) const
  {
    Check(rtkb_geometry_write_xml(m_G, filename.c_str()), "WriteGeometry");
  }
  const rtkb_geometry *
  GetHandle() const
  {
    return m_G;
  }

private:
  explicit ThreeDCircularProjectionGeometry(rtkb_geometry * g)
    : m_G(g)
  {}
  rtkb_geometry * m_G;
};

/* Common part of the filters: geometry, volume and projection stack. */
class ProjectorBase
{
public:
  void
  SetGeometry(const ThreeDCircularProjectionGeometry & g)
  {
    m_Geometry = g.GetHandle();
  }
  void
  SetStream(void * stream)
  {
    m_Stream = stream;
  }
  /* volume description with its input (added to) and output buffers (may be equal) */
  void
  SetVolume(const rtkb_image_desc & d, const float * in, float * out)
  {
    m_Vol = d;
    m_VolIn = in;
    m_VolOut = out;
  }
  void
  SetProjections(const rtkb_image_desc & d, const float * in, float * out = nullptr)
  {
    m_Proj = d;
    m_ProjIn = in;
    m_ProjOut = out;
  }

protected:
  const rtkb_geometry * m_Geometry = nullptr;
  void *                m_Stream = nullptr;
  rtkb_image_desc       m_Vol{}, m_Proj{};
  const float *         m_VolIn = nullptr;
  float *               m_VolOut = nullptr;
  const float *         m_ProjIn = nullptr;
  float *               m_ProjOut = nullptr;
};

/* rtk::FDKBackProjectionImageFilter: volume out = volume in + FDK-weighted backprojection */
class FDKBackProjectionImageFilter : public ProjectorBase
{
public:
  void
  Update()
  {
    Check(rtkb_fdk_backproject(m_Geometry, &m_Vol, &m_Proj, m_ProjIn, m_VolIn, m_VolOut, m_Stream),
          "FDKBackProjectionImageFilter");
  }
};

/* rtk::FDKWeightProjectionFilter: projections out = FDK-weighted projections in (out may equal in) */
class FDKWeightProjectionFilter : public ProjectorBase
{
public:
  void
  Update()
  {
    Check(rtkb_fdk_weight(m_Geometry, &m_Proj, m_ProjIn, m_ProjOut, m_Stream), "FDKWeightProjectionFilter");
  }
};

/* rtk::ParkerShortScanImageFilter; a full scan copies the projections */
class ParkerShortScanImageFilter : public ProjectorBase
{
public:
  void
  SetAngularGapThreshold(double radians)
  {
    m_Threshold = radians;
  }
  void
  Update()
  {
    int s = 0;
    Check(rtkb_parker_short_scan(m_Geometry, &m_Proj, m_Threshold, m_ProjIn, m_ProjOut, m_Stream, &s),
          "ParkerShortScanImageFilter");
    m_Short = s != 0;
  }
  /* after Update: whether the scan was short (weights applied) */
  bool
  GetIsShortScan() const
  {
    return m_Short;
  }

private:
  double m_Threshold = 3.14159265358979323846 / 9;
  bool   m_Short = false;
};

/* rtk::DisplacedDetectorImageFilter; the output may be wider than the input
 * (padded on the truncated side): size its buffer from GetOutputRegion(). */
class DisplacedDetectorImageFilter : public ProjectorBase
{
public:
  void
  SetPadOnTruncatedSide(bool pad)
  {
    m_Pad = pad;
  }
  rtkb_image_desc
  GetOutputRegion() const
  {
    rtkb_image_desc out{};
    int             weighted = 0;
    Check(rtkb_displaced_detector_region(m_Geometry, &m_Proj, m_Pad ? 1 : 0, &out, &weighted),
          "DisplacedDetectorImageFilter");
    return out;
  }
  void
  Update()
  {
    Check(rtkb_displaced_detector(m_Geometry, &m_Proj, m_Pad ? 1 : 0, m_ProjIn, m_ProjOut, m_Stream),
          "DisplacedDetectorImageFilter");
  }

private:
  bool m_Pad = true;
};

/* rtk::DisplacedDetectorForOffsetFieldOfViewImageFilter: padding and weights
 * from the stack's field of view (always padded on the truncated side) */
class DisplacedDetectorForOffsetFieldOfViewImageFilter : public ProjectorBase
{
public:
  rtkb_image_desc
  GetOutputRegion() const
  {
    rtkb_image_desc out{};
    int             weighted = 0;
    Check(rtkb_displaced_detector_offset_fov_region(m_Geometry, &m_Proj, &out, &weighted),
          "DisplacedDetectorForOffsetFieldOfViewImageFilter");
    return out;
  }
  void
  Update()
  {
    Check(rtkb_displaced_detector_offset_fov(m_Geometry, &m_Proj, m_ProjIn, m_ProjOut, m_Stream),
          "DisplacedDetectorForOffsetFieldOfViewImageFilter");
  }
};

/* rtk::FFTRampImageFilter (no geometry): window cut frequencies as RTK's setters */
class FFTRampImageFilter : public ProjectorBase
{
public:
  FFTRampImageFilter() { m_R = rtkb_ramp_params{ 0., 0., 0., 0., 0., 0., 2, 2, 0., 2 }; }
  void SetHannCutFrequency(double f) { m_R.hann_cut = f; }
  void SetCosineCutFrequency(double f) { m_R.cosine_cut = f; }
  void SetHammingFrequency(double f) { m_R.hamming = f; }
  void SetRamLakCutFrequency(double f) { m_R.ramlak_cut = f; }
  void SetSheppLoganCutFrequency(double f) { m_R.shepplogan_cut = f; }
  void SetTruncationCorrection(double t) { m_R.truncation_correction = t; }
  void SetZeroPadFactor(int z) { m_R.zero_pad_factor = z; }
  void SetHannCutFrequencyY(double f) { m_R.hann_cut_y = f; }
  /* ZeroPadFactors (x, y) as RTK's SetZeroPadFactors */
  void
  SetZeroPadFactors(int zx, int zy)
  {
    m_R.zero_pad_factor = zx;
    m_R.zero_pad_factor_y = zy;
  }
  void
  Update()
  {
    Check(rtkb_ramp_filter(&m_Proj, &m_R, m_ProjIn, m_ProjOut, m_Stream), "FFTRampImageFilter");
  }

protected:
  rtkb_ramp_params m_R;
};

/* rtk::FDKConeBeamReconstructionFilter: weighting and ramp filtering of the
 * projections (in one pass; optionally the displaced-detector and Parker
 * weights of the filters rtkfdk chains before it) into a caller-provided
 * buffer, then the FDK backprojection into the volume.  The filtered buffer
 * holds GetFilteredRegion()'s pixels. */
class FDKConeBeamReconstructionFilter : public FFTRampImageFilter
{
public:
  void SetDisplacedDetector(bool on) { m_Displaced = on; }
  void SetShortScan(bool on) { m_Short = on; }
  void SetFilteredProjectionsBuffer(float * d) { m_Filtered = d; }
  rtkb_image_desc
  GetFilteredRegion() const
  {
    if (!m_Displaced)
      return m_Proj;
    rtkb_image_desc out{};
    int             weighted = 0;
    Check(rtkb_displaced_detector_region(m_Geometry, &m_Proj, 1, &out, &weighted), "FDKConeBeamReconstructionFilter");
    return out;
  }
  void
  Update()
  {
    if (!m_Filtered)
      throw Exception("FDKConeBeamReconstructionFilter: no buffer for the filtered projections");
    rtkb_fdk_preprocess_params p{};
    p.displaced_detector = m_Displaced ? 1 : 0;
    p.pad_on_truncated_side = 1;
    p.short_scan = m_Short ? 1 : 0;
    p.angular_gap_threshold = 0.;
    p.ramp = m_R;
    rtkb_image_desc f{};
    Check(rtkb_fdk_preprocess(m_Geometry, &m_Proj, &p, &f, m_ProjIn, m_Filtered, m_Stream),
          "FDKConeBeamReconstructionFilter");
    Check(rtkb_fdk_backproject(m_Geometry, &m_Vol, &f, m_Filtered, m_VolIn, m_VolOut, m_Stream),
          "FDKConeBeamReconstructionFilter");
  }

private:
  bool    m_Displaced = false, m_Short = false;
  float * m_Filtered = nullptr;
};

/* rtk::BackProjectionImageFilter (voxel-based) */
class BackProjectionImageFilter : public ProjectorBase
{
public:
  void
  Update()
  {
    Check(rtkb_voxel_backproject(m_Geometry, &m_Vol, &m_Proj, m_ProjIn, m_VolIn, m_VolOut, m_Stream),
          "BackProjectionImageFilter");
  }
};

/* rtk::JosephForwardProjectionImageFilter: projections out = projections in + line integrals of the volume */
class JosephForwardProjectionImageFilter : public ProjectorBase
{
public:
  void
  Update()
  {
    Check(rtkb_joseph_forward_project(m_Geometry, &m_Vol, &m_Proj, m_VolIn, m_ProjIn, m_ProjOut, m_Stream),
          "JosephForwardProjectionImageFilter");
  }
};

/* rtk::JosephBackProjectionImageFilter */
class JosephBackProjectionImageFilter : public ProjectorBase
{
public:
  void
  Update()
  {
    Check(rtkb_joseph_back_project(m_Geometry, &m_Vol, &m_Proj, m_ProjIn, m_VolIn, m_VolOut, m_Stream),
          "JosephBackProjectionImageFilter");
  }
};

/* rtk::ConjugateGradientConeBeamReconstructionFilter (Joseph pair): the
 * volume buffer holds x0 and receives the result. */
class ConjugateGradientConeBeamReconstructionFilter : public ProjectorBase
{
public:
  ~ConjugateGradientConeBeamReconstructionFilter() { rtkb_cg_destroy(m_Plan); }
  void
  SetNumberOfIterations(int n)
  {
    m_Iterations = n;
  }
  void
  SetTikhonov(double t)
  {
    m_Params.tikhonov = t;
  }
  void
  SetGamma(double g)
  {
    m_Params.gamma = g;
  }
  /* IterativeConeBeamReconstructionFilter::SetBackProjectionFilter with RTK's
   * BackProjectionType values: 0 BP_VOXELBASED (default), 1 BP_JOSEPH,
   * 2 BP_CUDAVOXELBASED; the forward projector is Joseph. */
  void
  SetBackProjectionFilter(int bptype)
  {
    m_Params.backprojector = bptype;
  }
  void
  SetInputWeights(const float * w)
  {
    m_Weights = w;
  }
  void
  SetSupportMask(const float * m)
  {
    m_Mask = m;
  }
  void
  SetDisableDisplacedDetectorFilter(bool d)
  {
    m_Displaced = !d;
  }
  void
  Update()
  {
    rtkb_cg_destroy(m_Plan);
    m_Plan = nullptr;
    m_Params.use_cuda_graph = 1;
    Check(rtkb_cg_create(m_Geometry, &m_Vol, &m_Proj, &m_Params, &m_Plan), "ConjugateGradient (create)");
    if (m_Mask)
      Check(rtkb_cg_set_support_mask(m_Plan, m_Mask), "SetSupportMask");
    Check(rtkb_cg_start(m_Plan, m_ProjIn, m_Weights, m_Displaced ? 1 : 0, m_VolOut, m_Stream),
          "ConjugateGradient (start)");
    Check(rtkb_cg_iterate(m_Plan, m_Iterations, m_Stream), "ConjugateGradient (iterate)");
    Check(rtkb_cg_finish(m_Plan, m_Stream), "ConjugateGradient (support mask)");
  }

private:
  rtkb_cg *      m_Plan = nullptr;
  rtkb_cg_params m_Params{ 0., 1, 0, 0., 0 };
  int            m_Iterations = 3;
  const float *  m_Weights = nullptr;
  const float *  m_Mask = nullptr;
  bool           m_Displaced = true;
};

/* rtk::SARTConeBeamReconstructionFilter (RTK's defaults), in place on the volume output buffer */
class SARTConeBeamReconstructionFilter : public ProjectorBase
{
public:
  SARTConeBeamReconstructionFilter() { m_P = { 3, 0.3, 0, 1, 0, 1e-5, nullptr, 0ULL }; }
  void SetNumberOfIterations(int n) { m_P.niter = n; }
  void SetLambda(double l) { m_P.lambda = l; }
  void SetEnforcePositivity(bool b) { m_P.positivity = b ? 1 : 0; }
  void SetNumberOfProjectionsPerSubset(int n) { m_P.projections_per_subset = n; }
  void SetDisableDisplacedDetectorFilter(bool d) { m_P.disable_displaced_detector = d ? 1 : 0; }
  void SetDivisionThreshold(double t) { m_P.division_threshold = t; }
  /* processing order (a permutation of the stack's projections), or a seed for a shuffled one */
  void SetOrder(std::vector<int> o) { m_Order = std::move(o); }
  void SetSeed(unsigned long long s) { m_P.seed = s; }
  void
  Update()
  {
    m_P.order = m_Order.empty() ? nullptr : m_Order.data();
    Check(rtkb_sart(m_Geometry, &m_Vol, &m_Proj, m_ProjIn, m_VolOut, &m_P, m_Stream), "SARTConeBeamReconstructionFilter");
  }

private:
  rtkb_sart_params m_P;
  std::vector<int> m_Order;
};

/* rtk::OSEMConeBeamReconstructionFilter (RTK's defaults), in place on the volume output buffer */
class OSEMConeBeamReconstructionFilter : public ProjectorBase
{
public:
  OSEMConeBeamReconstructionFilter() { m_P = { 3, 1, 0., 1, RTKB_OSEM_BP_VOXEL, nullptr, 0ULL }; }
  void SetNumberOfIterations(int n) { m_P.niter = n; }
  void SetNumberOfProjectionsPerSubset(int n) { m_P.projections_per_subset = n; }
  void SetBetaRegularization(double b) { m_P.beta = b; }
  void SetStoreNormalizationImages(bool s) { m_P.store_normalization = s ? 1 : 0; }
  /* RTKB_OSEM_BP_VOXEL (BP_VOXELBASED) or RTKB_OSEM_BP_JOSEPH (BP_JOSEPH) */
  void SetBackProjectionFilter(int bp) { m_P.backprojector = bp; }
  void SetOrder(std::vector<int> o) { m_Order = std::move(o); }
  void SetSeed(unsigned long long s) { m_P.seed = s; }
  void
  Update()
  {
    m_P.order = m_Order.empty() ? nullptr : m_Order.data();
    Check(rtkb_osem(m_Geometry, &m_Vol, &m_Proj, m_ProjIn, m_VolOut, &m_P, m_Stream), "OSEMConeBeamReconstructionFilter");
  }

private:
  rtkb_osem_params m_P;
  std::vector<int> m_Order;
};

/* rtk::IterativeFDKConeBeamReconstructionFilter (RTK's defaults), in place on the volume output buffer */
class IterativeFDKConeBeamReconstructionFilter : public ProjectorBase
{
public:
  IterativeFDKConeBeamReconstructionFilter()
  {
    m_P = {};
    m_P.niter = 3;
    m_P.lambda = 0.3;
    m_P.fdk.displaced_detector = 1;
    m_P.fdk.pad_on_truncated_side = 1;
    m_P.fdk.short_scan = 1;
    m_P.fdk.angular_gap_threshold = 3.14159265358979323846 / 9.;
    m_P.fdk.ramp = { 0., 0., 0., 0., 0., 0., 2, 2, 0., 2 }; // no window, no truncation correction; powers of 2, zero pad x2
  }
  void SetNumberOfIterations(int n) { m_P.niter = n; }
  void SetLambda(double l) { m_P.lambda = l; }
  void SetEnforcePositivity(bool b) { m_P.positivity = b ? 1 : 0; }
  void SetDisableDisplacedDetectorFilter(bool d) { m_P.fdk.displaced_detector = d ? 0 : 1; }
  void SetTruncationCorrection(double t) { m_P.fdk.ramp.truncation_correction = t; }
  void SetHannCutFrequency(double h) { m_P.fdk.ramp.hann_cut = h; }
  void SetHannCutFrequencyY(double h) { m_P.fdk.ramp.hann_cut_y = h; }
  void
  Update()
  {
    Check(rtkb_iterative_fdk(m_Geometry, &m_Vol, &m_Proj, m_ProjIn, m_VolOut, &m_P, m_Stream),
          "IterativeFDKConeBeamReconstructionFilter");
  }

private:
  rtkb_iterative_fdk_params m_P;
};

/* rtk::RegularizedConjugateGradientConeBeamReconstructionFilter (RTK's defaults; no wavelets step),
 * in place on the volume output buffer; Update() waits for the stream */
class RegularizedConjugateGradientConeBeamReconstructionFilter : public ProjectorBase
{
public:
  RegularizedConjugateGradientConeBeamReconstructionFilter()
  {
    m_P = { 10, 4, 0., 0., 1, 1, 5e-5, 10, nullptr, 0, 1e-3, 0, nullptr };
  }
  void SetMainLoop_iterations(int n) { m_P.main_loop_iterations = n; }
  void SetCG_iterations(int n) { m_P.cg_iterations = n; }
  void SetTikhonov(double t) { m_P.tikhonov = t; }
  void SetGamma(double g) { m_P.gamma = g; }
  void SetPerformPositivity(bool b) { m_P.positivity = b ? 1 : 0; }
  void SetPerformTVSpatialDenoising(bool b) { m_P.tv = b ? 1 : 0; }
  void SetGammaTV(double g) { m_P.gamma_tv = g; }
  void SetTV_iterations(int n) { m_P.tv_iterations = n; }
  void
  SetDimensionsProcessedForTV(const bool dims[3])
  {
    for (int d = 0; d < 3; d++)
      m_Dims[d] = dims[d] ? 1 : 0;
    m_P.tv_dimensions = m_Dims;
  }
  void SetPerformSoftThresholdOnImage(bool b) { m_P.soft_threshold_on_image = b ? 1 : 0; }
  void SetSoftThresholdOnImage(double t) { m_P.soft_threshold = t; }
  void SetDisableDisplacedDetectorFilter(bool d) { m_P.disable_displaced_detector = d ? 1 : 0; }
  void SetSupportMask(const float * m) { m_P.support_mask = m; }
  void SetInputWeights(const float * w) { m_Weights = w; }
  void
  Update()
  {
    Check(rtkb_regularized_cg(m_Geometry, &m_Vol, &m_Proj, m_ProjIn, m_Weights, m_VolOut, &m_P, m_Stream),
          "RegularizedConjugateGradientConeBeamReconstructionFilter");
  }

private:
  rtkb_regularized_cg_params m_P;
  int                        m_Dims[3] = { 1, 1, 1 };
  const float *              m_Weights = nullptr;
};

/* rtk::TotalVariationDenoisingBPDQImageFilter on a device volume (out may equal in) */
class TotalVariationDenoisingBPDQImageFilter
{
public:
  void SetInput(const rtkb_image_desc & d, const float * in) { m_Desc = d; m_In = in; }
  void SetOutput(float * out) { m_Out = out; }
  void SetGamma(double g) { m_Gamma = g; }
  void SetNumberOfIterations(int n) { m_Iterations = n; }
  void
  SetDimensionsProcessed(const bool dims[3])
  {
    for (int d = 0; d < 3; d++)
      m_Dims[d] = dims[d] ? 1 : 0;
  }
  void SetStream(void * s) { m_Stream = s; }
  void
  Update()
  {
    Check(rtkb_tv_denoising_bpdq(&m_Desc, m_In, m_Out, m_Gamma, m_Iterations, m_Dims, m_Stream),
          "TotalVariationDenoisingBPDQImageFilter");
  }

private:
  rtkb_image_desc m_Desc{};
  const float *   m_In = nullptr;
  float *         m_Out = nullptr;
  double          m_Gamma = 1.;
  int             m_Iterations = 1;
  int             m_Dims[3] = { 1, 1, 1 };
  void *          m_Stream = nullptr;
};

/* rtk::I0EstimationProjectionFilter on a device 16-bit raw image (waits for the stream) */
class I0EstimationProjectionFilter
{
public:
  void SetInput(const rtkb_image_desc & d, const unsigned short * raw) { m_Desc = d; m_Raw = raw; }
  void SetBitShift(int b) { m_Shift = b; }
  void SetDynThreshold(unsigned int t) { m_Threshold = t; }
  void SetStream(void * s) { m_Stream = s; }
  void
  Update()
  {
    Check(rtkb_i0_estimation(&m_Desc, m_Raw, m_Shift, m_Threshold, &m_Estimate, m_Stream),
          "I0EstimationProjectionFilter");
  }
  double GetI0() const { return m_Estimate.i0; }
  double GetI0fwhm() const { return m_Estimate.i0_fwhm; }
  const rtkb_i0_estimate & GetEstimate() const { return m_Estimate; }

private:
  rtkb_image_desc        m_Desc{};
  const unsigned short * m_Raw = nullptr;
  int                    m_Shift = 2;
  unsigned int           m_Threshold = 20;
  rtkb_i0_estimate       m_Estimate{};
  void *                 m_Stream = nullptr;
};

/* rtk::LUTbasedVariableI0RawToAttenuationImageFilter: device 16-bit raw in, float line integrals out */
class LUTbasedVariableI0RawToAttenuationImageFilter
{
public:
  void SetInput(const rtkb_image_desc & d, const unsigned short * raw) { m_Desc = d; m_Raw = raw; }
  void SetOutput(float * out) { m_Out = out; }
  void SetI0(double i0) { m_I0 = i0; }
  void SetIDark(double d) { m_IDark = d; }
  void SetStream(void * s) { m_Stream = s; }
  void
  Update()
  {
    Check(rtkb_raw_to_attenuation(&m_Desc, m_Raw, m_I0, m_IDark, m_Out, m_Stream),
          "LUTbasedVariableI0RawToAttenuationImageFilter");
  }

private:
  rtkb_image_desc        m_Desc{};
  const unsigned short * m_Raw = nullptr;
  float *                m_Out = nullptr;
  double                 m_I0 = 65535., m_IDark = 0.;
  void *                 m_Stream = nullptr;
};

/* rtk::WaterPrecorrectionImageFilter on device line integrals (out may equal in) */
class WaterPrecorrectionImageFilter
{
public:
  void SetInput(const rtkb_image_desc & d, const float * in) { m_Desc = d; m_In = in; }
  void SetOutput(float * out) { m_Out = out; }
  void SetCoefficients(std::vector<double> c) { m_C = std::move(c); }
  void SetStream(void * s) { m_Stream = s; }
  void
  Update()
  {
    Check(rtkb_water_precorrection(&m_Desc, m_In, m_Out, m_C.data(), (int)m_C.size(), m_Stream),
          "WaterPrecorrectionImageFilter");
  }

private:
  rtkb_image_desc     m_Desc{};
  const float *       m_In = nullptr;
  float *             m_Out = nullptr;
  std::vector<double> m_C{ 0., 1. };
  void *              m_Stream = nullptr;
};

} // namespace rtkb

#endif

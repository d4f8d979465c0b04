// rtkb_filters.h -- internal declarations of the projection-domain filters
// (FDK weighting, Parker, displaced detector, ramp).
#pragma once

#include "rtkb_internal.h"

namespace rtkb
{

// Per-projection FDK weighting parameters (FP64):
// [0] factor, [1] numpart1, [2] sin(tilt), [3] sdd*tan(tilt), [4] sdd^2,
// [5] x of column 0, [6] y of row 0, [7] parallel flag, [8] x step, [9] y step.
constexpr int kFdkWeightParams = 10;
void fdk_weight_params(const Geometry & g, const rtkb_image_desc & proj, std::vector<double> & out);

// Parker weights per (projection, column); false when the scan is not short.
bool parker_weights(const Geometry & g, const rtkb_image_desc & proj, double threshold, std::vector<float> & w);

struct DisplacedInfo
{
  rtkb_image_desc out; // output image (x doubled on the truncated side when padded)
  bool            weighted;
  int             shift; // output column of input column 0
  double          inf, sup;
  // DisplacedDetectorForOffsetFieldOfViewImageFilter: the field of view's disc
  bool            offset_fov = false;
  double          fov_x = 0., fov_z = 0., fov_r = -1.;
};
// FieldOfViewImageFilter::ComputeFOVRadius: type 0 RADIUSINF, 1 RADIUSSUP,
// 2 RADIUSBOTH; RTKB_OK with the disc, an error code when there is none
int  fov_radius(const Geometry & g, const rtkb_image_desc & proj, int type, double & x, double & z, double & r);
int  offset_fov_region(const Geometry & g, const rtkb_image_desc & proj, DisplacedInfo & info);
void offset_fov_weights(const Geometry & g, const rtkb_image_desc & proj, const DisplacedInfo & info,
                        std::vector<float> & w);
int  displaced_region(const Geometry & g, const rtkb_image_desc & proj, bool pad, DisplacedInfo & info);
void displaced_weights(const Geometry & g, const rtkb_image_desc & proj, const DisplacedInfo & info,
                       std::vector<float> & w);

int  ramp_padded_size(int nu, const rtkb_ramp_params & p);
int  ramp_padded_size_y(int nv, const rtkb_ramp_params & p); // nv without the 2-D kernel
void ramp_window_y(int padded_y, const rtkb_ramp_params & p, std::vector<double> & w); // padded_y/2+1
// FFT length for a circular convolution of period P: P itself when a power of
// two, else the power of two >= 2P - 1 that embed_spectrum targets
int  fft_length_for_period(int P);
// spectrum (M/2+1) on a length-M FFT of the even period-P kernel K (P/2+1)
void embed_spectrum(int P, int M, const std::vector<double> & K, std::vector<double> & KM);
void ramp_kernel(int padded, double spacing, const rtkb_ramp_params & p, std::vector<double> & K);
void twiddles(int n, std::vector<float> & tw);
void truncation_mirror_weights(int next, std::vector<float> & mw);

} // namespace rtkb

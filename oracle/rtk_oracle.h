/*
 * rtk_oracle.h -- FP64 CPU restatement of RTK's projector pair, FDK weighting,
 * ramp filtering, Parker / displaced-detector weighting and conjugate gradient.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA product
 * in rtk_b200/.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.  The product never links or calls it.
 *
 * Parity status: partially pinned.  ITK is absent, so RTK's own filters cannot
 * be built or run here.  The geometry is pinned exactly against the two
 * known-answer matrices published in RTK's documentation/docs/Geometry.md.
 * The operators are pinned against RTK's own analytic tests with RTK's
 * thresholds (FDK of the Shepp-Logan phantom, Joseph projection of a box
 * against ray-box lengths, Joseph FP/BP adjointness), and each function cites
 * the reference file:line it restates.
 *
 * Image convention (ITK): data are row-major with x fastest: a volume is
 * [z][y][x], a projection stack [projection][v][u].  An image descriptor holds
 * the largest-possible region (index, size), origin, spacing and direction.
 */
#ifndef RTK_ORACLE_H
#define RTK_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_image
{
  int    size[3];
  int    index[3];
  double origin[3];
  double spacing[3];
  double direction[9]; /* row-major 3x3 */
} orc_image;

typedef struct orc_geometry orc_geometry;

/* ---- geometry (src/rtkThreeDCircularProjectionGeometry.cxx) ---- */
orc_geometry * orc_geometry_new(void);
/* SetRadiusCylindricalDetector (0: flat panel) */
void orc_geometry_set_radius_cylindrical(orc_geometry * g, double radius);
void           orc_geometry_free(orc_geometry * g);
int            orc_geometry_add_projection(orc_geometry * g, double sid, double sdd, double gantry_deg,
                                           double proj_offset_x, double proj_offset_y, double out_of_plane_deg,
                                           double in_plane_deg, double source_offset_x, double source_offset_y);
int            orc_geometry_add_projection_rad(orc_geometry * g, double sid, double sdd, double gantry,
                                               double proj_offset_x, double proj_offset_y, double out_of_plane,
                                               double in_plane, double source_offset_x, double source_offset_y);
int            orc_geometry_size(const orc_geometry * g);
void           orc_geometry_matrix(const orc_geometry * g, int i, double m[12]);
void           orc_geometry_source_position(const orc_geometry * g, int i, double s[4]);
void           orc_geometry_proj_coords_to_fixed(const orc_geometry * g, int i, double m[16]);
void           orc_geometry_parameters(const orc_geometry * g, int i, double p[10]);
void           orc_geometry_source_angles(const orc_geometry * g, double * out);
void           orc_geometry_gantry_angles(const orc_geometry * g, double * out);
void           orc_geometry_tilt_angles(const orc_geometry * g, double * out);
void           orc_geometry_angular_gaps(const orc_geometry * g, const double * angles, double * out);
void           orc_geometry_angular_gaps_with_next(const orc_geometry * g, const double * angles, double * out);
double         orc_geometry_to_untilted(const orc_geometry * g, int i, double tilted);

/* ---- image index <-> physical (include/rtkHomogeneousMatrix.h:38-81) ---- */
void orc_index_to_physical(const orc_image * im, double m[16]);
void orc_physical_to_index(const orc_image * im, double m[16]);

/* ---- backprojection (include/rtkBackProjectionImageFilter.hxx,
 *      include/rtkFDKBackProjectionImageFilter.hxx) ---- */
/* Index-to-index matrix of projection i (volume index -> projection index),
 * untransposed, FDK-normalised when fdk != 0.  Returns the path RTK takes:
 * 1 = optimised X, 2 = optimised Y, 0 = generic interpolator path. */
int  orc_bp_matrix(const orc_geometry * g, const orc_image * vol, const orc_image * proj, int i, int fdk,
                   double m[12]);
/* Independent voxel -> pixel map (the ray from the source through the
 * physical point meets the detector plane, from the source position and the
 * detector frame): out = (u, v) absolute continuous projection index of
 * projection k, and the FDK weight (1 when fdk == 0); returns the path mode as
 * orc_bp_matrix does.  orc_backproject uses this map for flat panels. */
int  orc_bp_project(const orc_geometry * g, const orc_image * vol, const orc_image * proj, int k, int fdk,
                    const double * physical, double out[3]);
/* vol_out = vol_in + sum over projections.  proj data = stack buffer; stack
 * slice s is geometry projection proj->index[2] + s. */
void orc_backproject(const orc_geometry * g, const orc_image * vol, const orc_image * proj, const double * proj_data,
                     const double * vol_in, double * vol_out, int fdk, int nthreads);

/* ---- Joseph projector pair (include/rtkJosephForwardProjectionImageFilter.hxx,
 *      include/rtkJosephBackProjectionImageFilter.hxx) ---- */
void   orc_joseph_forward(const orc_geometry * g, const orc_image * vol, const double * vol_data,
                          const orc_image * proj, const double * proj_in, double * proj_out, int nthreads);
void   orc_joseph_back(const orc_geometry * g, const orc_image * vol, const double * vol_in, double * vol_out,
                       const orc_image * proj, const double * proj_data);
/* the same back projection split over nthreads (FP64 partial volumes) */
void   orc_joseph_back_mt(const orc_geometry * g, const orc_image * vol, const double * vol_in, double * vol_out,
                          const orc_image * proj, const double * proj_data, int nthreads);
/* Number of bilinear samples the Joseph forward projector takes (work count). */
double orc_joseph_sample_count(const orc_geometry * g, const orc_image * vol, const orc_image * proj, int nthreads);

/* ---- projection weighting ---- */
void orc_fdk_weight(const orc_geometry * g, const orc_image * proj, const double * in, double * out);
/* returns 1 when the scan is a short scan (weights applied), 0 otherwise */
/* Parker's short-scan detection, delta and first gantry angle (returns 1 for a short scan) */
int    orc_parker_params(const orc_geometry * g, double threshold, double * delta, double * first_angle);
int  orc_parker_weight(const orc_geometry * g, const orc_image * proj, double angular_gap_threshold,
                       const double * in, double * out);
/* Computes the displaced-detector output region. out_index0/out_size0 receive the
 * output's x index/size.  Returns 0 when not displaced (copy), 1 when weighted,
 * -1 on error (displacement larger than half the panel). */
int  orc_displaced_detector_region(const orc_geometry * g, const orc_image * proj, int pad_on_truncated_side,
                                   int * out_index0, int * out_size0, double * inf_corner, double * sup_corner);
int  orc_displaced_detector(const orc_geometry * g, const orc_image * proj, int pad_on_truncated_side,
                            const double * in, double * out);

/* ---- ramp filter (include/rtkFFTRampImageFilter.hxx,
 *      include/rtkFFTProjectionsConvolutionImageFilter.hxx) ---- */
typedef struct orc_ramp_params
{
  double hann_cut;
  double cosine_cut;
  double hamming;
  double ramlak_cut;
  double shepplogan_cut;
  double truncation_correction;
  int    greatest_prime_factor; /* 2 without FFTW, 13 with */
  int    zero_pad_factor;       /* 2 */
  double hann_cut_y;            /* HannCutFrequencyY: > 0 makes the kernel 2-D */
  int    zero_pad_factor_y;     /* ZeroPadFactors[1], used with the 2-D kernel; <= 0 means 2 */
} orc_ramp_params;
int  orc_ramp_padded_size(int nu, const orc_ramp_params * p);
/* padded height with the 2-D kernel (hann_cut_y > 0), else nv */
int  orc_ramp_padded_size_y(int nv, const orc_ramp_params * p);
/* vertical window of the 2-D kernel, w[j] for j = 0..padded_y/2 (row j and
 * row padded_y - j of the kernel carry w[j]) */
void orc_ramp_window_y(int padded_y, const orc_ramp_params * p, double * w);
/* frequency-domain kernel, length padded/2+1, real (the spatial kernel is even) */
void orc_ramp_kernel(int padded, double spacing, const orc_ramp_params * p, double * kernel);
void orc_ramp_filter(const orc_image * proj, const orc_ramp_params * p, const double * in, double * out,
                     int nthreads);

/* ---- conjugate gradient (include/rtkConjugateGradientImageFilter.hxx,
 *      include/rtkReconstructionConjugateGradientOperator.hxx) ---- */
/* A x = BP(W .* FP(x)) + tikhonov * x with the Joseph pair; b = BP(W .* p).
 * Runs niter iterations from x (in/out).  residuals[k] = ||r_k||^2 for
 * k = 0..niter (may be NULL).  weights may be NULL (all ones). */
/* orc_cg_joseph with the back projector chosen as RTK's iterative filters
 * choose it: backprojector 0 = Joseph, 1 = voxel-based (not the exact adjoint
 * of the Joseph forward projector; RTK's rtkconjugategradient default). */
void orc_cg(const orc_geometry * g, const orc_image * vol, const orc_image * proj, const double * proj_data,
            const double * weights, const double * mask, double tikhonov, double gamma, int niter, double * x,
            double * residuals, int backprojector, int nthreads);
void orc_cg_joseph(const orc_geometry * g, const orc_image * vol, const orc_image * proj, const double * proj_data,
                   const double * weights, const double * mask, double tikhonov, double gamma, int niter, double * x,
                   double * residuals, int nthreads);
/* RayBoxIntersectionImageFilter with SetBoxFromImage(vol, false): per-pixel length (mm) of the ray in the box */
void orc_ray_box(const orc_geometry * g, const orc_image * vol, const orc_image * proj, double * out, int nthreads);
/* the same for the box between two corners (SetBoxMin / SetBoxMax) */
void orc_ray_box_corners(const orc_geometry * g, const orc_image * proj, const double * bmin, const double * bmax,
                         double * out, int nthreads);
/* SARTConeBeamReconstructionFilter with the Joseph forward and voxel-based back projectors, in place on x */
void orc_sart(const orc_geometry * g, const orc_image * vol, const orc_image * proj, const double * proj_data, double * x,
              int niter, double lambda, int positivity, int projections_per_subset, int displaced_detector,
              double threshold, const int * order, int nthreads);
/* DePierroRegularizationImageFilter: out = (A + sqrt(A^2 + 8 beta 26 update)) / 2,
 * A = norm - beta K(xk), K the 26-neighbour sum plus 26 xk (zero outside); norm may be NULL (ones) */
void orc_de_pierro(const orc_image * vol, const double * xk, const double * update, const double * norm, double beta,
                   double * out);
/* OSEMConeBeamReconstructionFilter with the Joseph forward projector and the voxel-based (joseph_bp = 0) or Joseph
 * back projector, in place on x */
void orc_osem(const orc_geometry * g, const orc_image * vol, const orc_image * proj, const double * proj_data, double * x,
              int niter, int projections_per_subset, double beta, int joseph_bp, const int * order, int nthreads);
/* TotalVariationDenoisingBPDQImageFilter: niter >= 1 iterations, dims: processed dimensions (0/1) */
void orc_tv_denoising_bpdq(const orc_image * vol, const double * f, double * out, double gamma, int niter,
                           const int dims[3]);
/* TotalVariationImageFilter: sum of forward-difference gradient norms */
double orc_total_variation(const orc_image * vol, const double * x);
/* RegularizedConjugateGradientConeBeamReconstructionFilter with the Joseph pair (CG, positivity, TV, soft
 * threshold on the image), in place on x; weights = the CG's W or NULL */
void orc_regularized_cg(const orc_geometry * g, const orc_image * vol, const orc_image * proj, const double * proj_data,
                        const double * weights, const double * mask, double * x, int main_iterations, int cg_iterations, double tikhonov,
                        double gamma, int positivity, int tv, double gamma_tv, int tv_iterations, const int tv_dims[3],
                        int soft_threshold, double soft_threshold_value, int nthreads);
/* I0EstimationProjectionFilter on n 16-bit pixels: out = I0, I0 FWHM, Imin, Imax, low bound, high bound */
void orc_i0_estimation(const unsigned short * raw, long n, int shift, unsigned int dyn_threshold, double out[6]);
/* LUTbasedVariableI0RawToAttenuationImageFilter: out = lut[raw] */
void orc_raw_to_attenuation(const unsigned short * raw, long n, double i0, double idark, float * out);
/* RTK's LaplacianImageFilter (Neumann boundary, spacing-scaled): out = Laplacian(x) */
void orc_laplacian(const orc_image * vol, const double * x, double * out);

/* ---- phantoms (test input generators; src/rtkQuadricShape.cxx semantics) ---- */
/* ellipsoids: per ellipsoid 16 doubles: cx cy cz, ax ay az, R (3x3 row-major, local->world), density */
void orc_project_ellipsoids(const orc_geometry * g, const orc_image * proj, int n_ell, const double * ell,
                            double * proj_out, int nthreads);
void orc_draw_ellipsoids(const orc_image * vol, int n_ell, const double * ell, double * vol_out, int nthreads);

/* ---- timed CPU baseline: RTK's CPU FDK backprojector as RTK runs it (FP32 data,
 * FP64 coordinates, transposed projections, OptimizedBackprojectionY loop order),
 * over nthreads threads splitting the volume along z. ---- */
int orc_fdk_backproject_f32_rtk(const orc_geometry * g, const orc_image * vol, const orc_image * proj,
                                const float * proj_data, float * vol_inout, int nthreads);

#ifdef __cplusplus
}
#endif
#endif

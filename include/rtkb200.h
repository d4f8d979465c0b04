/*
 * rtkb200.h -- C ABI of the B200-native RTK hot path (librtkb200.so).
 *
 * Every entry point is extern "C", takes plain pointers and sizes, returns an
 * int status (RTKB_OK on success) and never throws.  The message of the last
 * failure on the calling host thread is returned by rtkb_last_error().
 *
 * Buffers: all d_* arguments are caller-owned device pointers to float32
 * images in ITK layout (row-major, x fastest: volume [z][y][x], projection
 * stack [projection][v][u]).  Kernels are enqueued on the caller's stream
 * (a cudaStream_t passed as void*, NULL = legacy default stream) and return
 * without synchronising.  Calls on different streams are independent: there is
 * no process-global __constant__ state, unlike the entry points they replace.
 *
 * Images are described by rtkb_image_desc: the largest-possible region
 * (index, size), origin, spacing and direction, as ITK holds them.  Slice s of
 * a projection stack is geometry projection index[2] + s, as in RTK filters
 * whose input stack starts at a non-zero projection index.
 *
 * Reference interfaces replaced (paths in the RTK repository):
 *   CUDA_reconstruct_conebeam   include/rtkCudaFDKBackProjectionImageFilter.hcu:22-29
 *   CUDA_back_project           src/rtkCudaBackProjectionImageFilter.cu:125-135
 *   CUDA_forward_project        include/rtkCudaForwardProjectionImageFilter.hcu:24-38
 *   CUDA_ray_cast_back_project  src/rtkCudaRayCastBackProjectionImageFilter.cu:186-199
 *   CUDA_weight_projection      src/rtkCudaFDKWeightProjectionFilter.cu:85-95
 *   CUDA_parker_weight          src/rtkCudaParkerShortScanImageFilter.cu:106-118
 *   CUDA_displaced_weight       src/rtkCudaDisplacedDetectorImageFilter.cu:132-185
 *   CUDA_padding / CUDA_fft_convolution
 *                               src/rtkCudaFFTProjectionsConvolutionImageFilter.cu:70-75,175-181
 *   CUDA_conjugate_gradient     src/rtkCudaConjugateGradientImageFilter.cu:80-166
 */
#ifndef RTKB200_H
#define RTKB200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define RTKB_OK 0
#define RTKB_ERR_INVALID_ARGUMENT 1
#define RTKB_ERR_CUDA 2
#define RTKB_ERR_UNSUPPORTED 3
#define RTKB_ERR_TIMEOUT 4
#define RTKB_ERR_OUT_OF_MEMORY 5

/* ---- image description (itk::ImageBase metadata) ---- */
typedef struct rtkb_image_desc
{
  int    size[3];      /* largest-possible region size, x y z */
  int    index[3];     /* largest-possible region start index */
  double origin[3];    /* physical position of index (0,0,0) */
  double spacing[3];   /* pixel spacing */
  double direction[9]; /* row-major direction cosines */
} rtkb_image_desc;

/* ---- library ---- */
/* Message of the last failure on this host thread ("" if none). */
const char * rtkb_last_error(void);
/* Library version string. */
const char * rtkb_version(void);
/* Waits for `stream`, then reads and clears the device-side status word that
 * kernels set when a bounded wait gives up or an internal check fails.
 * *status receives 0 when no kernel reported a problem, RTKB_ERR_TIMEOUT when a
 * wait gave up, RTKB_ERR_CUDA for a failed internal check. */
int rtkb_device_status(void * stream, int * status);
/* Temporary device memory of every entry point comes from one stream-ordered
 * memory pool per device that the library owns; memory freed there stays
 * reserved for later calls (the caller's default pool is not touched).
 * rtkb_trim_memory_pool returns the unused part to the driver (*reserved_after,
 * may be NULL: bytes still reserved, those of work not yet finished in stream
 * order); rtkb_memory_pool_reserved reads the reserved size.  Current device.
 * No reference counterpart (ITK's CUDA images allocate per image). */
int rtkb_trim_memory_pool(long long * reserved_after);
int rtkb_memory_pool_reserved(long long * reserved);

/* ---- failure detection (testing aids; no counterpart in the reference, whose
 * CUDA_CHECK_ERROR, include/rtkCudaUtilities.hcu:30-35, only reports launch
 * errors) ----
 * rtkb_device_status reports RTKB_ERR_TIMEOUT when a bounded device-side wait
 * gave up.  rtkb_set_wait_limit sets how many polls such a wait makes before
 * it gives up (default 4194304, about a second or more; current device;
 * *previous may be NULL).  rtkb_wait_self_test launches one CTA whose bounded
 * wait is on an mbarrier that nobody arrives at: it gives up after the limit,
 * records the timeout and returns, leaving the context usable.
 * rtkb_inject_allocation_failures makes the library's next `count` scratch
 * allocations fail as if the device were out of memory, which exercises the
 * pool's trim-and-retry path (a failed retry is returned to the caller as an
 * error before any of the call's kernels is enqueued). */
int rtkb_set_wait_limit(unsigned int polls, unsigned int * previous);
int rtkb_wait_self_test(void * stream);
int rtkb_inject_allocation_failures(int count);

/* ---- geometry: rtk::ThreeDCircularProjectionGeometry, FP64 ----
 * src/rtkThreeDCircularProjectionGeometry.cxx:56-153 (AddProjection),
 * :407-663 (getters).  Angles in degrees for add_projection, radians for
 * add_projection_in_radians, as RTK. */
typedef struct rtkb_geometry rtkb_geometry;
rtkb_geometry * rtkb_geometry_new(void);
void            rtkb_geometry_free(rtkb_geometry * g);
int             rtkb_geometry_add_projection(rtkb_geometry * g, double sid, double sdd, double gantry_angle,
                                             double proj_offset_x, double proj_offset_y, double out_of_plane_angle,
                                             double in_plane_angle, double source_offset_x, double source_offset_y);
int             rtkb_geometry_add_projection_in_radians(rtkb_geometry * g, double sid, double sdd,
                                                        double gantry_angle, double proj_offset_x,
                                                        double proj_offset_y, double out_of_plane_angle,
                                                        double in_plane_angle, double source_offset_x,
                                                        double source_offset_y);
int             rtkb_geometry_number_of_projections(const rtkb_geometry * g);
/* 3x4 projection matrix of projection i (GetMatrices()[i]), row-major */
int             rtkb_geometry_get_matrix(const rtkb_geometry * g, int i, double out[12]);
/* homogeneous source position (GetSourcePosition(i)) */
int             rtkb_geometry_get_source_position(const rtkb_geometry * g, int i, double out[4]);
/* GetProjectionCoordinatesToFixedSystemMatrix(i), row-major 4x4 */
int             rtkb_geometry_get_projection_coordinates_to_fixed_system_matrix(const rtkb_geometry * g, int i,
                                                                                double out[16]);
/* which: 0 gantry, 1 source, 2 tilt, 3 out-of-plane, 4 in-plane angles (radians);
 * 5 SID, 6 SDD, 7 projection offsets X, 8 Y, 9 source offsets X, 10 Y;
 * 11 angular gaps of the source angles (GetAngularGaps(GetSourceAngles()));
 * 12-15 collimation U inf, U sup, V inf, V sup (DBL_MAX: unbounded) */
int             rtkb_geometry_get_parameters(const rtkb_geometry * g, int which, double * out);
/* SetCollimationOfLastProjection */
int             rtkb_geometry_set_collimation_of_last_projection(rtkb_geometry * g, double uinf, double usup,
                                                                 double vinf, double vsup);
/* rtk::ThreeDCircularProjectionGeometryXMLFileReader / rtk::ReadGeometry
 * (src/rtkThreeDCircularProjectionGeometryXMLFileReader.cxx): *out receives a
 * new geometry (free with rtkb_geometry_free); versions 3 and 2; a stored
 * matrix that differs from the recomputed one by more than 0.001 is an error.
 * rtk::ThreeDCircularProjectionGeometryXMLFileWriter
 * (src/rtkThreeDCircularProjectionGeometryXMLFileWriter.cxx): version 3, 15
 * significant digits, parameters equal over all projections written once. */
int             rtkb_geometry_read_xml(const char * filename, rtkb_geometry ** out);
int             rtkb_geometry_write_xml(const rtkb_geometry * g, const char * filename);
double          rtkb_geometry_to_untilted_coordinate_at_isocenter(const rtkb_geometry * g, int i, double tilted);
int             rtkb_geometry_set_radius_cylindrical_detector(rtkb_geometry * g, double radius);

/* ---- image files ----
 * MetaImage (.mha: header and data in one file; .mhd: data in a .raw/.zraw
 * beside it), the format RTK's applications read and write through ITK's
 * MetaImageIO.  Read: fills *desc (index 0, origin = the file's Offset) and,
 * when data is not NULL, converts the voxels (float, double, 8/16/32-bit
 * integers, either byte order, zlib-compressed or not) to float32 in data
 * (x fastest; capacity in voxels).  Write: float32, zlib-compressed when
 * compress != 0; Offset = the physical position of the region's first voxel. */
int rtkb_image_read_mha(const char * filename, rtkb_image_desc * desc, float * data, long long capacity);
int rtkb_image_write_mha(const char * filename, const rtkb_image_desc * desc, const float * data, int compress);

/* Volume-index -> projection-index matrices (3x4, row-major, untransposed) of
 * stack slices first..first+n-1 as BackProjectionImageFilter builds them
 * (include/rtkBackProjectionImageFilter.hxx:535-595), FDK-normalised when
 * fdk != 0 (include/rtkFDKBackProjectionImageFilter.hxx:80-104).  modes[s]
 * receives the path RTK takes: 1 optimised X, 2 optimised Y, 0 generic. */
int rtkb_backprojection_matrices(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                                 int first, int n, int fdk, double * out_matrices, int * modes);

/* ---- backprojection ----
 * rtk::FDKBackProjectionImageFilter / rtk::BackProjectionImageFilter:
 * d_vol_out = d_vol_in + sum over the stack of the (FDK-weighted) voxel-driven
 * bilinear backprojection.  d_vol_in may equal d_vol_out (in place). */
int rtkb_fdk_backproject(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                         const float * d_proj, const float * d_vol_in, float * d_vol_out, void * stream);
int rtkb_voxel_backproject(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                           const float * d_proj, const float * d_vol_in, float * d_vol_out, void * stream);
/* rtk::FDKBackProjectionImageFilter on host buffers, as RTK's CUDA pipeline
 * runs it from CPU images: the stack is streamed to the device in projection
 * subsets (include/rtkFDKConeBeamReconstructionFilter.hxx:116-157), each
 * copied on an internal stream into one of two device staging buffers while
 * the previous one is backprojected into a device copy of the volume.  The
 * subsets grow geometrically (x1.5) from chunk/12 to `chunk` projections
 * (chunk <= 0: a quarter of the stack), so that each copy hides behind the
 * previous subset's backprojection from the first, short one on; the last
 * subset takes the remainder (up to 1.5 chunk) and is backprojected in
 * z-slabs of whole 16-slice tile layers whose sizes halve (16, 8, 4, 2, 1, 1
 * layers of 32), each copied back while the next ones are computed (the
 * host<->device transfers ITK's CudaDataManager makes around
 * rtkCudaFDKBackProjectionImageFilter.cxx:34-125, overlapped).  h_vol_in may
 * be NULL (zero volume).  Asynchronous on `stream`
 * like cudaMemcpyAsync: h_vol_out is written when the stream reaches the end
 * of this work.  Pinned host buffers give full copy bandwidth and overlap. */
int rtkb_fdk_backproject_host(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                              const float * h_proj, const float * h_vol_in, float * h_vol_out, int chunk,
                              void * stream);
/* Batched backprojection (no counterpart in the reference): many independent
 * problems of uneven sizes in one persistent launch -- CTAs take (problem,
 * tile) work items from a shared queue until it is empty.  Each problem is a
 * full rtkb_fdk_backproject / rtkb_voxel_backproject call (its own geometry,
 * descriptions and buffers, float32 stacks).  config: backprojector
 * configuration (0..count-1 of rtkb_backproject_config) for the whole batch,
 * -1 for the first one whose box holds every problem's footprint;
 * *used_config (may be NULL) receives it.  Problems on RTK's generic path
 * (tilted detectors, rotated volumes) run as separate launches.  These one-shot
 * calls prepare, execute and release a batch and wait for `stream`. */
typedef struct rtkb_bp_problem
{
  const rtkb_geometry * geometry;
  rtkb_image_desc       vol, proj;
  const float *         d_proj;
  const float *         d_vol_in;
  float *               d_vol_out;
} rtkb_bp_problem;
int rtkb_fdk_backproject_batch(const rtkb_bp_problem * problems, int n, int config, int * used_config, void * stream);
int rtkb_voxel_backproject_batch(const rtkb_bp_problem * problems, int n, int config, int * used_config,
                                 void * stream);
/* Prepared batch: the host work (matrices, footprints, TMA descriptors,
 * device tables) done once; each execute is one persistent launch on
 * `stream` (asynchronous).  The problems' buffers must stay valid while the
 * batch is used.  rtkb_bp_batch_config returns the configuration it runs. */
typedef struct rtkb_bp_batch rtkb_bp_batch;
int  rtkb_bp_batch_create(const rtkb_bp_problem * problems, int n, int fdk, int config, rtkb_bp_batch ** batch);
int  rtkb_bp_batch_execute(rtkb_bp_batch * batch, void * stream);
int  rtkb_bp_batch_config(const rtkb_bp_batch * batch);
void rtkb_bp_batch_destroy(rtkb_bp_batch * batch);
/* Autotuner: times every backprojector configuration on this batch (a
 * prepared batch per configuration, one warm-up and `repeats` timed executes
 * each, CUDA events on `stream`) and returns
 * the fastest in *best_config (its time in *best_ms, every configuration's in
 * config_ms[count] when not NULL).  With n == 1 it times the single-problem
 * path (rtkb_fdk_backproject / rtkb_voxel_backproject with the configuration
 * forced), whose calls then take the result through rtkb_backproject_config.  Writes the problems' outputs, which must
 * not alias their inputs.  Use the result as `config` of the batch calls or
 * with rtkb_backproject_config for single calls. */
int rtkb_backproject_autotune(const rtkb_bp_problem * problems, int n, int fdk, int repeats, int * best_config,
                              double * best_ms, double * config_ms, void * stream);

/* BF16 storage variant (no counterpart in the reference, whose stacks are
 * float): the same backprojections from a bfloat16 projection stack
 * (d_proj_bf16, same layout; RTK's arithmetic with FP32 interpolation and
 * accumulation, FP32 volume).  Halves the stack's memory and bandwidth. */
int rtkb_fdk_backproject_bf16(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                              const void * d_proj_bf16, const float * d_vol_in, float * d_vol_out, void * stream);
int rtkb_voxel_backproject_bf16(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                                const void * d_proj_bf16, const float * d_vol_in, float * d_vol_out, void * stream);
/* d_out[i] = bfloat16(d_in[i]), round to nearest even, i < n. */
int rtkb_convert_to_bf16(const float * d_in, void * d_out, long long n, void * stream);
/* rtkb_fdk_backproject without device allocations (no counterpart in the
 * reference).  For callers that cannot allocate device memory during a
 * reconstruction: an application whose device memory is reserved by its own
 * allocator, or an on-line loop that must avoid cudaMalloc's implicit device
 * synchronisation.  Same arguments and results as rtkb_fdk_backproject; its
 * only scratch (the stack's FP64 matrices and path modes) is a file-scope
 * device array sized for at most 2048 projections (about 200 KB, held by every
 * GPU that loads the library until the process exits); larger stacks are
 * rejected with RTKB_ERR_INVALID_ARGUMENT.  It calls no cudaMalloc, cudaFree
 * or allocating library routine.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) with that device current,
 * and so does the first call after the device's context changed (after a
 * cudaDeviceReset the array lives at a new address); make that first call
 * before any stream capture.  All calls share the array
 * and it keeps the last call's contents: calls whose GPU work overlaps (other
 * streams, other host threads) race on it and must be serialised by the
 * caller. */
int rtkb_fdk_backproject_static_scratch(const rtkb_geometry * g, const rtkb_image_desc * vol,
                                        const rtkb_image_desc * proj, const float * d_proj, const float * d_vol_in,
                                        float * d_vol_out, void * stream);
/* Matrix-level form mirroring CUDA_reconstruct_conebeam: n_proj FP64
 * matrices (volume buffer index -> projection buffer index), modes as above,
 * weighting 1 = FDK (1/w^2), 0 = none. */
int rtkb_backproject_matrices(const int vol_size[3], const int proj_size[3], int n_proj, const double * matrices,
                              const int * modes, int weighting, const float * d_proj, const float * d_vol_in,
                              float * d_vol_out, void * stream);

/* ---- raw projections to line integrals ----
 * rtk::I0EstimationProjectionFilter (include/rtkI0EstimationProjectionFilter.hxx):
 * the unattenuated intensity I0 of a 16-bit raw image (any region the caller
 * passes: one projection or a stack) as the mode of the histogram of
 * raw >> bit_shift in the upper quarter of its dynamic range; the range ends
 * are the outermost bins holding more than dyn_threshold counts.  RTK's
 * defaults: bit_shift 2, dyn_threshold 20.  All values in raw units; waits
 * for `stream`. */
typedef struct rtkb_i0_estimate
{
  double i0;         /* GetI0() */
  double i0_fwhm;    /* GetI0fwhm(): width of the mode at half its count */
  double imin, imax; /* the consistent dynamic range (GetImin, GetImax) */
  double low_bound, high_bound;
} rtkb_i0_estimate;
int rtkb_i0_estimation(const rtkb_image_desc * desc, const unsigned short * d_raw, int bit_shift,
                       unsigned int dyn_threshold, rtkb_i0_estimate * out, void * stream);
/* rtk::LUTbasedVariableI0RawToAttenuationImageFilter
 * (include/rtkLUTbasedVariableI0RawToAttenuationImageFilter.hxx): d_out =
 * log(max(I0 - IDark, 1)) - log(max(raw - IDark, 1)) through RTK's float
 * lookup table (RTK's defaults: I0 = 65535, IDark = 0).  d_out float32 of
 * the same size as d_raw. */
int rtkb_raw_to_attenuation(const rtkb_image_desc * desc, const unsigned short * d_raw, double i0, double idark,
                            float * d_out, void * stream);
/* rtk::WaterPrecorrectionImageFilter (include/rtkWaterPrecorrectionImageFilter.hxx):
 * d_out = c0 + c1 v + c2 v^2 + ... of the line integrals v (at most 16
 * coefficients; RTK's default (0, 1) and a single 0 pass v through).  d_out may
 * equal d_in. */
int rtkb_water_precorrection(const rtkb_image_desc * desc, const float * d_in, float * d_out,
                             const double * coefficients, int n_coefficients, void * stream);

/* ---- Joseph projector pair ----
 * rtk::JosephForwardProjectionImageFilter
 * (include/rtkJosephForwardProjectionImageFilter.hxx:182-427):
 * d_proj_out = d_proj_in + line integrals of d_vol (one bilinear sample per
 * main-direction slice, partial end weights, times the step length in mm).
 * Replaces CUDA_forward_project.  d_proj_out may equal d_proj_in. */
int rtkb_joseph_forward_project(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                                const float * d_vol, const float * d_proj_in, float * d_proj_out, void * stream);
/* rtk::JosephBackProjectionImageFilter
 * (include/rtkJosephBackProjectionImageFilter.hxx:57-323): the exact adjoint
 * (bilinear splat), d_vol_out = d_vol_in + BP(d_proj).  Replaces
 * CUDA_ray_cast_back_project.  d_vol_out may equal d_vol_in. */
int rtkb_joseph_back_project(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                             const float * d_proj, const float * d_vol_in, float * d_vol_out, void * stream);

/* Number of bilinear samples rtkb_joseph_forward_project takes for these
 * images (the algorithmic work of the ray-cast throughput figure); waits for
 * `stream`.  No reference counterpart (RTK's tests count ray-box lengths). */
int rtkb_joseph_sample_count(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                             double * count, void * stream);

/* ---- conjugate gradient ----
 * rtk::ConjugateGradientConeBeamReconstructionFilter
 * (include/rtkConjugateGradientConeBeamReconstructionFilter.hxx:192-305) with
 * rtk::ConjugateGradientImageFilter's iteration
 * (include/rtkConjugateGradientImageFilter.hxx:108-258): normal equations
 * A x = b, A = BP(W .* FP(.)) + tikhonov I with the Joseph pair, b = BP(W .* p),
 * W = displaced-detector weights (no padding) of the input weights.  Vectors
 * FP32; dot products, alpha and beta FP64, kept on the device.  Replaces
 * CUDA_conjugate_gradient.
 *
 * A plan owns all device memory; one iteration is captured as a CUDA graph at
 * start (on a private stream) and replayed by rtkb_cg_iterate. */
typedef struct rtkb_cg_params
{
  double tikhonov;       /* Tikhonov weight (RTK's SetTikhonov), 0 = none */
  int    use_cuda_graph; /* 1: replay a captured iteration graph */
  int    storage;        /* precision study (no counterpart in the reference, whose images are float):
                            0: FP32; 1: BF16 storage of the normal-equation vectors (r, p, A p) and of the
                            projection-domain temporary; 2: BF16 storage of the direction p and of the
                            projection-domain temporary, r, A p and the iterate FP32 (the residual
                            recurrence stays in FP32).  FP32 arithmetic and FP64 dots, alpha and beta in
                            all; the iterate stays in the caller's FP32 buffer; FP32 plans only for the
                            learned preconditioner, the support mask and the voxel-based back projector */
  double gamma;          /* Laplacian regularisation weight (RTK's SetGamma): A x += gamma * (-Laplacian(x)) */
  int    backprojector;  /* IterativeConeBeamReconstructionFilter's BackProjectionType
                            (include/rtkIterativeConeBeamReconstructionFilter.h:80-88, .hxx:33-103), the back
                            projector of b = BP(W .* p) and of A x = BP(W .* FP(x)), with RTK's values:
                            0 = BP_VOXELBASED (RTK's default, and so that of zero-initialised parameters; FP32
                            storage and flat panels; not the exact adjoint of the forward projector),
                            1 = BP_JOSEPH (the Joseph forward projector's exact adjoint), 2 = BP_CUDAVOXELBASED
                            (the same voxel-based back projector here).  The forward projector is Joseph
                            (FP_JOSEPH) either way. */
} rtkb_cg_params;
/* rtk::LaplacianImageFilter / CudaLaplacianImageFilter (include/rtkLaplacianImageFilter.hxx;
 * src/rtkCudaLaplacianImageFilter.cu): d_out = Laplacian(d_in), the
 * backward-difference divergence of the forward-difference gradient with a
 * zero-flux Neumann boundary, spacing-scaled. */
int  rtkb_laplacian(const rtkb_image_desc * vol, const float * d_in, float * d_out, void * stream);
typedef struct rtkb_cg rtkb_cg;
int  rtkb_cg_create(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                    const rtkb_cg_params * params, rtkb_cg ** plan);
/* Binds the iterate d_x (holds x0 on entry, updated in place) and computes
 * r0 = b - A x0, p0 = r0.  d_weights may be NULL (all ones). */
int  rtkb_cg_start(rtkb_cg * plan, const float * d_proj, const float * d_weights, int displaced_detector, float * d_x,
                   void * stream);
/* As rtkb_cg_start, but for a given normal-equation right-hand side d_b
 * (a volume) instead of b = BP(W .* p); W keeps its current value (1 unless a
 * previous rtkb_cg_start set it).  No reference counterpart: used to run CG on
 * synthetic problems A x = b whose solution is known (training data of the
 * learned preconditioner). */
int  rtkb_cg_start_rhs(rtkb_cg * plan, const float * d_b, float * d_x, void * stream);
int  rtkb_cg_iterate(rtkb_cg * plan, int n, void * stream);
/* Support mask (ConjugateGradientConeBeamReconstructionFilter::SetSupportMask,
 * include/rtkConjugateGradientConeBeamReconstructionFilter.hxx:246-258 and
 * include/rtkReconstructionConjugateGradientOperator.hxx:203-262): with a
 * volume M, b = M .* BP(W .* p) and A x = M .* (BP(W .* FP(M .* x)) + gamma
 * (-Laplacian(M .* x)) + tikhonov M .* x); rtkb_cg_finish multiplies the
 * iterate by M, the filter's output multiplication.  d_mask is the caller's
 * device volume (NULL removes the mask), read until the plan is destroyed or
 * the mask changes; set it before rtkb_cg_start.  FP32 plans without a
 * learned preconditioner.  rtkb_cg_finish does nothing without a mask. */
int  rtkb_cg_set_support_mask(rtkb_cg * plan, const float * d_mask);
int  rtkb_cg_finish(rtkb_cg * plan, void * stream);
/* Waits for `stream`; *rr = ||r_k||^2 of the normal equations, *rr0 = ||r_0||^2. */
int  rtkb_cg_residual(rtkb_cg * plan, double * rr, double * rr0, int * iterations, void * stream);
void rtkb_cg_destroy(rtkb_cg * plan);
/* Checkpoint / resume of a CG plan between iterations (no reference
 * counterpart: RTK resumes only by a warm start from a saved iterate, which
 * restarts the Krylov recurrence).  rtkb_cg_state_bytes gives the size of the
 * state -- a 64-byte header, the FP64 scalars (rr, rr0, alpha, beta, pAp), the
 * residual and direction vectors in the plan's storage types, and the
 * iteration count.  rtkb_cg_save_state writes it to `buffer` (device or host
 * memory; waits for `stream`).  rtkb_cg_load_state restores it into a plan of
 * the same volume size and storage that was started (rtkb_cg_start or
 * rtkb_cg_start_rhs) on the saved iterate; the next rtkb_cg_iterate then
 * continues the saved recurrence.  The iterate itself is the caller's
 * buffer.  Plans with a learned preconditioner are refused (UNSUPPORTED). */
int  rtkb_cg_state_bytes(const rtkb_cg * plan, long long * bytes);
int  rtkb_cg_save_state(rtkb_cg * plan, void * buffer, void * stream);
int  rtkb_cg_load_state(rtkb_cg * plan, const void * buffer, void * stream);
/* Whole reconstruction: at most max_iterations iterations, stopping early when
 * ||r_k|| <= relative_residual * ||r_0|| (relative_residual <= 0: never). */
int  rtkb_conjugate_gradient(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                             const rtkb_cg_params * params, const float * d_proj, const float * d_weights,
                             int displaced_detector, float * d_x, int max_iterations, double relative_residual,
                             int * iterations, double * final_relative_residual, void * stream);
/* Batched CG (no counterpart in the reference): many independent problems of
 * uneven sizes, each a full rtkb_cg_start problem (own geometry,
 * descriptions, stack, weights and iterate).  rtkb_cg_batch_iterate runs
 * `niter` iterations of every problem as ONE CUDA graph launch: the graph,
 * captured on the first call for a given niter, holds each problem's
 * iterations on its own branch, so the problems' kernels run concurrently.
 * rtkb_cg_batch_plan returns problem i's plan for rtkb_cg_residual. */
typedef struct rtkb_cg_batch_problem
{
  const rtkb_geometry * geometry;
  rtkb_image_desc       vol, proj;
  const float *         d_proj;
  const float *         d_weights; /* may be NULL */
  int                   displaced_detector;
  float *               d_x; /* x0 on entry, the iterate afterwards */
} rtkb_cg_batch_problem;
typedef struct rtkb_cg_batch rtkb_cg_batch;
int       rtkb_cg_batch_create(const rtkb_cg_batch_problem * problems, int n, const rtkb_cg_params * params,
                               rtkb_cg_batch ** batch);
int       rtkb_cg_batch_start(rtkb_cg_batch * batch, const rtkb_cg_batch_problem * problems, void * stream);
int       rtkb_cg_batch_iterate(rtkb_cg_batch * batch, int niter, void * stream);
rtkb_cg * rtkb_cg_batch_plan(rtkb_cg_batch * batch, int i);
void      rtkb_cg_batch_destroy(rtkb_cg_batch * batch);
/* rtk::RayBoxIntersectionImageFilter with BoxShape::SetBoxFromImage(volume,
 * false) (include/rtkRayConvexIntersectionImageFilter.hxx:57-84,
 * src/rtkBoxShape.cxx): per pixel, the length (mm) of the source-to-pixel ray
 * inside the box from the volume's origin to origin + D (spacing x (size-1)). */
int rtkb_ray_box_lengths(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                         float * d_out, void * stream);
/* rtk::SARTConeBeamReconstructionFilter (include/rtkSARTConeBeamReconstructionFilter.hxx)
 * with the Joseph forward and voxel-based back projectors, in place on d_x.
 * order: the processing order (np projection positions in the stack, a
 * permutation) or NULL for a Fisher-Yates shuffle driven by SplitMix64(seed)
 * (RTK shuffles with std::default_random_engine, whose sequence the standard
 * leaves to the implementation).  Defaults in RTK: niter 3, lambda 0.3, no
 * positivity, 1 projection per subset, displaced-detector filter on,
 * division threshold 1e-5. */
typedef struct rtkb_sart_params
{
  int                niter;
  double             lambda;
  int                positivity;
  int                projections_per_subset;
  int                disable_displaced_detector;
  double             division_threshold;
  const int *        order;
  unsigned long long seed;
} rtkb_sart_params;
int rtkb_sart(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj, const float * d_proj,
              float * d_x, const rtkb_sart_params * params, void * stream);
/* rtk::OSEMConeBeamReconstructionFilter
 * (include/rtkOSEMConeBeamReconstructionFilter.hxx:84-273) with the Joseph
 * forward projector and the voxel-based (BP_VOXELBASED, RTK's default) or
 * Joseph (BP_JOSEPH) back projector, in place on d_x.  Per subset:
 * x = (x BP(p / FP(x))) / R with De Pierro's factor R
 * (rtk::DePierroRegularizationImageFilter; R = BP(1) when beta = 0); both
 * divisions are itk::DivideOrZeroOutImageFilter's (threshold 1e-5, constants 1
 * and 0).  order / seed as for SART.  store_normalization keeps BP(1) of each
 * subset on the device after the first iteration (RTK's
 * StoreNormalizationImages; the result is the same either way).  Defaults in
 * RTK: niter 3, 1 projection per subset, beta 0, normalisation stored. */
#define RTKB_OSEM_BP_VOXEL 0
#define RTKB_OSEM_BP_JOSEPH 1
typedef struct rtkb_osem_params
{
  int                niter;
  int                projections_per_subset;
  double             beta;
  int                store_normalization;
  int                backprojector;
  const int *        order;
  unsigned long long seed;
} rtkb_osem_params;
int rtkb_osem(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj, const float * d_proj,
              float * d_x, const rtkb_osem_params * params, void * stream);
/* rtk::RegularizedConjugateGradientConeBeamReconstructionFilter
 * (include/rtkRegularizedConjugateGradientConeBeamReconstructionFilter.hxx:171-296)
 * with the Joseph pair: main_loop_iterations times, CG restarted from the
 * current volume for cg_iterations iterations (the plan of rtkb_cg_create with
 * tikhonov and gamma; weights W = displaced-detector weighting of d_weights,
 * NULL = ones, unless disable_displaced_detector), then positivity
 * (ThresholdBelow(0) -> 0), TV denoising (rtkb_tv_denoising_bpdq with gamma_tv,
 * tv_iterations, tv_dimensions) and soft thresholding of the image
 * (sgn(x) max(|x| - soft_threshold, 0)), each when enabled.  In place on d_x;
 * waits for `stream` before returning.  Defaults in RTK: 10 main iterations,
 * 4 CG iterations, positivity and TV on (gamma_tv 5e-5, 10 iterations, all
 * dimensions), soft threshold off (0.001).  RTK's wavelets denoising step
 * (Daubechies) is not provided. */
typedef struct rtkb_regularized_cg_params
{
  int         main_loop_iterations;
  int         cg_iterations;
  double      tikhonov;
  double      gamma;
  int         positivity;
  int         tv;
  double      gamma_tv;
  int         tv_iterations;
  const int * tv_dimensions; /* 3 flags (x, y, z); NULL: all */
  int         soft_threshold_on_image;
  double      soft_threshold;
  int         disable_displaced_detector;
  const float * support_mask; /* NULL: none (the CG's SetSupportMask, its output multiplied by it) */
} rtkb_regularized_cg_params;
int rtkb_regularized_cg(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                        const float * d_proj, const float * d_weights, float * d_x,
                        const rtkb_regularized_cg_params * params, void * stream);
/* rtk::TotalVariationDenoisingBPDQImageFilter
 * (include/rtkTotalVariationDenoisingBPDQImageFilter.hxx,
 * include/rtkDenoisingBPDQImageFilter.hxx:60-148): niter >= 1 iterations of
 * basis pursuit dequantisation with threshold gamma over the dimensions whose
 * flag is set (NULL: all).  d_out may equal d_in. */
int rtkb_tv_denoising_bpdq(const rtkb_image_desc * vol, const float * d_in, float * d_out, double gamma, int niter,
                           const int dims_processed[3], void * stream);
/* rtk::TotalVariationImageFilter (include/rtkTotalVariationImageFilter.hxx):
 * *tv = sum over voxels of the forward-difference gradient norm (zero-flux
 * Neumann, spacing-scaled); waits for `stream`. */
int rtkb_total_variation(const rtkb_image_desc * vol, const float * d_in, double * tv, void * stream);
/* rtk::DePierroRegularizationImageFilter
 * (include/rtkDePierroRegularizationImageFilter.hxx:26-131): d_out =
 * (A + sqrt(A^2 + 8 beta 26 d_update)) / 2, A = d_norm - beta K(d_xk), K the
 * 3x3x3 neighbourhood sum (26 at the centre, 1 elsewhere, zero outside the
 * image).  d_norm NULL: a volume of ones (the filter's default normalisation).
 * d_out may alias d_update or d_norm, and d_xk only when beta = 0. */
int rtkb_de_pierro_regularization(const rtkb_image_desc * vol, const float * d_xk, const float * d_update,
                                  const float * d_norm, double beta, float * d_out, void * stream);
/* d_out = A d_in with the plan's operator (weights W = 1 until rtkb_cg_start
 * sets them).  Used to generate (A e, e) training pairs for the learned
 * preconditioner.  No reference counterpart (RTK's operator is internal to
 * rtk::ReconstructionConjugateGradientOperator). */
int  rtkb_cg_apply_operator(rtkb_cg * plan, const float * d_in, float * d_out, void * stream);

/* ---- learned preconditioner (no reference counterpart) ----
 * A 3-level 3D U-Net (16/32/64 channels, 3x3x3 convolutions, ReLU, no biases,
 * average pooling, nearest up-sampling, concatenated skips, 1x1x1 output),
 * BF16 weights and activations with FP32 accumulation on the tensor cores,
 * FP32 master weights and Adam.  Volumes are float32 [batch][z][y][x] whose
 * sizes are multiples of 4.  Parameters (host order): for each of the ten 3x3x3
 * layers W[tap][c_in][c_out] with tap = (kz*3+ky)*3+kx (cross-correlation,
 * zero padding 1), then the 16 output weights. */
typedef struct rtkb_unet rtkb_unet;
int       rtkb_unet_create(unsigned long long seed, rtkb_unet ** net); /* He-normal initialisation */
long long rtkb_unet_num_parameters(const rtkb_unet * net);
int       rtkb_unet_get_parameters(const rtkb_unet * net, float * host, long long n);
int       rtkb_unet_set_parameters(rtkb_unet * net, const float * host, long long n); /* resets Adam */
/* Gradients of the last rtkb_unet_train_step (mean squared error). */
int       rtkb_unet_get_gradients(const rtkb_unet * net, float * host, long long n);
/* Sizes the activation workspace (allocates; call outside stream capture). */
int       rtkb_unet_reserve(rtkb_unet * net, int batch, int nx, int ny, int nz);
/* d_out = s N(d_in / s) with s = rms(d_in) when normalize, else N(d_in). */
int       rtkb_unet_forward(rtkb_unet * net, int batch, int nx, int ny, int nz, const float * d_in, float * d_out,
                            int normalize, void * stream);
/* One step on the mean squared error between N(d_in) and d_target (no
 * normalisation) over the voxels at least loss_margin voxels inside every face
 * of each volume (crops see their surroundings as zeros, so their borders
 * cannot be fitted): gradients always, an Adam update when `update`; *loss (if
 * not NULL, synchronises) = mean squared error before the update. */
int       rtkb_unet_train_step(rtkb_unet * net, int batch, int nx, int ny, int nz, const float * d_in,
                               const float * d_target, int loss_margin, double learning_rate, int update,
                               double * loss, void * stream);
void      rtkb_unet_destroy(rtkb_unet * net);
/* Selects the forward / data-gradient convolution kernel (process-wide; no counterpart in the
 * reference): 1 (default) = halo and weights of each input-channel chunk loaded by TMA into one
 * shared-memory stage; 2 = the same with two stages, the next chunk's loads overlapping the current
 * chunk's tcgen05 MMAs (one stage where two do not fit); 0 = halo gathered by the threads.  All
 * compute the same MMAs in the same order; kept to compare them. */
int       rtkb_unet_set_conv_pipeline(int enable);
/* Weight-gradient kernel of the U-Net's convolutions, for later training
 * steps in this process: 0 warp-level mma.sync (default, fastest for these
 * layer widths); 1 tcgen05 with the output channels as M = 64 (tiles of
 * 8 x 16 x 4 voxels); 2 tcgen05 with M = 128 (tiles of 8 x 16 x 2 voxels).
 * All three give the same gradients up to FP32 summation order. */
int       rtkb_unet_set_wgrad_kernel(int kernel);

/* Flexible PCG: with a network set (before rtkb_cg_start; NULL removes it) each
 * iteration preconditions the residual, z = s N(r / s), steps with
 * alpha = <p,r>/<p,Ap> and A-orthogonalises the next direction against the
 * last `history` (1..16) directions, p = z - sum_j <z,Ap_j>/<p_j,Ap_j> p_j
 * (truncated flexible CG; history 1 is the Polak-Ribiere flexible CG).  It
 * keeps 2 x history extra volumes on the device.  rtkb_cg_iterate reads the
 * normal-equation residual after every preconditioned iteration and continues
 * as plain CG from the current iterate (p = r) once ||r|| has not improved on
 * its best value for two consecutive iterations.  The network must outlive the
 * plan; volume sizes must be multiples of 4. */
int  rtkb_cg_set_preconditioner(rtkb_cg * plan, rtkb_unet * net, int history);
/* *active: 1 while the network is in use; *fallback_iteration: iteration at
 * which plain CG took over (-1: never). */
int  rtkb_cg_preconditioner_status(const rtkb_cg * plan, int * active, int * fallback_iteration);

/* Autotuner hook of the tiled backprojector (no reference counterpart):
 * force >= 0 selects configuration `force` (box size, voxels per thread
 * column, occupancy target) for later calls on this host thread, -1 restores
 * the footprint heuristic.  *last_used receives the configuration of the last
 * tiled launch on this thread (-1 if none), *count the number of
 * configurations.  Either pointer may be NULL. */
int rtkb_backproject_config(int force, int * last_used, int * count);
/* Tile schedule of the FDK / voxel-based tiled backprojector (no reference
 * counterpart), for later calls in this process.  0 (default): every tile
 * walks the stack from projection 0 -- sums in a fixed order, identical from
 * run to run.  1: projection sweep -- the CTAs count the chunks of
 * 2^sweep_shift projections they have issued in one device counter, and a
 * tile starts where the resident CTAs are on average and wraps around the
 * stack, so the tiles in flight read the same projections and share them in
 * L2 (about 5x less DRAM traffic on a 720-projection stack); a voxel's
 * projections are then summed in an order that varies from run to run (FP32
 * rounding differences, ~5e-7 relative).  sweep_shift in 0..10. */
int rtkb_bp_set_schedule(int schedule, int sweep_shift);
/* Detector rows per band of the Joseph projectors' grids (no reference
 * counterpart), for later calls in this process: every projection of a band
 * runs before the next band, so the blocks in flight touch one y-slab of the
 * volume's copies and accumulators, which stays in L2.  8, 16, 32 or 64 rows
 * for the forward and the back projector (default 8 and 8); the forward
 * projection is identical whatever the band, the back projection up to FP32
 * summation order.  rtk_b200.ops.joseph_autotune times the choices on the
 * caller's problem.  rtkb_joseph_get_band_rows reads the current values. */
int rtkb_joseph_set_band_rows(int forward_rows, int back_rows);
int rtkb_joseph_get_band_rows(int * forward_rows, int * back_rows);

/* ---- projection weighting and ramp filtering ----
 * All take a projection stack description `proj` (slice s = geometry
 * projection proj->index[2] + s) and float32 device buffers.  d_out may equal
 * d_in except for the displaced-detector filter when it pads. */

/* rtk::FDKWeightProjectionFilter (include/rtkFDKWeightProjectionFilter.hxx:40-128):
 * angular-gap x ramp-scaling factor times cos(gamma), computed in FP64.
 * Replaces CUDA_weight_projection. */
int rtkb_fdk_weight(const rtkb_geometry * g, const rtkb_image_desc * proj, const float * d_in, float * d_out,
                    void * stream);

/* rtk::ParkerShortScanImageFilter (include/rtkParkerShortScanImageFilter.hxx:41-209);
 * angular_gap_threshold in radians (RTK's default is pi/9).  *is_short_scan
 * (may be NULL) receives 0 when the largest gap is below the threshold, in
 * which case the projections are copied.  Replaces CUDA_parker_weight. */
int rtkb_parker_short_scan(const rtkb_geometry * g, const rtkb_image_desc * proj, double angular_gap_threshold,
                           const float * d_in, float * d_out, void * stream, int * is_short_scan);

/* rtk::DisplacedDetectorImageFilter (include/rtkDisplacedDetectorImageFilter.hxx:83-323).
 * _region computes the output image (x size doubled on the truncated side when
 * pad_on_truncated_side and the detector is displaced) and *weighted; the
 * filter writes that image.  Replaces CUDA_displaced_weight. */
int rtkb_displaced_detector_region(const rtkb_geometry * g, const rtkb_image_desc * proj, int pad_on_truncated_side,
                                   rtkb_image_desc * out, int * weighted);
int rtkb_displaced_detector(const rtkb_geometry * g, const rtkb_image_desc * proj, int pad_on_truncated_side,
                            const float * d_in, float * d_out, void * stream);
/* rtk::DisplacedDetectorForOffsetFieldOfViewImageFilter
 * (include/rtkDisplacedDetectorForOffsetFieldOfViewImageFilter.hxx), the
 * variant RTK's CPU rtkfdk chains: the padding and the weights follow the
 * stack's field of view (the largest disc every projection sees, below)
 * instead of the detector corners; always padded on the truncated side. */
int rtkb_displaced_detector_offset_fov_region(const rtkb_geometry * g, const rtkb_image_desc * proj,
                                              rtkb_image_desc * out, int * weighted);
int rtkb_displaced_detector_offset_fov(const rtkb_geometry * g, const rtkb_image_desc * proj, const float * d_in,
                                       float * d_out, void * stream);
/* rtk::FieldOfViewImageFilter::ComputeFOVRadius (include/rtkFieldOfViewImageFilter.hxx:41-187),
 * host only: the centre (x, z) and radius r of the largest disc in the
 * rotation plane that every projection of the geometry sees through the
 * stack's detector; type 0 RADIUSINF (the first column's rays only), 1
 * RADIUSSUP (the last column's), 2 RADIUSBOTH.  The linear programme RTK gives
 * lp_solve is solved exactly (its dual, revised simplex).  RTKB_ERR_INVALID_ARGUMENT
 * when no such disc exists. */
int rtkb_field_of_view_radius(const rtkb_geometry * g, const rtkb_image_desc * proj, int type, double * x, double * z,
                              double * r);

/* Ramp filter parameters of rtk::FFTRampImageFilter (include/rtkFFTRampImageFilter.h)
 * and rtk::FFTProjectionsConvolutionImageFilter: window cut frequencies (0 =
 * off, first non-zero wins in this order), Ohnesorge truncation correction,
 * greatest prime factor of the padded size (2 as in RTK built without FFTW, 13
 * as with FFTW: a padded length that is not a power of two is the period of
 * the circular convolution, run embedded in a power-of-two FFT of at least
 * twice that length) and zero-pad factor (2).  hann_cut_y is
 * HannCutFrequencyY: > 0 makes the kernel 2-D (the 1-D kernel times a Hann
 * window along the detector rows' frequency, rows zero-padded by
 * zero_pad_factor_y, ZeroPadFactors[1]: 1 or 2, <= 0 meaning RTK's default 2). */
typedef struct rtkb_ramp_params
{
  double hann_cut;
  double cosine_cut;
  double hamming;
  double ramlak_cut;
  double shepplogan_cut;
  double truncation_correction;
  int    greatest_prime_factor;
  int    zero_pad_factor;
  double hann_cut_y;
  int    zero_pad_factor_y;
} rtkb_ramp_params;

/* Padded FFT length for rows of nu pixels and, when kernel != NULL, the
 * windowed frequency kernel (padded/2+1 FP64 values). */
int rtkb_ramp_kernel(int nu, double spacing_u, const rtkb_ramp_params * params, int * padded, double * kernel);

/* Row-wise ramp filtering: pad (and mirror), FFT, multiply, inverse FFT, crop
 * -- a hand-written shared-memory FFT, two rows per complex transform.
 * Replaces CUDA_padding + CUDA_fft_convolution + the crop filter. */
int rtkb_ramp_filter(const rtkb_image_desc * proj, const rtkb_ramp_params * params, const float * d_in,
                     float * d_out, void * stream);

/* FDK projection preprocessing fused into one pass over the stack: displaced
 * detector (optional), Parker short-scan weighting (optional), FDK weighting
 * and ramp filtering.  `out` receives the filtered stack's description (the
 * displaced detector may double its width); size d_out accordingly (query it
 * with rtkb_displaced_detector_region when displaced != 0). */
typedef struct rtkb_fdk_preprocess_params
{
  int              displaced_detector; /* 0 off, 1 DisplacedDetectorImageFilter, 2 ...ForOffsetFieldOfView */
  int              pad_on_truncated_side;
  int              short_scan;          /* 0 off, 1 Parker weighting when the scan is short */
  double           angular_gap_threshold;
  rtkb_ramp_params ramp;
} rtkb_fdk_preprocess_params;
int rtkb_fdk_preprocess(const rtkb_geometry * g, const rtkb_image_desc * proj, const rtkb_fdk_preprocess_params * p,
                        rtkb_image_desc * out, const float * d_in, float * d_out, void * stream);
/* Batched preprocessing (no counterpart in the reference): rtkb_fdk_preprocess
 * of many independent stacks (own geometry, description and buffers each)
 * with the same parameters, in one launch per padded row length: the ramp
 * kernel's CTAs take row pairs of every stack of that length.  Each problem's
 * output description is written to its `out`.  Results are those of one
 * rtkb_fdk_preprocess call per stack, bit for bit.  Nothing is launched unless
 * every problem is valid. */
typedef struct rtkb_fdk_preprocess_problem
{
  const rtkb_geometry * geometry;
  rtkb_image_desc       proj;
  const float *         d_in;
  float *               d_out;
  rtkb_image_desc       out; /* written */
} rtkb_fdk_preprocess_problem;
int rtkb_fdk_preprocess_batch(rtkb_fdk_preprocess_problem * problems, int n, const rtkb_fdk_preprocess_params * p,
                              void * stream);
/* rtk::IterativeFDKConeBeamReconstructionFilter
 * (include/rtkIterativeFDKConeBeamReconstructionFilter.hxx:171-218): d_x (x0 in,
 * result out) += FDK(p), then niter - 1 times += FDK(lambda (p - JosephFP(x)) /
 * raybox), where raybox is the ray length (mm) in the box from the volume's
 * origin to origin + size x spacing (0 below 1e-5); with positivity every result
 * is thresholded below 0.  FDK = rtkb_fdk_preprocess(fdk) then the FDK back
 * projector.  Defaults in RTK: niter 3, lambda 0.3, no positivity, displaced
 * detector on with padding on the truncated side, Parker short-scan weighting,
 * ramp without truncation correction or Hann window. */
typedef struct rtkb_iterative_fdk_params
{
  int                        niter;
  double                     lambda;
  int                        positivity;
  rtkb_fdk_preprocess_params fdk;
} rtkb_iterative_fdk_params;
int rtkb_iterative_fdk(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj,
                       const float * d_proj, float * d_x, const rtkb_iterative_fdk_params * params, void * stream);

/* ---- phantoms ----
 * Analytic line integrals of ellipsoids (rtk::ProjectGeometricPhantomImageFilter
 * semantics, include/rtkRayConvexIntersectionImageFilter.hxx:57-84): d_out =
 * sum over ellipsoids of density x length of the source-to-pixel segment inside
 * it.  Each ellipsoid is 16 doubles: centre (3), semi-axes (3), rotation
 * (3x3 row-major, local -> world), density.  FP64 arithmetic. */
int rtkb_project_ellipsoids(const rtkb_geometry * g, const rtkb_image_desc * proj, int n_ellipsoids,
                            const double * ellipsoids, float * d_out, void * stream);

/* ---- measurement ----
 * Shared-memory gather peak (no reference counterpart): n_blocks CTAs of 256
 * threads each perform `iters` bilinear-footprint gathers (4 x 4 bytes) from
 * shared memory without bank conflicts.  Bytes moved = n_blocks*256*iters*16;
 * the caller times the launch.  d_sink: n_blocks floats, never written in
 * practice (defeats dead-code elimination). */
int rtkb_probe_smem_gather(int n_blocks, int iters, float * d_sink, void * stream);

#ifdef __cplusplus
}
#endif
#endif

// rtkb_internal.h -- shared host-side helpers of librtkb200 (not part of the ABI).
#pragma once

#include "rtkb200.h"

#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

namespace rtkb
{

// NVTX range around a C-ABI entry point (header-only NVTX 3): a push and a pop
// that cost nothing without a tool attached, and name each call on an ncu or
// Nsight timeline (ncu --nvtx --nvtx-include "rtkb_fdk_backproject/").
struct TraceRange
{
  explicit TraceRange(const char * name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange &) = delete;
  TraceRange & operator=(const TraceRange &) = delete;
};


// ---- error reporting -------------------------------------------------------
void         set_error(const std::string & msg);
const char * g_last_error_cstr();
void clear_error();
int  fail(int code, const std::string & msg);
int  cuda_fail(cudaError_t err, const char * what);

#define RTKB_CUDA_TRY(expr)                                                                                            \
  do                                                                                                                   \
  {                                                                                                                    \
    cudaError_t _e = (expr);                                                                                           \
    if (_e != cudaSuccess)                                                                                             \
      return ::rtkb::cuda_fail(_e, #expr);                                                                             \
  } while (0)

// ---- small FP64 matrix helpers (row-major) ----------------------------------
struct Mat4
{
  double m[16];
};

void mat_mul(const double * a, const double * b, double * c, int n, int k, int m);
void mat4_identity(double * m);
bool affine4_inverse(const double * m, double * r);
void index_to_physical(const rtkb_image_desc & im, double m[16]);
bool physical_to_index(const rtkb_image_desc & im, double m[16]);
bool desc_valid(const rtkb_image_desc * d, std::string & why);
inline long long
num_pixels(const rtkb_image_desc & d)
{
  return (long long)d.size[0] * d.size[1] * d.size[2];
}

// ---- geometry (rtk::ThreeDCircularProjectionGeometry) -----------------------
struct Geometry
{
  struct Proj
  {
    double sid, sdd, gantry, pox, poy, oop, ip, sox, soy, source_angle;
    double coll_uinf, coll_usup, coll_vinf, coll_vsup; // collimation (unbounded: DBL_MAX)
    double rot[16];  // 4x4 rotation (homogeneous)
    double mag[12];  // 3x4 magnification
    double srct[16]; // 4x4 source translation
    double projt[9]; // 3x3 projection translation
    double mat[12];  // 3x4 final projection matrix
  };
  std::vector<Proj> p;
  double            radius_cylindrical = 0.;

  int  add_projection_rad(double sid, double sdd, double ga, double pox, double poy, double oop, double ip,
                          double sox, double soy);
  void source_position(int i, double out[4]) const;
  void proj_coords_to_fixed(int i, double out[16]) const;
  void proj_coords_to_detector(int i, double out[16]) const; // GetProjectionCoordinatesToDetectorSystemMatrix
  void inverse_rotation(int i, double out[16]) const;        // GetRotationMatrices()[i] inverse
  // Parallel beam (SDD 0): pixel - source of RTK's parallel ray iterator, in
  // mm (-2 SID x row 2 of the rotation matrix); false for a divergent beam.
  bool parallel_source_to_pixel(int i, double out[3]) const;
  void source_angles(std::vector<double> & out) const;
  void gantry_angles(std::vector<double> & out) const;
  void tilt_angles(std::vector<double> & out) const;
  void angular_gaps(const std::vector<double> & angles, std::vector<double> & out) const;
  void angular_gaps_with_next(const std::vector<double> & angles, std::vector<double> & out) const;
  double to_untilted(int i, double tilted) const;
};

// Index-to-index backprojection matrix (volume index -> projection index),
// untransposed; returns RTK's path (1 opt X, 2 opt Y, 0 generic).
int bp_matrix(const Geometry & g, const rtkb_image_desc & vol, const rtkb_image_desc & proj, int i, bool fdk,
              double m[12]);

// Per-device library state: cached TMA encoder entry point.
typedef int (*EncodeTiledFn)(void *, int, unsigned, void *, const unsigned long long *, const unsigned long long *,
                             const unsigned *, const unsigned *, int, int, int, int);
EncodeTiledFn tensor_map_encoder();

// Stream-ordered scratch from the library's own per-device memory pool (kept
// reserved between calls; rtkb_trim_memory_pool returns it).
cudaError_t scratch_malloc(void ** p, size_t bytes, cudaStream_t st);
template <class T>
cudaError_t
scratch_malloc(T ** p, size_t bytes, cudaStream_t st)
{
  return scratch_malloc(reinterpret_cast<void **>(p), bytes, st);
}
cudaError_t scratch_free(void * p, cudaStream_t st);

// The conjugate-gradient plan's weights W (displaced-detector weighting of
// d_weights, ones when NULL) and right-hand side d_b = BP(W .* d_proj), FP32;
// rtkb_cg_start_rhs(plan, d_b, ...) then restarts from any volume with them.
int cg_rhs(rtkb_cg * c, const float * d_proj, const float * d_weights, int displaced_detector, float * d_b,
           cudaStream_t st);

// The voxel-based back projector for a cylindrical detector centred on the
// source (float32 stack): d_vout = d_vin + BP(d_proj).
int cylindrical_backproject(const rtkb_geometry * g, const rtkb_image_desc & vol, const rtkb_image_desc & proj,
                            const float * d_proj, const float * d_vin, float * d_vout, cudaStream_t st);

// Projection processing order of the iterative solvers when the caller gives
// none: 0..n-1 shuffled by Fisher-Yates driven by SplitMix64(seed).
void seeded_order(int n, unsigned long long seed, std::vector<int> & order);

} // namespace rtkb

struct rtkb_geometry
{
  rtkb::Geometry g;
};

#define RTKB_TRACE() rtkb::TraceRange rtkb_trace_range_(__func__)

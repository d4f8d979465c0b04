// rtkb_joseph.h -- internal interface of the Joseph projector pair, shared by
// the C ABI entry points and the conjugate-gradient plan.
#pragma once

#include "rtkb_internal.h"

namespace rtkb
{

struct RayProj
{
  double pix2vol[12]; // rows 0-2 of the projection-index -> volume-index matrix
  double src[3];      // source in volume index coordinates; parallel beam: pixel - source (volume index units)
  double parallel;    // 1: parallel beam (every pixel has its own source, RTK's parallel ray iterator)
};

// Cylindrical panel (ProjectionsRegionConstIteratorRayBasedWithCylindricalPanel):
// projection index -> flat detector coordinates (u along the arc, v, w), and
// detector coordinates -> volume index, rows 0-2 of each.
struct CylProj
{
  double idx2det[12];
  double det2vol[12];
};

struct JosephArgs
{
  const RayProj * P;
  const CylProj * C;      // per-projection cylindrical tables, nullptr for a flat panel
  double          radius; // cylindrical panel radius (with C)
  int             nu, nv, np;
  int             pidx0, pidx1, pidx2; // absolute index of buffer pixel (0, 0, 0)
  int             n[3];                // volume size
  int             vidx[3];             // volume region index
  double          spacing[3];
  double          bmin[3], bmax[3];
};


// Per-projection ray tables of a stack (host side).
// (cyl: filled for a cylindrical panel, left empty for a flat one)
int  joseph_tables(const Geometry & g, const rtkb_image_desc & vol, const rtkb_image_desc & proj,
                   std::vector<RayProj> & out, std::vector<CylProj> * cyl = nullptr);
// Device bytes of both tables, each 256-byte aligned.
size_t joseph_table_bytes(const std::vector<RayProj> & tab, const std::vector<CylProj> & cyl);
// Copies both tables to d_mem (joseph_table_bytes bytes) on st and points a's tables there.
cudaError_t joseph_upload_tables(const std::vector<RayProj> & tab, const std::vector<CylProj> & cyl, double radius,
                                 void * d_mem, JosephArgs & a, cudaStream_t st);
void joseph_args(JosephArgs & a, const rtkb_image_desc & vol, const rtkb_image_desc & proj, const RayProj * d_tab);

int joseph_check(const rtkb_geometry * g, const rtkb_image_desc * vol, const rtkb_image_desc * proj);

// Storage type of a volume or projection stack (arithmetic is FP32 either way).
enum class Elem
{
  F32,
  BF16
};

// Scratch of either projector: joseph_forward_scratch_bytes(voxels) bytes,
// 256-byte aligned (equal to joseph_back_scratch_bytes, so one buffer serves
// both): transposed, widened and quad-expanded copies of the volume for the
// forward projector, scalar and quad accumulators for the back projector.
size_t joseph_forward_scratch_bytes(long long nvox);
size_t joseph_back_scratch_bytes(long long nvox);

// Enqueue the forward projector: pout = w * (pin + FP(V)); pin, w may be null.
// V has storage ve, pin and pout storage pe.
cudaError_t joseph_forward_launch(const JosephArgs & a, const void * V, Elem ve, void * scratch, const void * pin,
                                  void * pout, Elem pe, const float * w, cudaStream_t st);
inline cudaError_t
joseph_forward_launch(const JosephArgs & a, const float * V, void * scratch, const float * pin, float * pout,
                      const float * w, cudaStream_t st)
{
  return joseph_forward_launch(a, V, Elem::F32, scratch, pin, pout, Elem::F32, w, st);
}
// Enqueue the back projector: vout = vin + BP(proj) + tau * x; vin, x may be
// null.  proj has storage pe, vin and vout storage ve, x storage xe.  Zeroes
// its accumulators in the scratch.
cudaError_t joseph_back_launch(const JosephArgs & a, const void * proj, Elem pe, void * scratch, const void * vin,
                               void * vout, Elem ve, const void * x, Elem xe, float tau, cudaStream_t st);
inline cudaError_t
joseph_back_launch(const JosephArgs & a, const float * proj, void * scratch, const float * vin, float * vout,
                   const float * x, float tau, cudaStream_t st)
{
  return joseph_back_launch(a, proj, Elem::F32, scratch, vin, vout, Elem::F32, x, Elem::F32, tau, st);
}

} // namespace rtkb

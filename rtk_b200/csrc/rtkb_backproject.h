// rtkb_backproject.h -- internal interface of the voxel-based back projector
// as a reusable object, for plans that replay it (the CG plan's voxel-based
// back projector inside its captured iteration graph).
#pragma once

#include "rtkb_internal.h"

#include <cuda.h>

namespace rtkb
{

// Host-side decisions of one backprojection (see bp_prepare in backproject.cu).
struct BpPrepared
{
  bool        generic = false; // some projection leaves RTK's optimised-Y path: FP64 per-voxel kernel
  bool        use_tma = false;
  bool        fdk = false;
  int         cfg = 0;
  int         nproj = 0, nu = 0, nv = 0, nx = 0, ny = 0, nz = 0;
  long long   np_total = 0;
  CUtensorMap tmap;
};

struct VoxelBackprojector
{
  BpPrepared    prep;
  const float * d_proj = nullptr; // the stack it reads (fixed address)
  double *      d_mats = nullptr; // buffer-index matrices, uploaded at creation
  int *         d_modes = nullptr;
  unsigned *    d_progress = nullptr; // the tile schedule's sweep counter
};

// Device bytes of the matrix and mode tables of nproj projections and the
// tile schedule's sweep counter.
size_t voxel_backprojector_bytes(int nproj);
// Builds RTK's voxel-based (non-FDK) back projector of the stack d_proj
// (description proj) into volumes described by vol; uploads its tables into
// d_mem (voxel_backprojector_bytes), synchronously.  Flat panels only.
int voxel_backprojector_create(const rtkb_geometry * g, const rtkb_image_desc & vol, const rtkb_image_desc & proj,
                               const float * d_proj, void * d_mem, VoxelBackprojector & out);
// d_vout = d_vin + BP(stack); d_vin may equal d_vout; stream-ordered, capturable.
int voxel_backprojector_launch(const VoxelBackprojector & b, const float * d_vin, float * d_vout, cudaStream_t st);

} // namespace rtkb

/* Stand-in for RTK's CMake-generated rtkConfiguration.h: the projection slab
 * size of RTK's CUDA projectors (RTK_CUDA_PROJECTIONS_SLAB_SIZE, default 16,
 * CMakeLists.txt:208). */
#ifndef RTKB_STUB_RTKCONFIGURATION_H
#define RTKB_STUB_RTKCONFIGURATION_H
#define SLAB_SIZE 16
#endif

// rtk_cuda_fdk_driver.cu -- C entry point around RTK's own CUDA FDK back
// projector (CUDA_reconstruct_conebeam, compiled unchanged from the RTK
// sources), so that tests and bench.py can time it and compare it with the
// oracle.  TEST INFRASTRUCTURE ONLY: never part of the product.
//
// rtkcuda_fdk_backproject runs the slab loop of
// CudaFDKBackProjectionImageFilter::GPUGenerateData
// (src/rtkCudaFDKBackProjectionImageFilter.cxx:99-113): the stack goes to
// CUDA_reconstruct_conebeam SLAB_SIZE projections at a time, the output of
// one slab being the input of the next.  `matrices` are the filter's float
// matrices (12 per projection, texture-centred and normalised at the rotation
// centre, :74-97), computed by the caller.  Returns 0, or -1 with the message
// of the exception RTK's error macro threw (rtkcuda_last_error).
#include "rtkCudaFDKBackProjectionImageFilter.hcu"
#include "rtkConfiguration.h"

#include <cstring>
#include <exception>
#include <string>

static std::string g_error;

extern "C" const char *
rtkcuda_last_error(void)
{
  return g_error.c_str();
}

extern "C" int
rtkcuda_slab_size(void)
{
  return SLAB_SIZE;
}

extern "C" int
rtkcuda_fdk_backproject(const int proj_size[3], const int vol_size[3], const float * matrices, float * dev_vol_in,
                        float * dev_vol_out, float * dev_proj)
{
  try
  {
    int          ps[3] = { proj_size[0], proj_size[1], proj_size[2] };
    int          vs[3] = { vol_size[0], vol_size[1], vol_size[2] };
    const long   plane = (long)ps[0] * ps[1];
    const int    n = proj_size[2];
    float *      pin = dev_vol_in;
    for (int i = 0; i < n; i += SLAB_SIZE)
    {
      ps[2] = (n - i < SLAB_SIZE) ? n - i : SLAB_SIZE;
      CUDA_reconstruct_conebeam(ps, vs, const_cast<float *>(matrices) + 12 * i, pin, dev_vol_out,
                                dev_proj + plane * i);
      pin = dev_vol_out;
    }
    return 0;
  }
  catch (const std::exception & e)
  {
    g_error = e.what();
    return -1;
  }
}

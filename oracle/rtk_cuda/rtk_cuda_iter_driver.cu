// rtk_cuda_iter_driver.cu -- C entry points around RTK's own CUDA projectors
// and iterative-reconstruction pieces, compiled unchanged from the RTK
// sources: the ray-casting forward and back projectors, the voxel-based back projector,
// the Laplacian, total-variation denoising (BPDQ) and the conjugate-gradient
// vector update.  Tests and bench.py use them to pin the oracle's conventions
// to the reference's GPU code and to time the reference beside the product.
// TEST INFRASTRUCTURE ONLY: never part of the product.
//
// Each entry returns 0, or -1 with the message of the exception RTK's error
// macro threw (rtkcuda_iter_last_error).  Images are whole buffers (requested
// region = buffered region, index 0), as the callers in tests/ build them.
#include "rtkConfiguration.h"
#include "rtkCudaBackProjectionImageFilter.hcu"
#include "rtkCudaConjugateGradientImageFilter.hcu"
#include "rtkCudaForwardProjectionImageFilter.hcu"
#include "rtkCudaLaplacianImageFilter.hcu"
#include "rtkCudaRayCastBackProjectionImageFilter.hcu"
#include "rtkCudaTotalVariationDenoisingBPDQImageFilter.hcu"

#include <cstddef>
#include <exception>
#include <string>

static std::string g_error;

extern "C" const char *
rtkcuda_iter_last_error(void)
{
  return g_error.c_str();
}

template <typename F>
static int
guarded(F && f)
{
  try
  {
    f();
    return 0;
  }
  catch (const std::exception & e)
  {
    g_error = e.what();
    return -1;
  }
}

// CudaForwardProjectionImageFilter::GPUGenerateData
// (include/rtkCudaForwardProjectionImageFilter.hxx:169-193), flat panel: the
// stack goes to CUDA_forward_project SLAB_SIZE projections at a time.
// `pixel_to_volume` holds the filter's translatedProjectionIndexTransformMatrices
// (12 floats per projection: detector index -> volume texture coordinates) and
// `sources` its source positions in volume texture coordinates (3 per
// projection); box and spacing as the filter sets them (:60-83).
extern "C" int
rtkcuda_forward_project(const int proj_size[3], const int vol_size[3], const float * pixel_to_volume,
                        const float * sources, float * dev_proj_in, float * dev_proj_out, float * dev_vol, float t_step,
                        const float box_min[3], const float box_max[3], const float spacing[3])
{
  return guarded([&] {
    int          ps[3] = { proj_size[0], proj_size[1], proj_size[2] };
    int          vs[3] = { vol_size[0], vol_size[1], vol_size[2] };
    float        bmin[3] = { box_min[0], box_min[1], box_min[2] }, bmax[3] = { box_max[0], box_max[1], box_max[2] };
    float        sp[3] = { spacing[0], spacing[1], spacing[2] };
    const size_t plane = (size_t)ps[0] * ps[1];
    const int    n = proj_size[2];
    for (int i = 0; i < n; i += SLAB_SIZE)
    {
      ps[2] = (n - i < SLAB_SIZE) ? n - i : SLAB_SIZE;
      float * m = const_cast<float *>(pixel_to_volume) + 12 * i;
      // the volume transforms are read only for cylindrical panels
      CUDA_forward_project(ps, vs, m, m, dev_proj_in + plane * i, dev_proj_out + plane * i, dev_vol, t_step,
                           const_cast<float *>(sources) + 3 * i, 0.f, bmin, bmax, sp, 1);
    }
  });
}

// CudaRayCastBackProjectionImageFilter::GPUGenerateData
// (src/rtkCudaRayCastBackProjectionImageFilter.cxx:35-186), flat panel: slabs
// of SLAB_SIZE projections, the output of one slab the input of the next;
// `pixel_to_volume` and `sources` as for the forward projector (the same
// matrices, :115-156), the box from the first to the last voxel index and the
// step the minimum spacing (:57-76), all computed by the caller.
extern "C" int
rtkcuda_ray_cast_back_project(const int proj_size[3], const int vol_size[3], const float * pixel_to_volume,
                              const float * sources, float * dev_vol_in, float * dev_vol_out, float * dev_proj,
                              float t_step, const float box_min[3], const float box_max[3], const float spacing[3])
{
  return guarded([&] {
    int          ps[3] = { proj_size[0], proj_size[1], proj_size[2] };
    int          vs[3] = { vol_size[0], vol_size[1], vol_size[2] };
    float        bmin[3] = { box_min[0], box_min[1], box_min[2] }, bmax[3] = { box_max[0], box_max[1], box_max[2] };
    float        sp[3] = { spacing[0], spacing[1], spacing[2] };
    const size_t plane = (size_t)ps[0] * ps[1];
    const int    n = proj_size[2];
    float *      pin = dev_vol_in;
    for (int i = 0; i < n; i += SLAB_SIZE)
    {
      ps[2] = (n - i < SLAB_SIZE) ? n - i : SLAB_SIZE;
      float * m = const_cast<float *>(pixel_to_volume) + 12 * i;
      // the filter passes its float source array through a double pointer
      // that the kernel reads back as floats (:155, :173)
      CUDA_ray_cast_back_project(ps, vs, m, m, pin, dev_vol_out, dev_proj + plane * i, t_step,
                                 reinterpret_cast<double *>(const_cast<float *>(sources) + 3 * i), 0.f, bmin, bmax, sp);
      pin = dev_vol_out;
    }
  });
}

// CudaBackProjectionImageFilter::GPUGenerateData
// (include/rtkCudaBackProjectionImageFilter.hxx:158-176), flat panel: slabs of
// SLAB_SIZE projections, the output of one slab the input of the next.
// `matrices` are the filter's fMatrix (12 floats per projection).
extern "C" int
rtkcuda_back_project(const int proj_size[3], const int vol_size[3], const float * matrices, float * dev_vol_in,
                     float * dev_vol_out, float * dev_proj)
{
  return guarded([&] {
    int          ps[3] = { proj_size[0], proj_size[1], proj_size[2] };
    int          vs[3] = { vol_size[0], vol_size[1], vol_size[2] };
    float        unused9[9] = { 0.f };
    const size_t plane = (size_t)ps[0] * ps[1];
    const int    n = proj_size[2];
    float *      pin = dev_vol_in;
    for (int i = 0; i < n; i += SLAB_SIZE)
    {
      ps[2] = (n - i < SLAB_SIZE) ? n - i : SLAB_SIZE;
      float * m = const_cast<float *>(matrices) + 12 * i;
      // the volume-index-to-detector matrices are read only for cylindrical panels
      CUDA_back_project(ps, vs, m, m, unused9, pin, dev_vol_out, dev_proj + plane * i, 0., 1);
      pin = dev_vol_out;
    }
  });
}

// CudaLaplacianImageFilter::GPUGenerateData (src/rtkCudaLaplacianImageFilter.cxx)
extern "C" int
rtkcuda_laplacian(const int size[3], const float spacing[3], float * dev_in, float * dev_out)
{
  return guarded([&] {
    int   s[3] = { size[0], size[1], size[2] };
    float sp[3] = { spacing[0], spacing[1], spacing[2] };
    CUDA_laplacian(s, sp, dev_in, dev_out);
  });
}

// CudaTotalVariationDenoisingBPDQImageFilter::GPUGenerateData
// (src/rtkCudaTotalVariationDenoisingBPDQImageFilter.cxx:30-62); beta as
// DenoisingBPDQImageFilter::GenerateOutputInformation sets it
// (include/rtkDenoisingBPDQImageFilter.hxx:86), computed by the caller.
extern "C" int
rtkcuda_total_variation(const int size[3], const float spacing[3], float * dev_in, float * dev_out, float gamma,
                        float beta, int niter)
{
  return guarded([&] {
    int   s[3] = { size[0], size[1], size[2] };
    float sp[3] = { spacing[0], spacing[1], spacing[2] };
    CUDA_total_variation(s, sp, dev_in, dev_out, gamma, beta, niter);
  });
}

// The vector steps of CudaConjugateGradientImageFilter::GPUGenerateData
// (include/rtkCudaConjugateGradientImageFilter.hxx:58-105); the caller
// applies the operator between them.
extern "C" int
rtkcuda_cg_copy(size_t n, float * in, float * out)
{
  return guarded([&] { CUDA_copy(n, in, out); });
}

extern "C" int
rtkcuda_cg_subtract(size_t n, float * out, float * to_be_subtracted)
{
  return guarded([&] { CUDA_subtract(n, out, to_be_subtracted); });
}

extern "C" int
rtkcuda_cg_update(size_t n, float * x, float * r, float * p, float * ap)
{
  return guarded([&] { CUDA_conjugate_gradient(n, x, r, p, ap); });
}

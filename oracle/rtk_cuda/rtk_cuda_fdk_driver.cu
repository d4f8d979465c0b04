// rtk_cuda_fdk_driver.cu -- C entry points around RTK's own CUDA FDK back
// projector (CUDA_reconstruct_conebeam), its CUDA projection weighting filters
// and its CUDA ramp filter (CUDA_padding, CUDA_fft_convolution), compiled
// unchanged from the RTK sources, so that tests and bench.py can time them and
// compare them with the oracle.  TEST INFRASTRUCTURE ONLY: never part of the product.
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
#include "rtkCudaFFTProjectionsConvolutionImageFilter.hcu"
#include "rtkConfiguration.h"

#include <cstring>
#include <exception>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

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

// ---- RTK's CUDA projection weighting filters (compiled unchanged), on whole
// images (requested region = buffered region).  The scalar state that their
// ITK filters compute on the host (angular-gap factors, Parker's delta and
// first angle, the displaced detector's corners) is passed in by the caller.

#include "rtkCudaDisplacedDetectorImageFilter.hcu"
#include "rtkCudaFDKWeightProjectionFilter.hcu"
#include "rtkCudaParkerShortScanImageFilter.hcu"

// CudaFDKWeightProjectionFilter::GPUGenerateData
// (src/rtkCudaFDKWeightProjectionFilter.cxx:31-124): geometry = 7 floats per
// projection (sdd, sid, projection offset x, y, source offset y, weight
// factor, tilt angle).
extern "C" int
rtkcuda_fdk_weight(const int proj_idx[2], const int proj_size[3], float * dev_in, float * dev_out, const float * geometry,
                   const float proj_orig[2], const float proj_row[2], const float proj_col[2])
{
  try
  {
    int   idx[2] = { proj_idx[0], proj_idx[1] }, size[3] = { proj_size[0], proj_size[1], proj_size[2] };
    int   buf[2] = { proj_size[0], proj_size[1] };
    float o[2] = { proj_orig[0], proj_orig[1] }, r[2] = { proj_row[0], proj_row[1] }, c[2] = { proj_col[0], proj_col[1] };
    CUDA_weight_projection(idx, size, buf, buf, dev_in, dev_out, const_cast<float *>(geometry), o, r, c);
    return 0;
  }
  catch (const std::exception & e)
  {
    g_error = e.what();
    return -1;
  }
}

// CudaParkerShortScanImageFilter::GPUGenerateData
// (src/rtkCudaParkerShortScanImageFilter.cxx:30-120), short-scan branch:
// geometry = 5 floats per projection (sdd, source offset x, projection offset
// x, sid, gantry angle).
extern "C" int
rtkcuda_parker_weight(const int proj_idx[2], const int proj_size[3], float * dev_in, float * dev_out,
                      const float * geometry, float delta, float first_angle, float proj_orig, float proj_row,
                      float proj_col)
{
  try
  {
    int idx[2] = { proj_idx[0], proj_idx[1] }, size[3] = { proj_size[0], proj_size[1], proj_size[2] };
    int buf[2] = { proj_size[0], proj_size[1] };
    CUDA_parker_weight(idx, size, buf, buf, dev_in, dev_out, const_cast<float *>(geometry), delta, first_angle,
                       proj_orig, proj_row, proj_col);
    return 0;
  }
  catch (const std::exception & e)
  {
    g_error = e.what();
    return -1;
  }
}

// CudaDisplacedDetectorImageFilter::GPUGenerateData
// (src/rtkCudaDisplacedDetectorImageFilter.cxx:30-140): input stack region
// (idx_in, size_in), output region (idx_out, size_out, padded on the
// truncated side), geometry = 4 floats per projection (sdd, source offset x,
// projection offset x, sid), theta = min(-inferior corner, superior corner).
extern "C" int
rtkcuda_displaced_weight(const int idx_in[3], const int size_in[3], const int idx_out[3], const int size_out[3],
                         float * dev_in, float * dev_out, const float * geometry, float theta, int positive_case,
                         float proj_orig, float proj_row, float proj_col)
{
  try
  {
    int ii[3] = { idx_in[0], idx_in[1], idx_in[2] }, si[3] = { size_in[0], size_in[1], size_in[2] };
    int io[3] = { idx_out[0], idx_out[1], idx_out[2] }, so[3] = { size_out[0], size_out[1], size_out[2] };
    int bi[2] = { size_in[0], size_in[1] }, bo[2] = { size_out[0], size_out[1] };
    CUDA_displaced_weight(ii, si, bi, io, so, bo, dev_in, dev_out, const_cast<float *>(geometry), theta,
                          positive_case != 0, proj_orig, proj_row, proj_col);
    return 0;
  }
  catch (const std::exception & e)
  {
    g_error = e.what();
    return -1;
  }
}

// CudaFFTProjectionsConvolutionImageFilter::GPUGenerateData
// (include/rtkCudaFFTProjectionsConvolutionImageFilter.hxx) for the ramp
// filter of a whole stack (requested region = buffered region, index 0):
// PadInputImageRegion's CUDA_padding into a stack of `padded` columns with
// the input at column (padded - nu) / 2 and `padded_y` rows (nv, or the
// padded height of the 2-D kernel) with the input at row 0, and the Ohnesorge
// mirror weights `mirror_weights` (n_weights = truncation extent + 1, as
// UpdateTruncationMirrorWeights sizes them); CUDA_fft_convolution with the
// kernel spectrum `kernel_fft` (kernel_rows rows of padded / 2 + 1 complex
// values: 1 row for the 1-D kernel, padded_y rows for the 2-D one, already
// scaled by 1 / (padded * padded_y * np) as the filter does for cuFFT); then the
// crop back to nv rows of nu columns (CudaCropImageFilter's copy) into dev_out.
extern "C" int
rtkcuda_fft_ramp(const int proj_size[3], int padded, int padded_y, const float * kernel_fft, int kernel_rows,
                 const float * mirror_weights, int n_weights, float * dev_in, float * dev_out)
{
  float *  d_pad = nullptr;
  float2 * d_kernel = nullptr;
  int      rc = 0;
  try
  {
    const int    nu = proj_size[0], nv = proj_size[1], np = proj_size[2];
    const int    zeroext = (padded - nu) / 2;
    const size_t nk = (size_t)(padded / 2 + 1) * kernel_rows;
    if (cudaMalloc((void **)&d_pad, sizeof(float) * (size_t)padded * padded_y * np) != cudaSuccess ||
        cudaMalloc((void **)&d_kernel, sizeof(float2) * nk) != cudaSuccess)
      throw std::runtime_error("cudaMalloc failed");
    cudaMemcpy(d_kernel, kernel_fft, sizeof(float2) * nk, cudaMemcpyHostToDevice);
    int3               idx = { zeroext, 0, 0 };
    uint3              sz = { (unsigned)padded, (unsigned)padded_y, (unsigned)np };
    uint3              sz_i = { (unsigned)nu, (unsigned)nv, (unsigned)np };
    std::vector<float> mw(mirror_weights, mirror_weights + n_weights);
    CUDA_padding(idx, sz, sz_i, dev_in, d_pad, mw);
    int3 dim = { padded, padded_y, np };
    if (dim.y == 1 && dim.z > 1)
      std::swap(dim.y, dim.z);
    int2 kdim = { padded / 2 + 1, kernel_rows };
    CUDA_fft_convolution(dim, kdim, d_pad, d_kernel);
    for (int s = 0; s < np; s++)
      if (cudaMemcpy2D(dev_out + (size_t)s * nv * nu, sizeof(float) * nu,
                       d_pad + (size_t)s * padded_y * padded + zeroext, sizeof(float) * padded, sizeof(float) * nu,
                       (size_t)nv, cudaMemcpyDeviceToDevice) != cudaSuccess)
        throw std::runtime_error("crop copy failed");
  }
  catch (const std::exception & e)
  {
    g_error = e.what();
    rc = -1;
  }
  cudaFree(d_pad);
  cudaFree(d_kernel);
  return rc;
}

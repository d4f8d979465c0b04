// probe.cu -- shared-memory gather peak on this GPU: the denominator of the
// backprojectors' L1/shared-memory roofline.  Every thread performs bilinear-
// footprint gathers (four 4-byte loads: p, p+1, p+W, p+W+1) from a shared
// array at bank-conflict-free addresses, 100% on-chip hits, so the kernel runs
// at the shared-memory load bandwidth (one 128-byte wavefront per SM per
// cycle).  Bytes counted: n_blocks * 256 threads * iters * 16.
#include "rtkb_internal.h"

namespace
{
constexpr int kW = 64;

__global__ void __launch_bounds__(256)
smem_gather_kernel(int iters, float * sink)
{
  __shared__ float buf[kW * 33];
  for (int i = threadIdx.x; i < kW * 33; i += blockDim.x)
    buf[i] = (float)(i & 7);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // lanes read consecutive words of one row: conflict-free; the +1 / +W taps
  // of the footprint are again consecutive across lanes.  Rows cycle 0..31,
  // so the largest address is 31 * kW + 31 + kW + 1 < kW * 33.
  int   row = warp & 31;
  float acc = 0.f;
#pragma unroll 4
  for (int it = 0; it < iters; it++)
  {
    const float * q = buf + row * kW + lane;
    acc += q[0] + q[1] + q[kW] + q[kW + 1];
    row = (row + 1) & 31;
  }
  if (acc == -1.f)
    sink[blockIdx.x] = acc;
}
} // namespace

extern "C" int
rtkb_probe_smem_gather(int n_blocks, int iters, float * d_sink, void * stream)
{
  if (n_blocks <= 0 || iters <= 0 || !d_sink)
    return rtkb::fail(RTKB_ERR_INVALID_ARGUMENT, "invalid probe arguments");
  smem_gather_kernel<<<n_blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(iters, d_sink);
  RTKB_CUDA_TRY(cudaGetLastError());
  return RTKB_OK;
}

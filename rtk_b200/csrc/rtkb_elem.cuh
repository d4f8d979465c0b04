// rtkb_elem.cuh -- element access for the storage types of volumes and
// projection stacks: float, or bfloat16 (the CG plan's BF16 storage variant).
// Arithmetic is always FP32: BF16 values are widened on load and rounded to
// nearest even on store.
#pragma once

#include <cuda_bf16.h>

namespace rtkb
{
__device__ __forceinline__ float
ld_elem(const float * p, long long i)
{
  return p[i];
}
__device__ __forceinline__ float
ld_elem(const __nv_bfloat16 * p, long long i)
{
  return __bfloat162float(p[i]);
}
__device__ __forceinline__ void
st_elem(float * p, long long i, float v)
{
  p[i] = v;
}
__device__ __forceinline__ void
st_elem(__nv_bfloat16 * p, long long i, float v)
{
  p[i] = __float2bfloat16_rn(v);
}
} // namespace rtkb

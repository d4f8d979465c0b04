// rtkb_ptx.cuh -- hand-written PTX wrappers for sm_100a (mbarrier, TMA) with
// bounded waits.  Every wait gives up after g_wait_limit polls (4 M unless
// rtkb_set_wait_limit changed it), records RTKB_STATUS_TIMEOUT in the device
// status word and returns false, so a kernel can never spin forever.
#pragma once

#include <cstdint>
#include <cuda.h>

#define RTKB_STATUS_TIMEOUT 1u
#define RTKB_STATUS_BAD_FOOTPRINT 2u

namespace rtkb
{
namespace dev
{

extern __device__ unsigned int g_device_status;
// polls of try_wait (each suspends for a bounded, hardware-defined time)
// before a bounded wait gives up; set from the host (rtkb_set_wait_limit)
extern __device__ unsigned int g_wait_limit;

constexpr uint32_t kDefaultWaitLimit = 1u << 22;

__device__ __forceinline__ uint32_t
smem_u32(const void * p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void
mbar_init(uint64_t * bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void
fence_barrier_init()
{
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void
mbar_arrive(uint64_t * bar)
{
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void
mbar_arrive_expect_tx(uint64_t * bar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool
mbar_try_wait(uint64_t * bar, uint32_t parity)
{
  uint32_t ok;
  asm volatile("{\n\t.reg .pred p;\n\t"
               "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
               "selp.u32 %0, 1, 0, p;\n\t}"
               : "=r"(ok)
               : "r"(smem_u32(bar)), "r"(parity)
               : "memory");
  return ok != 0;
}

// Bounded wait for the phase with the given parity to complete (the limit is
// read only when the first poll fails).
__device__ __forceinline__ bool
mbar_wait(uint64_t * bar, uint32_t parity)
{
  if (mbar_try_wait(bar, parity))
    return true;
  const uint32_t limit = *static_cast<volatile unsigned int *>(&g_wait_limit);
  for (uint32_t it = 1; it < limit; ++it)
    if (mbar_try_wait(bar, parity))
      return true;
  atomicOr(&g_device_status, RTKB_STATUS_TIMEOUT);
  return false;
}

// 3-D tiled TMA load (no multicast) of a box into shared memory, completion
// signalled on `bar` as transaction bytes.  c0 * element size must be a
// multiple of 16 bytes (the caller rounds c0 down to a multiple of 4 floats).
__device__ __forceinline__ void
tma_load_3d(void * dst, const CUtensorMap * map, int c0, int c1, int c2, uint64_t * bar)
{
  asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
               " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
               "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void
prefetch_tensor_map(const CUtensorMap * map)
{
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

} // namespace dev
} // namespace rtkb

// pool.cpp -- the library's stream-ordered scratch memory.
//
// Every entry point that needs temporary device memory (projector tables and
// quad-expanded volume copies, solver work vectors, staging chunks) takes it
// from one cudaMemPool_t per device that this library owns, with an unbounded
// release threshold: memory freed in stream order stays reserved for the next
// call instead of going back to the driver at the caller's next synchronise
// (the default pool's threshold of 0 would unmap it there, and the next call
// would pay the mapping again, about 5 ms for a 640 MB projector scratch on a
// B200).  The caller's default pool is left alone.  rtkb_trim_memory_pool
// returns the reserved memory; an allocation that fails trims the pool and
// retries once.
#include "rtkb200.h"
#include "rtkb_internal.h"

#include <atomic>
#include <cstdint>
#include <mutex>

namespace
{
constexpr int    kMaxDevices = 64;
std::mutex       g_pool_mutex;
cudaMemPool_t    g_pools[kMaxDevices] = {};
std::atomic<int> g_injected_failures{ 0 }; // allocations still to fail (rtkb_inject_allocation_failures)

// the pool allocation, or an injected out-of-memory failure
cudaError_t
pool_alloc(void ** p, size_t bytes, cudaMemPool_t pool, cudaStream_t st)
{
  int left = g_injected_failures.load();
  while (left > 0)
    if (g_injected_failures.compare_exchange_weak(left, left - 1))
      return cudaErrorMemoryAllocation;
  return cudaMallocFromPoolAsync(p, bytes, pool, st);
}

cudaError_t
pool_for(int dev, cudaMemPool_t * out)
{
  if (dev < 0 || dev >= kMaxDevices)
    return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_pool_mutex);
  if (!g_pools[dev])
  {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    cudaError_t   e = cudaMemPoolCreate(&pool, &props);
    if (e != cudaSuccess)
      return e;
    uint64_t keep = UINT64_MAX;
    e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess)
    {
      cudaMemPoolDestroy(pool);
      return e;
    }
    g_pools[dev] = pool;
  }
  *out = g_pools[dev];
  return cudaSuccess;
}
} // namespace

namespace rtkb
{
cudaError_t
scratch_malloc(void ** p, size_t bytes, cudaStream_t st)
{
  int         dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  cudaMemPool_t pool = nullptr;
  if (e == cudaSuccess)
    e = pool_for(dev, &pool);
  if (e != cudaSuccess)
    return e;
  e = pool_alloc(p, bytes, pool, st);
  if (e == cudaErrorMemoryAllocation)
  {
    cudaGetLastError();
    // free what the pool holds (the stream's pending frees first), then retry
    e = cudaStreamSynchronize(st);
    if (e == cudaSuccess)
      e = cudaMemPoolTrimTo(pool, 0);
    if (e == cudaSuccess)
      e = pool_alloc(p, bytes, pool, st);
  }
  return e;
}

cudaError_t
scratch_free(void * p, cudaStream_t st)
{
  return cudaFreeAsync(p, st);
}
} // namespace rtkb

extern "C" int
rtkb_trim_memory_pool(long long * reserved_after)
{
  using namespace rtkb;
  int         dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  cudaMemPool_t pool = nullptr;
  if (e == cudaSuccess)
    e = pool_for(dev, &pool);
  if (e == cudaSuccess)
    e = cudaMemPoolTrimTo(pool, 0);
  uint64_t reserved = 0;
  if (e == cudaSuccess)
    e = cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
  if (e != cudaSuccess)
    return cuda_fail(e, "rtkb_trim_memory_pool");
  if (reserved_after)
    *reserved_after = (long long)reserved;
  return RTKB_OK;
}

extern "C" int
rtkb_memory_pool_reserved(long long * reserved)
{
  using namespace rtkb;
  if (!reserved)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  int         dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  cudaMemPool_t pool = nullptr;
  if (e == cudaSuccess)
    e = pool_for(dev, &pool);
  uint64_t r = 0;
  if (e == cudaSuccess)
    e = cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &r);
  if (e != cudaSuccess)
    return cuda_fail(e, "rtkb_memory_pool_reserved");
  *reserved = (long long)r;
  return RTKB_OK;
}

extern "C" int
rtkb_inject_allocation_failures(int count)
{
  if (count < 0)
    return rtkb::fail(RTKB_ERR_INVALID_ARGUMENT, "count must not be negative");
  g_injected_failures.store(count);
  return RTKB_OK;
}

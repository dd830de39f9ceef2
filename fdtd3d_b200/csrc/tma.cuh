// tma.cuh - PTX helpers shared by the TMA-pipelined sweep kernels:
// mbarriers with bounded waits and 3-D tiled bulk tensor loads (no
// multicast).  Every wait gives up after about one second of %globaltimer.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace fdtdb {
namespace tma {

__device__ __forceinline__ uint32_t smem_addr (const void *p)
{
  return (uint32_t) __cvta_generic_to_shared (p);
}

__device__ __forceinline__ void mbar_init (uint32_t bar, unsigned count)
{
  asm volatile ("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx (uint32_t bar, unsigned bytes)
{
  asm volatile ("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait (uint32_t bar, unsigned parity)
{
  unsigned ok;
  asm volatile (
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns ()
{
  unsigned long long t;
  asm volatile ("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Wait for the phase with the given parity; false after about one second.
static __device__ __noinline__ bool mbar_wait (uint32_t bar, unsigned parity)
{
  if (mbar_try_wait (bar, parity))
    return true;
  const unsigned long long t0 = global_ns ();
  while (!mbar_try_wait (bar, parity))
    if (global_ns () - t0 > 1000000000ull)
      return false;
  return true;
}

// Box of a 3-D tensor map at (c0 = z, c1 = y, c2 = x) into shared memory at
// dst, completion counted on the mbarrier bar.  c0 times the element size
// must be a multiple of 16 bytes.
__device__ __forceinline__ void load_3d (uint32_t dst, const CUtensorMap *map, int c0, int c1, int c2, uint32_t bar)
{
  asm volatile (
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
      : "memory");
}

}  // namespace tma
}  // namespace fdtdb

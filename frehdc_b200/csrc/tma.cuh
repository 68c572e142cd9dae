// Device helpers of the TMA-fed kernels (cg1.cu, step_kernels.cu): mbarriers
// with bounded waits, 2-D tiled bulk-tensor loads into shared memory, and the
// acquire fence for tensor maps written by host copies.  Plain (non-multicast)
// loads only.
#ifndef FREHD_TMA_CUH
#define FREHD_TMA_CUH

#include <cuda.h>

#include "cg_common.cuh"

namespace frehd {

static __device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

static __device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

static __device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

static __device__ __forceinline__ bool mbar_test(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for the phase `parity` of `bar` to complete, for at most `limit_ns`.
static __device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity,
                                          unsigned long long limit_ns) {
  if (mbar_test(bar, parity)) return true;
  const unsigned long long t0 = gtimer_ns();
  while (!mbar_test(bar, parity)) {
    if (gtimer_ns() - t0 > limit_ns) return false;
  }
  return true;
}

static __device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map,
                                            unsigned long long *bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

static __device__ __forceinline__ void acquire_maps(const CUtensorMap *maps, int n) {
  // the maps were written to global memory by a host copy: make them visible to the TMA unit
  for (int q = 0; q < n; ++q)
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(maps + q) : "memory");
}

}  // namespace frehd

#endif

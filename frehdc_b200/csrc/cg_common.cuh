// Device helpers of the persistent CG kernels (cg.cu, noalloc.cu): constants of
// the tile decomposition, L2-coherent loads, and the fused grid reduction and
// barrier with a bounded wait.
#ifndef FREHD_CG_COMMON_CUH
#define FREHD_CG_COMMON_CUH

#include "domain.cuh"
#include "kernels.cuh"

namespace frehd {

constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;  // 2 s per wait
constexpr int kStallIters = 400;  // CG iterations without ||r|| halving that count as a stall
constexpr int CTX = 128, CTY = kCgThreads / 32;   // tile: 4 cells per thread along a row
constexpr int HX = CTX + 2, HY = CTY + 2;         // tile + halo
constexpr int CPT = 4;                            // cells per thread, stride 32 along a row
constexpr int NWARP = kCgThreads / 32;

__device__ __forceinline__ unsigned long long gtimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ double ld(const double *a, long k) { return __ldcg(a + k); }

// Sum of NV values over all threads of the nblocks blocks that share `sc`,
// identical in every block, and a barrier among them.  rank: this block's
// number among them (blockIdx.x when the grid is one group).  partials: STRIDE
// doubles per block; totals: NV doubles.
template <int NV, int STRIDE = 4>
static __device__ __forceinline__ bool grid_allreduce(double (&v)[NV], Scratch *sc, double *partials,
                                                      double *totals, unsigned nblocks,
                                                      unsigned rank = blockIdx.x) {
  static_assert(NV <= STRIDE, "NV values per block must fit the partials stride");
  __shared__ double sh[STRIDE][NWARP];
  __shared__ int s_last, s_ok;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int m = 0; m < NV; ++m) {
    const double s = warp_sum(v[m]);
    if (lane == 0) sh[m][wid] = s;
  }
  __syncthreads();
  if (nblocks == 1) {
    // A lone block: every thread forms the total the general path would give
    // (thread 0's fixed-order sum over the warps) from shared memory.  Thread 0
    // makes the block's writes visible at device scope, as the general path's
    // fence does, before it issues the next TMA loads.
#pragma unroll
    for (int m = 0; m < NV; ++m) {
      double a = 0;
      for (int q = 0; q < NWARP; ++q) a += sh[m][q];
      v[m] = a;
    }
    if (threadIdx.x == 0) __threadfence();
    __syncthreads();  // sh is rewritten by the next call
    return true;
  }
  unsigned my_gen = 0;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int m = 0; m < NV; ++m) {
      double a = 0;
      for (int q = 0; q < NWARP; ++q) a += sh[m][q];
      partials[STRIDE * rank + m] = a;
    }
    // the generation can only move once every block (this one too) arrived
    my_gen = *(volatile unsigned *)&sc->bar_gen;
    __threadfence();
    const unsigned arrived = atomicAdd(&sc->bar_count, 1u);
    s_last = arrived == nblocks - 1;
    s_ok = 1;
  }
  __syncthreads();
  if (s_last) {
    // every partial is visible: sum them in a fixed order, publish, release
    __threadfence();
    double a[NV];
#pragma unroll
    for (int m = 0; m < NV; ++m) a[m] = 0;
    for (unsigned q = threadIdx.x; q < nblocks; q += blockDim.x) {
#pragma unroll
      for (int m = 0; m < NV; ++m) a[m] += ld(partials, STRIDE * (long)q + m);
    }
    __syncthreads();  // sh is reused
#pragma unroll
    for (int m = 0; m < NV; ++m) {
      const double s = warp_sum(a[m]);
      if (lane == 0) sh[m][wid] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
      for (int m = 0; m < NV; ++m) {
        double t = 0;
        for (int q = 0; q < NWARP; ++q) t += sh[m][q];
        totals[m] = t;
      }
      *(volatile unsigned *)&sc->bar_count = 0;
      __threadfence();
      atomicAdd(&sc->bar_gen, 1u);
    }
  } else if (threadIdx.x == 0) {
    volatile unsigned *gen = &sc->bar_gen;
    const unsigned long long lim = sc->wait_limit_ns ? sc->wait_limit_ns : kBarrierTimeoutNs;
    const unsigned long long t0 = gtimer_ns();
    while (*gen == my_gen) {
      if (gtimer_ns() - t0 > lim) {
        set_status(sc, FREHD_ERR_TIMEOUT);
        s_ok = 0;
        break;
      }
      __nanosleep(16);
    }
    __threadfence();
  }
  __syncthreads();
  if (!s_ok || *(volatile int *)&sc->status == FREHD_ERR_TIMEOUT) return false;
#pragma unroll
  for (int m = 0; m < NV; ++m) v[m] = ld(totals, m);
  return true;
}

// Failure-path testing (frehd_domain_set_wait_test): true in the one CTA of a
// solve that is to leave before its first grid barrier without arriving, so that
// its partners' bounded wait runs out and the solve reports FREHD_ERR_TIMEOUT.
// Nothing is in flight at that point (no TMA load, no partial sum).
static __device__ __forceinline__ bool test_skip_barrier(const Scratch *sc, unsigned rank) {
  return *(const volatile int *)&sc->skip_barrier_rank1 == (int)rank + 1;
}

struct TileIt {
  int ntx, nty, ntiles;
};

__device__ __forceinline__ void tile_origin(const TileIt &t, int tile, int *i0, int *j0) {
  *i0 = (tile % t.ntx) * CTX;
  *j0 = (tile / t.ntx) * CTY;
}

}  // namespace frehd

#endif

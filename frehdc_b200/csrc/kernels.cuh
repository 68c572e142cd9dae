// Kernel declarations and small device helpers shared by the .cu files.
#ifndef FREHD_KERNELS_CUH
#define FREHD_KERNELS_CUH

#include "domain.cuh"

namespace frehd {

// Step statistics written by k_finish (device memory, read by the host).
struct StepOut {
  int step, cg_iters, status, n_cfl_warn, n_fix, cg_fallback;
  double cg_rr, cg_bb, max_cflx, max_cfly, volume;
  long long cg_iters_total;
  int cg_noconv, pad;
  long long cg_noconv_steps;  // running count of steps whose solve stopped at maxIter
};

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ int warp_sum_int(int v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

__global__ void k_explicit(View w);
__global__ void k_update_geo(View w);
__global__ void k_update_geo_init(View w);
__global__ void k_update_vel(View w);
__global__ void k_update_vel_tvd(View w);
__global__ void k_finish(View w, int nblocks_vel, StepOut *out);
__global__ void k_ref_to_padded(double *dst, const double *src, long n, int nx, int ny, int pitch);
__global__ void k_padded_to_ref(double *dst, const double *src, long n, int nx, int ny, int pitch);
__global__ void k_ref_to_padded_int(int *dst, const int *src, long n, int nx, int ny, int pitch);
__global__ void k_padded_to_ref_int(int *dst, const int *src, long n, int nx, int ny, int pitch);
__global__ void k_fill(double *a, long n, double v);
// Batched launches over many domains (views2[2*d + half]: domain d's view with
// ping-pong half `half` current).
struct BatchTile {
  int d, bx, by, gx;  // domain slot, first tile's coordinates, the domain's tile-grid width
  int nt, pad;        // tiles nt along x from (bx, by), one after another in one block
};
struct FinishJob {
  int d, nblocks_vel;  // domain slot, its k_update_vel tile count
  StepOut *out;
  int *status;         // the domain's device status after the step, in host-mapped memory
};
__global__ void k_explicit_batch(const View *views2, const BatchTile *tiles);
__global__ void k_update_geo_batch(const View *views2, const BatchTile *tiles);
__global__ void k_update_vel_batch(const View *views2, const BatchTile *tiles);
__global__ void k_update_vel_tvd_batch(const View *views2, const BatchTile *tiles);
__global__ void k_finish_batch(const View *views2, const FinishJob *jobs, Scratch *bsync);
__global__ void k_interp_velocity(View w, double *uuYP, double *vvXP);
__global__ void k_system_to_ref(View w, double *GnCt, double *GnXP, double *GnXM, double *GnYP,
                                double *GnYM, double *z, double *xs);
__global__ void k_solution_from_ref(View w, const double *xs);

// Persistent Jacobi-preconditioned CG (cg.cu).
__global__ void k_cg(View w, int x0_surface, int eliminate);

constexpr int kCgThreads = 512;

}  // namespace frehd

#endif

// Host interface of the single-sweep CG (cg1.cu): TMA descriptors of the
// arrays it reads as halo boxes, launch size and launch.
#ifndef FREHD_CG1_H
#define FREHD_CG1_H

#include <cuda.h>
#include <cuda_runtime.h>

#include "domain.cuh"

namespace frehd {

// Tensor maps over the padded layout: the scaled residual and direction (two
// buffers each) and the scaled face couplings Hx, Hy, in FP64, and the same
// arrays of the mixed-precision solve in FP32 (zero when it is not enabled).
// The kernel reads them from global memory (a device copy, 64-byte aligned).
struct Cg1Maps {
  CUtensorMap r[2], p[2], hx, hy;
  CUtensorMap fr[2], fp[2], fhx, fhy;
  CUtensorMap tfr[2], tfp[2], tfhx, tfhy;  // the FP32 arrays as 128 x 32-tile boxes
};

int cg1_make_maps(const Grid &g, double *r0, double *r1, double *p0, double *p1, double *hx,
                  double *hy, Cg1Maps *m);
// The FP32 maps of the mixed-precision solve.
int cg1_make_maps_f32(const Grid &g, float *r0, float *r1, float *p0, float *p1, float *hx,
                      float *hy, Cg1Maps *m);
size_t cg1_smem_bytes();
// Co-resident blocks for a cooperative launch, at most one per tile.
int cg1_blocks(int device, const Grid &g, int *blocks);
int cg1_launch(const View &w, const Cg1Maps *m_dev, int blocks, int x0_surface, int eliminate,
               cudaStream_t stream);
// Partial sums per block the single-sweep CG keeps in the partials buffer.
constexpr int kCg1PartialStride = 8;

// One CTA's share of one domain's solve in a batched launch.
struct CgJob {
  int d;      // domain slot (views2[2*d + parity])
  int rank;   // this CTA's rank in the domain's group
  int nb;     // CTAs of the group (all co-resident)
  int flags;  // bit 0: x0 = surface; bit 1: decoupled rows eliminated
};
// Launch the batched solve: nctas CTAs, CTA c runs jobs[job_start[c] ..
// job_start[c+1]), then single-CTA jobs from `singles` (nsingles of them;
// *taken zero at the launch, reset by k_finish_batch).
int cg1_launch_batch(const View *views2, const Cg1Maps *const *maps, const int *job_start,
                     const CgJob *jobs, const CgJob *singles, int nsingles, int *taken, int nctas,
                     int any_mixed, cudaStream_t stream);
// CTAs of the batched solve that fit on the device at once.
int cg1_batch_capacity(int device, int *ctas);

// ---- batched solve over one list of every domain's tiles (k_cg1_tiles)
// One admitted domain of the solve (built by the host).
struct BDom {
  int slot;          // views2[2*slot + parity], maps[slot]
  int tile0, ntiles; // its CG tiles in the global list, in its own tile order
  int ntx;           // its tiles along x
  int flags;         // bit 0: x0 = surface; bit 1: decoupled rows eliminated
  int pad;
};
// One entry of the global tile list.
struct BTile {
  int dom;   // index into the BDom array
  int tile;  // the domain's own tile number
};
// The solve's state of one domain (device memory; written by its reducing CTA
// between the rounds of a launch, initialised at the launch's start).
struct BState {
  double alpha, beta, gamma, gamma_old, delta, e1, e2, e3, rr, bnorm, best, rr_prev, stop;
  int phase, it, it_all, attempt, elim, cur, outer, fallback, noconv, best_it, vpar, takeover;
};
// Partial sums kept per tile of the global list.
constexpr int kTilePartStride = 8;
// Launch: nctas CTAs over ntiles list entries of ndom domains.  part: ntiles *
// kTilePartStride doubles; bsync: the launch's barrier scratch (bar_count and
// n_done zero at the launch, reset by k_finish_batch); bpart: (nctas + 1) *
// kCg1PartialStride doubles.
int cg1_launch_tiles(const View *views2, const Cg1Maps *const *maps, const BDom *doms,
                     BState *states, const BTile *tiles, int ndom, int ntiles, double *part,
                     Scratch *bsync, double *bpart, int nctas, cudaStream_t stream);
int cg1_tiles_capacity(int device, int *ctas);

}  // namespace frehd

#endif

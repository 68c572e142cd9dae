// Device-side data layout and parameters of one domain.
//
// Layout: every cell array is a padded 2-D array of (ny + 2) rows of `pitch`
// doubles.  Cell (i, j), i in [-1, nx], j in [-1, ny], lives at
//   (j + 1) * pitch + (i + kXOff)
// so the ghost ring of the reference (its "N2ct" entries) is stored in place:
// row j = -1 / ny are the south / north ghosts, columns i = -1 / nx the west /
// east ghosts and the four corners sit at the row/column crossings.  kXOff = 4
// puts i = 0 on a 32-byte boundary; pitch is a multiple of 32 doubles, so each
// interior row starts 256-byte aligned and a warp reading 32 consecutive cells
// touches exactly eight 32-byte sectors.
#ifndef FREHD_DOMAIN_CUH
#define FREHD_DOMAIN_CUH

#include <cstdint>

#include "frehd_b200.h"

namespace frehd {

constexpr int kXOff = 4;

struct Grid {
  int nx, ny, pitch;
  long total;
  __host__ __device__ __forceinline__ long at(int i, int j) const {
    return (long)(j + 1) * pitch + (i + kXOff);
  }
  static Grid make(int nx, int ny) {
    Grid g;
    g.nx = nx;
    g.ny = ny;
    g.pitch = ((nx + kXOff + 1) + 31) / 32 * 32;
    g.total = (long)(ny + 2) * g.pitch;
    return g;
  }
};

// Map a reference linear index (map.c layout, [0, N2ct)) to padded (i, j).
__host__ __device__ __forceinline__ void ref_to_ij(long k, int nx, int ny, int *i, int *j) {
  const long N = (long)nx * ny;
  if (k < N) { *i = (int)(k % nx); *j = (int)(k / nx); }
  else if (k < N + nx) { *i = (int)(k - N); *j = ny; }
  else if (k < N + 2 * nx) { *i = (int)(k - N - nx); *j = -1; }
  else if (k < N + 2 * nx + ny) { *i = nx; *j = (int)(k - N - 2 * nx); }
  else if (k < N + 2 * nx + 2 * ny) { *i = -1; *j = (int)(k - N - 2 * nx - ny); }
  else {
    const long T = N + 2 * nx + 2 * ny + 4;
    const long c = k - (T - 4);  // corners: iMjP, iPjP, iPjM, iMjM (map.c:117-120)
    *i = (c == 0 || c == 3) ? -1 : nx;
    *j = (c == 0 || c == 1) ? ny : -1;
  }
}

// Constant parameters of a domain's step (the Config fields it reads).
struct Params {
  int nx, ny, pitch;
  double dx, dy, dt, g, NUx, NUy, Kx, Ky, manningN, hD, minDepth, wtfh, CFLl, CFLh;
  double offset, surfmin, dsurf, tidePS, subR, dxf, dyf, eps;
  int Ne, useThinLayer, useScalar, tideFirst, tideLen, maxIter;
  int scalarAdv;      // 1: first-order upwind, 2: TVD with the superbee limiter
  int nscalar;        // scalars transported (S and nscalar - 1 tracers)
  // inflow cells i in [inflowI0, inflowI1), j in [inflowJ0, inflowJ1) (inflowLen of them)
  int inflowLen, inflowI0, inflowI1, inflowJ0, inflowJ1;
  double inflowS;
  int useWind;        // windTerm (nsfunctions.c:609-648)
  double rhoa, Cw, CwT;
  int mixed;          // CG: FP32 inner iterations inside FP64 iterative refinement
  double eps_inner;   // relative residual reduction of one FP32 inner solve
  // geometry source
  int geom_fine;          // 0: tables, 1: fine bottoms
  int check_block;        // fine bottoms: block-check face areas (FREHD_GEOM_BLOCK_CHECK)
  const double *tab;      // tables: 10 * Ne * N, level-major (subgrid.c:118-119)
  const double *zf;       // fine bottoms, zf[fj*fpitch + fi]
  long fpitch;
  int r;
};

// Per-step counters and scratch shared by the kernels of one domain.
struct Scratch {
  unsigned int bar_count, bar_gen;  // grid barrier of the persistent CG
  int status;                       // FREHD_OK or the first error of the step
  int tt;                           // step index the captured kernels run
  int cg_iters;
  int n_cfl_warn;
  int n_fix;                        // scalar-singularity cells queued for the fix-up
  int cg_fallback;                  // 1: the last solve stalled and was redone in eliminated form
  int cur;                          // batched stepping: which ping-pong half holds the state
  double cg_rr, cg_bb;              // ||r||^2, ||b||^2 at CG exit
  unsigned long long max_cflx_bits, max_cfly_bits;  // positive doubles as ordered bits
  double volume;
  long long cg_iters_total;  // running sum over completed steps
  int cg_noconv;             // 1: the last solve stopped at maxIter with ||r|| >= eps*||b||
  int skip_barrier_rank1;    // failure-path testing: 1 + the rank of the CTA that leaves the
                             // next solve's first grid barrier without arriving (0: none)
  long long cg_noconv_steps; // running count of completed steps whose solve stopped at maxIter
  unsigned long long wait_limit_ns;  // bound of the grid-barrier waits (0: kBarrierTimeoutNs)
  int n_done;                // batched solve over a tile list: domains whose solve ended
  int pad2;
};

// Device pointers of the state and work arrays for one step.  `cur`/`nxt`
// buffers are swapped by the host between steps.
struct View {
  Params p;
  Grid gr;
  // persistent state
  double *surf_cur, *surf_nxt, *depth_cur, *depth_nxt, *S_cur, *S_nxt;
  double *Tr_cur[FREHD_MAX_SCALARS - 1], *Tr_nxt[FREHD_MAX_SCALARS - 1];  // tracers 1 ..
  int *ind_cur, *ind_nxt;
  double *u, *v, *CDXP, *CDYP, *CFLx, *CFLy;
  double *V, *Z, *Nx, *Oy, *Vx, *Vy, *Zx, *Zy;
  const double *bottomZ, *bottomXP, *bottomYP;
  // per-step work
  double *EnXP, *EnYP, *Gx, *Gy, *Ct, *b;
  double *Hx, *Hy;  // symmetrically scaled couplings of the single-sweep CG
  // FP32 arrays of the mixed-precision CG (null unless enabled): scaled residual
  // and direction (two buffers each), correction, scaled couplings
  float *fr0, *fr1, *fp0, *fp1, *fd, *fhx, *fhy;
  float *fs;  // mixed form: 1/sqrt|Ct| rounded to FP32 (the correction's unscaling)
  double *x, *r, *p0, *p1, *q;
  double *cellV, *Sm, *Fuu, *Fvv;
  unsigned char *rmv;
  int *fix_list;
  double *partials;  // per-block partial sums
  const double *tide;
  int ntide;
  const double *inflow;        // bc->inflow by step
  int ninflow;
  const double *wspd;          // bc->windspd by step
  int nwspd;
  const double *wcos, *wsin;   // cos/sin of the wind direction by step (nwdir + 1 entries;
  int nwdir;                   // the last one for steps past the series)
  double *dXP, *dYP;           // face depths of the last updateAllFaceDepth (wind only)
  // Level-value cache of the fine geometry (null with tables): per cell the ten
  // values of the last two levels it evaluated, one per parity of the level
  // index; lvc plane (slot * 10 + value) and lvi plane slot (the level held,
  // -1 = none) are padded grids like every cell array.
  double *lvc;
  int *lvi;
  Scratch *sc;
};

__device__ __forceinline__ double tide_value(const View &w) {
  const int tt = w.sc->tt;
  return (tt >= 0 && tt < w.ntide) ? w.tide[tt] : 0.0;
}

// bc->inflow[tt]; past the end of the series the reference reads its zeroed guard.
__device__ __forceinline__ double inflow_value(const View &w) {
  const int tt = w.sc->tt;
  return (tt >= 0 && tt < w.ninflow) ? w.inflow[tt] : 0.0;
}

// Inflow cell: inflowLoc[k] = jj*NX + ii - 1 (configuration.c:53-60).
__device__ __forceinline__ bool is_inflow(const Params &p, int i, int j) {
  return p.inflowLen > 0 && i >= p.inflowI0 && i < p.inflowI1 && j >= p.inflowJ0 && j < p.inflowJ1;
}

__device__ __forceinline__ bool is_tidal(const Params &p, int i, int j) {
  return j == p.ny - 1 && i >= p.tideFirst && i < p.tideFirst + p.tideLen;
}

// Record the first error status of the step.
__device__ __forceinline__ void set_status(Scratch *sc, int code) {
  atomicCAS(&sc->status, 0, code);
}

}  // namespace frehd

#endif

// Single-sweep Jacobi-PCG for the 5-point free-surface system (default solver),
// in FP64 or as FP32 inner iterations inside FP64 iterative refinement.
//
// Same system, preconditioner, start and stopping rule as k_cg (cg.cu): Jacobi
// M = diag|Ct|, x0 = 0 (or the surface), stop when ||r||_2 < eps*||b||_2
// checked before each iteration (rtc.c:53, itersolv.c:355-456), decoupled rows
// iterated as lambda = 1 components; their neighbours keep the coupling to them
// as in the reference's assembled (non-symmetric) matrix, or, with
// FREHD_DECOUPLED_ELIMINATED, see their exact value b/|Ct| in the right-hand
// side instead (cg.cu explains both).  Two things change:
//
// 1. The solve runs on the symmetrically scaled system
//      A~ = D^-1/2 A D^-1/2,  x~ = D^1/2 x,  r~ = D^-1/2 r,  D = diag|Ct|,
//    on which plain CG produces exactly the Jacobi-PCG iterates of A in exact
//    arithmetic (x = D^-1/2 x~ at every step; no symmetry of A is needed for
//    that change of variables).  A~ has a unit diagonal and the face couplings
//    H = G/sqrt(D_i D_j); a decoupled row applies none of them (its flag is the
//    sign bit of its own east coupling Hx), so an iteration needs no division.
//    The stopping test uses the unscaled residual, ||r||^2 = sum D r~^2.
// 2. One sweep per iteration: with p_i = r~_i + beta_i p_{i-1},
//      (p_i, A~ p_i) = (r~_i, A~ r~_i) + beta_i [(r~_i, A~ p_{i-1}) + (p_{i-1}, A~ r~_i)]
//                      + beta_i^2 (p_{i-1}, A~ p_{i-1}),
//    an identity that holds for any A~, so alpha_i = (r~_i, r~_i)/(p_i, A~ p_i)
//    of textbook CG (CGIter, itersolv.c:355-456) is known from dot products of
//    the previous sweep.  A sweep forms p_i, A~ p_i, r~_{i+1} and A~ r~_{i+1}
//    and ends in ONE grid reduction of those six sums instead of two
//    reductions.  (For symmetric A~ this is the ordering of Chronopoulos &
//    Gear, "s-step iterative methods for symmetric linear systems",
//    J. Comput. Appl. Math. 25, 1989.)
//
// One sweep per tile of 128 x 16 cells, with a two-cell halo loaded by TMA:
//   A  p_i = r~_i + beta p_{i-1}                 tile + 2 halo (in place)
//   B  s = A~ p_i, r~_{i+1} = r~_i - alpha s     tile + 1 halo (in place)
//   C  w = A~ r~_{i+1}; x~ += alpha p_i; sums    tile
// FP64 DRAM traffic per cell and iteration: read r~, p, Hx, Hy, x~, |Ct|; write
// r~, p, x~ = 72 bytes.  r~ and p ping-pong between two buffers (neighbouring
// blocks read the old halo while a block writes its new tile); x~ is updated in
// place and turned back into x = x~/sqrt|Ct| at the end.  The boxes of r~, p,
// Hx, Hy are double-buffered in shared memory behind one mbarrier per stage:
// the next tile's loads are in flight while the current tile computes.  Every
// array holds zeros outside the interior (ghost ring and row padding are never
// written; rows past the array come back as TMA zero fill), which is what lets
// the passes run without bounds tests.  All waits are bounded.
//
// Mixed precision (Params::mixed): the outer loop computes r = b - A x in FP64
// with x in FP64, solves the scaled system A~ d~ = r~ with the same sweep in
// FP32 (r~, p, d~, Hx, Hy in FP32, 32 bytes per cell and iteration; all dot
// products accumulated in FP64) until its residual fell by eps_inner, adds
// x += d~/sqrt|Ct| in FP64, and repeats until the FP64 residual meets the
// stopping rule above.  A refinement that does not reduce ||r|| tenfold hands
// the solve to the FP64 path (reported as cg_fallback = 2).
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstring>

#include "cg1.h"
#include "cg_common.cuh"
#include "tma.cuh"
#include "frehd_internal.h"

namespace frehd {

namespace {

constexpr int kTW = CTX, kTH = CTY;              // owned cells of a tile (128 x 16)
constexpr int kRedStride = 8;                    // partial sums per block in grid_allreduce
constexpr int kMaxOuter = 8;                     // refinements of one mixed-precision solve
static_assert(kTH == kCgThreads / 32, "one warp per tile row");
// The FP32 inner sweeps of the mixed solve work on tiles twice as tall (128 x 32,
// each warp two rows): the FP32 boxes move half the bytes of the FP64 ones, and
// the taller tile spreads each tile's barriers and TMA round trip over twice the
// cells.
constexpr int kTallTH = 2 * kTH;
// resident CTAs per SM the launch bounds ask for: 128 registers per thread either way
constexpr int kCg1MinBlocks = kCgThreads >= 512 ? 1 : 512 / kCgThreads;

// Box geometry of an element type: the tile sits kLeft cells into a box with a
// two-cell halo at least, kLeft chosen so that the box's first column is
// 16-byte aligned in the padded layout (column offset kXOff = 4, tiles start at
// multiples of 128 cells).
template <typename T, int TH = kTH>
struct Box {
  static constexpr int kRows = TH;                 // owned rows of a tile
  static constexpr int kRowsPerWarp = TH / (kCgThreads / 32);
  static constexpr int kLeft = sizeof(T) == 8 ? 2 : 4;
  static constexpr int kBW = kTW + 2 * kLeft;      // 132 (FP64) / 136 (FP32)
  static constexpr int kBH = TH + 4;               // 20 (36 for the tall FP32 tiles)
  static constexpr int kBox = kBW * kBH;
  static constexpr int kRing = 2 * (kTW + 2) + 2 * TH;  // cells of the one-cell halo ring
  static constexpr int kRingPer = (kRing + kCgThreads - 1) / kCgThreads;  // ring cells per thread
  static constexpr unsigned kArrBytes = kBox * (unsigned)sizeof(T);
  static constexpr unsigned kStageBytes = 4 * kArrBytes;  // r~, p, Hx, Hy
  static_assert(kArrBytes % 128 == 0, "TMA destinations must stay 128-byte aligned");
  static_assert((kBW * sizeof(T)) % 16 == 0, "TMA box rows must be a multiple of 16 bytes");
  static_assert(((kXOff - kLeft) * sizeof(T)) % 16 == 0, "box origin 16-byte aligned");
  static_assert(kBox % 2 == 0, "pass A works on pairs");
  // box position of tile cell (lx, ly), lx and ly from -1 (the halo ring)
  __device__ static __forceinline__ int q(int lx, int ly) { return (ly + 2) * kBW + kLeft + lx; }
  // box position of cell t of the one-cell halo ring (t < kRing)
  __device__ static __forceinline__ int ring(int t) {
    if (t < kTW + 2) return q(t - 1, -1);          // row above the tile
    t -= kTW + 2;
    if (t < kTW + 2) return q(t - 1, TH);          // row below
    t -= kTW + 2;
    if (t < TH) return q(-1, t);                   // column left
    t -= TH;
    return q(kTW, t);                              // column right
  }
  // origin (first owned cell) of tile `tile` of a grid of these tiles
  __device__ static __forceinline__ void origin(const TileIt &ti, int tile, int *i0, int *j0) {
    *i0 = (tile % ti.ntx) * kTW;
    *j0 = (tile / ti.ntx) * TH;
  }
};
constexpr unsigned kSmemStages = 2 * Box<double>::kStageBytes;  // FP64 stages are the larger
static_assert(2 * Box<float>::kStageBytes <= kSmemStages, "FP32 stages fit the FP64 ones");
static_assert(2 * Box<float, kTallTH>::kStageBytes <= kSmemStages, "tall FP32 stages fit too");

template <typename T>
struct Pair;
template <>
struct Pair<double> {
  using type = double2;
};
template <>
struct Pair<float> {
  using type = float2;
};

// Shared-memory arrays of one stage.
template <typename T, int TH = kTH>
struct Stage {
  T *R, *P, *HX, *HY;
  __device__ Stage(unsigned char *base) {
    R = reinterpret_cast<T *>(base);
    P = R + Box<T, TH>::kBox;
    HX = P + Box<T, TH>::kBox;
    HY = HX + Box<T, TH>::kBox;
  }
};

// The four maps one sweep reads.
struct SweepMaps {
  const CUtensorMap *r, *p, *hx, *hy;
};

// Issue the four box loads of tile `tile` into a stage (one thread).
template <typename T, int TH = kTH>
__device__ __forceinline__ void issue_tile(const SweepMaps &m, const TileIt &ti, int tile,
                                           unsigned char *stage_base, unsigned long long *bar) {
  using B = Box<T, TH>;
  int i0, j0;
  B::origin(ti, tile, &i0, &j0);
  // box origin: cell (i0 - kLeft, j0 - 2) = padded column i0 - kLeft + kXOff (16-byte aligned), row j0 - 1
  const int x = i0 - B::kLeft + kXOff, y = j0 - 2 + 1;
  Stage<T, TH> s(stage_base);
  // generic-proxy writes to this stage (the in-place passes) come before the TMA writes
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  mbar_expect_tx(bar, B::kStageBytes);
  tma_load_2d(s.R, m.r, bar, x, y);
  tma_load_2d(s.P, m.p, bar, x, y);
  tma_load_2d(s.HX, m.hx, bar, x, y);
  tma_load_2d(s.HY, m.hy, bar, x, y);
}

// A~ v at shared-memory position q of a box: unit diagonal, scaled couplings,
// none for a decoupled row (sign bit of its own HX).
template <typename T>
__device__ __forceinline__ T apply(const T *V, const T *HX, const T *HY, int q) {
  constexpr int W = Box<T>::kBW;
  const T he = HX[q];
  const T off = fabs(he) * V[q + 1] + fabs(HX[q - 1]) * V[q - 1] + HY[q] * V[q + W] + HY[q - W] * V[q - W];
  return signbit(he) ? V[q] : V[q] - off;
}

// One CG sweep over this CTA's tiles (rank of nb): p = r~ + beta p_old,
// s = A~ p, r~' = r~ - alpha s, w = A~ r~', X += alpha p; r~' and p stored to
// rn_out / pn_out.  red += (r~',r~'), (w,r~'), (r~',s), (p,w), (p,s) and
// sum D r~'^2 (kUnscaled; D = |Ct|) or (r~',r~') again.  seq: tiles this CTA
// consumed so far (stage and mbarrier phase).
template <typename T, bool kUnscaled, typename XT, int TH = kTH>
__device__ __forceinline__ bool sweep(const SweepMaps &m, T *rn_out, T *pn_out, XT *X, const double *Ct,
                                      const Grid &g, const TileIt &ti, unsigned rank, unsigned nb,
                                      T alpha, T beta, double (&red)[6], unsigned char *smem,
                                      unsigned long long *bars, unsigned &seq, Scratch *sc,
                                      bool x_zero = false) {
  // x_zero: X starts from zero (its stored values are not read)
  using B = Box<T, TH>;
  constexpr int RW = B::kRowsPerWarp, NW = kCgThreads / 32;
  __shared__ int s_ok;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  // generic writes of the previous sweep (all blocks) come before this sweep's TMA reads
  if (threadIdx.x == 0) {
    asm volatile("fence.proxy.async.global;" ::: "memory");
    if ((int)rank < ti.ntiles)
      issue_tile<T, TH>(m, ti, rank, smem + (seq & 1) * B::kStageBytes, &bars[seq & 1]);
  }
  for (int tile = rank; tile < ti.ntiles; tile += nb, ++seq) {
    const int st = seq & 1;
    const int next = tile + (int)nb;
    if (threadIdx.x == 0 && next < ti.ntiles)
      issue_tile<T, TH>(m, ti, next, smem + (st ^ 1) * B::kStageBytes, &bars[st ^ 1]);
    int i0, j0;
    B::origin(ti, tile, &i0, &j0);
    // X and |Ct| of the owned cells: in flight while the boxes arrive
    XT xs[RW][CPT];
    double ds[RW][CPT];
#pragma unroll
    for (int rr = 0; rr < RW; ++rr)
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        const int i = i0 + c * 32 + tx, j = j0 + ty + rr * NW;
        const bool in = i < g.nx && j < g.ny;
        const long k = g.at(in ? i : 0, in ? j : 0);
        xs[rr][c] = x_zero ? XT(0) : X[k];
        ds[rr][c] = kUnscaled ? fabs(Ct[k]) : 0.0;
      }
    if (threadIdx.x == 0) s_ok = mbar_wait(&bars[st], (seq >> 1) & 1, kBarrierTimeoutNs);
    __syncthreads();
    if (!s_ok) {
      // the other stage may hold a load issued for the next tile: let it land
      if (threadIdx.x == 0) {
        set_status(sc, FREHD_ERR_TIMEOUT);
        if (next < ti.ntiles) mbar_wait(&bars[st ^ 1], ((seq + 1) >> 1) & 1, kBarrierTimeoutNs);
      }
      return false;
    }
    mbar_wait(&bars[st], (seq >> 1) & 1, kBarrierTimeoutNs);  // completed: acquire in every thread
    Stage<T, TH> s(smem + st * B::kStageBytes);

    // pass A: p_i = r~_i + beta p_{i-1} on the whole box
    {
      using P2 = typename Pair<T>::type;
      P2 *pp = reinterpret_cast<P2 *>(s.P);
      const P2 *rp = reinterpret_cast<const P2 *>(s.R);
#pragma unroll
      for (int e = threadIdx.x; e < B::kBox / 2; e += kCgThreads) {
        const P2 rv = rp[e];
        P2 pv = pp[e];
        pv.x = rv.x + beta * pv.x;
        pv.y = rv.y + beta * pv.y;
        pp[e] = pv;
      }
    }
    __syncthreads();

    // pass B: r~_{i+1} = r~_i - alpha A~ p_i on the tile (4 cells per thread and row) and its
    // ring; it reads only P, HX, HY besides each thread's own R cells, so R is updated in place
    {
      T rb[RW][CPT];
#pragma unroll
      for (int rr = 0; rr < RW; ++rr)
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          const int ly = ty + rr * NW;
          const int q = B::q(c * 32 + tx, ly);
          const T sv = apply<T>(s.P, s.HX, s.HY, q);
          rb[rr][c] = s.R[q] - alpha * sv;
          if (i0 + c * 32 + tx < g.nx && j0 + ly < g.ny) {
            red[2] += (double)rb[rr][c] * (double)sv;
            red[4] += (double)s.P[q] * (double)sv;
          }
        }
      T rring[B::kRingPer];
      int qr[B::kRingPer];
#pragma unroll
      for (int t = 0; t < B::kRingPer; ++t) {
        const int e = threadIdx.x + t * kCgThreads;
        qr[t] = e < B::kRing ? B::ring(e) : 0;
        rring[t] = e < B::kRing ? s.R[qr[t]] - alpha * apply<T>(s.P, s.HX, s.HY, qr[t]) : T(0);
      }
#pragma unroll
      for (int rr = 0; rr < RW; ++rr)
#pragma unroll
        for (int c = 0; c < CPT; ++c) s.R[B::q(c * 32 + tx, ty + rr * NW)] = rb[rr][c];
#pragma unroll
      for (int t = 0; t < B::kRingPer; ++t)
        if (threadIdx.x + t * kCgThreads < B::kRing) s.R[qr[t]] = rring[t];
    }
    __syncthreads();

    // pass C: w = A~ r~_{i+1}; sums; X_{i+1} = X_i + alpha p_i; store r~, p, X
#pragma unroll
    for (int rr = 0; rr < RW; ++rr)
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        const int i = i0 + c * 32 + tx, ly = ty + rr * NW, j = j0 + ly;
        if (i < g.nx && j < g.ny) {
          const int q = B::q(c * 32 + tx, ly);
          const T u = s.R[q], pc = s.P[q];
          const T wv = apply<T>(s.R, s.HX, s.HY, q);
          const double ud = u;
          red[0] += ud * ud;
          red[1] += (double)wv * ud;
          red[3] += (double)pc * (double)wv;
          red[5] += kUnscaled ? ds[rr][c] * (ud * ud) : ud * ud;
          const long k = g.at(i, j);
          X[k] = xs[rr][c] + alpha * pc;
          rn_out[k] = u;
          pn_out[k] = pc;
        }
      }
    __syncthreads();  // stage st is free for the tile after next
  }
  // this thread's global writes before the next sweep's TMA reads (other blocks)
  asm volatile("fence.proxy.async.global;" ::: "memory");
  return true;
}

// delta0 = (A~ v, v) of a stored scaled vector v (plain halo loads into stage 0).
template <typename T, int TH = kTH>
__device__ __forceinline__ double first_delta(const T *V, const T *HXg, const T *HYg, const Grid &g,
                                              const TileIt &ti, unsigned rank, unsigned nb,
                                              unsigned char *smem) {
  using B = Box<T, TH>;
  constexpr int RW = B::kRowsPerWarp, NW = kCgThreads / 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  double d0 = 0.0;
  Stage<T, TH> s(smem);
  for (int tile = rank; tile < ti.ntiles; tile += nb) {
    int i0, j0;
    B::origin(ti, tile, &i0, &j0);
    __syncthreads();
    // V, Hx, Hy of the tile and its one-cell ring (zeros outside the interior)
    for (int e = threadIdx.x; e < (kTW + 2) * (TH + 2); e += kCgThreads) {
      const int ly = e / (kTW + 2) - 1, lx = e % (kTW + 2) - 1;
      const int i = i0 + lx, jj = j0 + ly;
      const bool in = (unsigned)i < (unsigned)g.nx && (unsigned)jj < (unsigned)g.ny;
      const long k = in ? g.at(i, jj) : 0;
      const int q = B::q(lx, ly);
      s.R[q] = in ? __ldcg(V + k) : T(0);
      s.HX[q] = in ? __ldcg(HXg + k) : T(0);
      s.HY[q] = in ? __ldcg(HYg + k) : T(0);
    }
    __syncthreads();
#pragma unroll
    for (int rr = 0; rr < RW; ++rr)
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        const int i = i0 + c * 32 + tx, ly = ty + rr * NW, j = j0 + ly;
        if (i < g.nx && j < g.ny) {
          const int q = B::q(c * 32 + tx, ly);
          d0 += (double)apply<T>(s.R, s.HX, s.HY, q) * (double)s.R[q];
        }
      }
  }
  __syncthreads();
  return d0;
}


}  // namespace

// FP64 solve of domain w by a group of nb CTAs, of which this CTA is number
// `rank`.  smem/bars: this CTA's two stages and their mbarriers (initialised by
// the kernel); seq counts the tiles this CTA consumed so far, across solves, and
// gives each wait its mbarrier phase.  Returns false after an error (status set).
static __device__ __forceinline__ bool cg1_fp64(const View &w, const Cg1Maps *__restrict__ m,
                                                int x0_surface, int eliminate, unsigned rank,
                                                unsigned nb, unsigned char *smem,
                                                unsigned long long *bars, unsigned &seq) {
  Scratch *sc = w.sc;
  const Grid g = w.gr;
  const Params &p = w.p;
  const int nx = g.nx, ny = g.ny;
  const long pitch = g.pitch;
  TileIt ti;
  ti.ntx = (nx + CTX - 1) / CTX;
  ti.nty = (ny + CTY - 1) / CTY;
  ti.ntiles = ti.ntx * ti.nty;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  double *partials = w.partials, *totals = w.partials + kRedStride * (long)nb;
  const double *Ct = w.Ct, *Gx = w.Gx, *Gy = w.Gy;
  double *const X = w.x;
  if (threadIdx.x == 0) acquire_maps(&m->r[0], 6);

  // A solve of the assembled (non-symmetric) matrix can stall: ||r|| stops
  // falling above eps*||b|| and laspack's CGIter runs on to maxIter.  When ||r||
  // has not halved for kStallIters iterations the solve starts again in the
  // eliminated (symmetric positive definite) form, and the step reports it.
  // (the stall bookkeeping lives in shared memory: written by thread 0 only,
  // read by all between grid reductions)
  __shared__ double s_best;
  __shared__ int s_best_it, s_it_all, s_fallback;
  int it = 0, noconv = 0;
  double rr = 0.0, bnorm = 0.0;
  if (threadIdx.x == 0) {
    s_it_all = 0;
    s_fallback = 0;
  }
  for (int attempt = 0;; ++attempt) {
    const int elim = eliminate | (attempt > 0);
    // ---- setup 1: scaled couplings, x~0 = sqrt|Ct| x0, p_{-1} = 0
    for (int tile = rank; tile < ti.ntiles; tile += nb) {
      int i0, j0;
      tile_origin(ti, tile, &i0, &j0);
      const int j = j0 + ty;
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        const int i = i0 + c * 32 + tx;
        if (i < nx && j < ny) {
          const long k = g.at(i, j);
          const double ct = Ct[k], ce = Ct[k + 1], cn = Ct[k + pitch];
          const double d = sqrt(fabs(ct));
          double hx = Gx[k] / (d * sqrt(fabs(ce))), hy = Gy[k] / (d * sqrt(fabs(cn)));
          if (elim) {  // no coupling across a face with a decoupled row or a ghost (Ct < 0)
            if (!(ct > 0 && ce > 0)) hx = 0.0;
            if (!(ct > 0 && cn > 0)) hy = 0.0;
          }
          // row k's decoupled flag rides in the sign bit of its own east coupling
          w.Hx[k] = ct < 0 ? -fabs(hx) : fabs(hx);
          w.Hy[k] = hy;
          X[k] = x0_surface ? d * w.surf_cur[k] : 0.0;
          w.p0[k] = 0.0;
        }
      }
    }
    {
      double none[1] = {0};
      if (!grid_allreduce<1, kRedStride>(none, sc, partials, totals, nb, rank)) return false;
    }

    // ---- setup 2: r0 = b - A x0 (eliminated: decoupled neighbours at their exact b/|Ct|),
    //      r~0 = r0/sqrt|Ct|
    double acc[3] = {0, 0, 0};
    for (int tile = rank; tile < ti.ntiles; tile += nb) {
      int i0, j0;
      tile_origin(ti, tile, &i0, &j0);
      const int j = j0 + ty;
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        const int i = i0 + c * 32 + tx;
        if (i < nx && j < ny) {
          const long k = g.at(i, j);
          const double ct = Ct[k], bk = w.b[k];
          auto x0 = [&](long kk) -> double { return x0_surface ? w.surf_cur[kk] : 0.0; };
          auto xv = [&](long kk) -> double {
            const double cc = Ct[kk];
            return (elim && cc < 0) ? w.b[kk] / (-cc) : x0(kk);
          };
          double r;
          if (ct > 0) {
            const double ax = ct * x0(k) - (Gx[k] * xv(k + 1) + Gx[k - 1] * xv(k - 1) +
                                            Gy[k] * xv(k + pitch) + Gy[k - pitch] * xv(k - pitch));
            r = bk - ax;
          } else {
            r = bk - (-ct) * x0(k);
          }
          const double rs = r / sqrt(fabs(ct));
          acc[0] += rs * rs;
          acc[1] += r * r;
          acc[2] += bk * bk;
          w.r[k] = rs;
        }
      }
    }
    if (!grid_allreduce<3, kRedStride>(acc, sc, partials, totals, nb, rank)) return false;
    double gamma = acc[0];
    rr = acc[1];
    bnorm = sqrt(acc[2]);

    // ---- setup 3: delta0 = (A~ r~0, r~0)
    double delta;
    {
      double d0[1] = {first_delta<double>(w.r, w.Hx, w.Hy, g, ti, rank, nb, smem)};
      if (!grid_allreduce<1, kRedStride>(d0, sc, partials, totals, nb, rank)) return false;
      delta = d0[0];
    }

    auto converged = [&](double rr_) {
      const double rn = sqrt(rr_);
      return rn < p.eps * bnorm || (bnorm == 0.0 && 1.0 + rn == 1.0);
    };
    double gamma_old = 1.0, e1 = 0.0, e2 = 0.0, e3 = 0.0;
    if (threadIdx.x == 0) {
      s_best = rr;
      s_best_it = 0;
    }
    __syncthreads();
    int cur = 0;
    bool stalled = false;
    it = 0;
    while (!converged(rr) && it < p.maxIter) {
      const double beta = it == 0 ? 0.0 : gamma / gamma_old;
      const double alpha = gamma / (delta + beta * (e1 + e2) + beta * beta * e3);
      ++it;
      double *rn_out = cur ? w.r : w.q, *pn_out = cur ? w.p0 : w.p1;
      // (r~', r~'), (A~ r~', r~'), (r~', A~ p), (p, A~ r~'), (p, A~ p), ||r'||^2; r~' = r~_{i+1}
      double red[6] = {0, 0, 0, 0, 0, 0};
      const SweepMaps sm{&m->r[cur], &m->p[cur], &m->hx, &m->hy};
      if (!sweep<double, true, double>(sm, rn_out, pn_out, X, Ct, g, ti, rank, nb, alpha, beta, red,
                                       smem, bars, seq, sc))
        return false;
      if (!grid_allreduce<6, kRedStride>(red, sc, partials, totals, nb, rank)) return false;
      gamma_old = gamma;
      gamma = red[0];
      delta = red[1];
      e1 = red[2];
      e2 = red[3];
      e3 = red[4];
      rr = red[5];
      cur ^= 1;
      // identical totals in every block: every block takes the same decision; every
      // thread reads the record before thread 0 may update it
      const double best = s_best;
      const int best_it = s_best_it;
      __syncthreads();
      if (rr < 0.25 * best) {
        if (threadIdx.x == 0) {
          s_best = rr;
          s_best_it = it;
        }
      } else if (!elim && it - best_it >= kStallIters) {
        stalled = true;
        break;
      }
    }
    if (threadIdx.x == 0) s_it_all += it;
    // maxIter reached first: laspack's CGIter stops there silently; the step reports it
    noconv = !stalled && !converged(rr);
    if (!stalled) break;
    if (threadIdx.x == 0) s_fallback = 1;
  }  // attempt

  // ---- x = x~ / sqrt|Ct| (each block its own tiles)
  for (int tile = rank; tile < ti.ntiles; tile += nb) {
    int i0, j0;
    tile_origin(ti, tile, &i0, &j0);
    const int j = j0 + ty;
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      const int i = i0 + c * 32 + tx;
      if (i < nx && j < ny) {
        const long k = g.at(i, j);
        X[k] = X[k] / sqrt(fabs(Ct[k]));
      }
    }
  }
  if (rank == 0 && threadIdx.x == 0) {
    sc->cg_iters = s_it_all;
    sc->cg_fallback = s_fallback;
    sc->cg_noconv = noconv;
    sc->cg_rr = rr;
    sc->cg_bb = bnorm * bnorm;
  }
  return true;
}

// Mixed-precision solve (FP32 inner iterations, FP64 refinement).  Returns 0
// after an error (status set), 1 when done, 2 when the refinement stalled and
// the FP64 solve must take over (x is then overwritten by it).
static __device__ __forceinline__ int cg1_mixed(const View &w, const Cg1Maps *__restrict__ m,
                                               int x0_surface, int elim, unsigned rank, unsigned nb,
                                               unsigned char *smem, unsigned long long *bars,
                                               unsigned &seq) {
  Scratch *sc = w.sc;
  const Grid g = w.gr;
  const Params &p = w.p;
  const int nx = g.nx, ny = g.ny;
  const long pitch = g.pitch;
  TileIt ti;
  ti.ntx = (nx + CTX - 1) / CTX;
  ti.nty = (ny + CTY - 1) / CTY;
  ti.ntiles = ti.ntx * ti.nty;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  double *partials = w.partials, *totals = w.partials + kRedStride * (long)nb;
  const double *Ct = w.Ct, *Gx = w.Gx, *Gy = w.Gy;
  double *const X = w.x;
  float *const FD = w.fd;
  if (threadIdx.x == 0) acquire_maps(&m->tfr[0], 6);
  // the inner sweeps' tiles: 128 x 32
  TileIt ti2;
  ti2.ntx = ti.ntx;
  ti2.nty = (ny + kTallTH - 1) / kTallTH;
  ti2.ntiles = ti2.ntx * ti2.nty;

  // ---- setup: x = x0 (FP64, unscaled), FP32 scaled couplings with the row flag
  for (int tile = rank; tile < ti.ntiles; tile += nb) {
    int i0, j0;
    tile_origin(ti, tile, &i0, &j0);
    const int j = j0 + ty;
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      const int i = i0 + c * 32 + tx;
      if (i < nx && j < ny) {
        const long k = g.at(i, j);
        const double ct = Ct[k], ce = Ct[k + 1], cn = Ct[k + pitch];
        const double d = sqrt(fabs(ct));
        double hx = Gx[k] / (d * sqrt(fabs(ce))), hy = Gy[k] / (d * sqrt(fabs(cn)));
        if (elim) {
          if (!(ct > 0 && ce > 0)) hx = 0.0;
          if (!(ct > 0 && cn > 0)) hy = 0.0;
        }
        const float hxf = fabsf((float)hx);
        w.fhx[k] = ct < 0 ? -hxf : hxf;
        w.fhy[k] = (float)hy;
        w.fs[k] = (float)(1.0 / d);
        X[k] = x0_surface ? w.surf_cur[k] : 0.0;
      }
    }
  }
  {
    double none[1] = {0};
    if (!grid_allreduce<1, kRedStride>(none, sc, partials, totals, nb, rank)) return 0;
  }
  auto converged = [&](double rr_, double bn) {
    const double rn = sqrt(rr_);
    return rn < p.eps * bn || (bn == 0.0 && 1.0 + rn == 1.0);
  };
  double rr = 0.0, rr_prev = 0.0, bnorm = 0.0;
  int it_all = 0, done = 0;
  // The correction x += d~ * fs (fs = 1/sqrt|Ct| in FP32: the correction
  // only needs FP32 accuracy, the next residual is exact in FP64 for whatever
  // x results) of an inner solve is applied inside the next residual pass:
  // every cell forms that sum for itself and its neighbours (the same
  // expression, so the same doubles) and writes its own into the other buffer;
  // x then alternates between w.x and w.q (the FP64 solve's work vector, free
  // in this form).
  double *xc = X, *xn = w.q;
  bool add_fd = false;
  for (int outer = 0; outer < kMaxOuter; ++outer) {
    // ---- residual in FP64: r = b - A x; r~ = r/sqrt|Ct| in FP32; p_{-1} = 0
    double acc[3] = {0, 0, 0};
    for (int tile = rank; tile < ti.ntiles; tile += nb) {
      int i0, j0;
      tile_origin(ti, tile, &i0, &j0);
      const int j = j0 + ty;
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        const int i = i0 + c * 32 + tx;
        if (i < nx && j < ny) {
          const long k = g.at(i, j);
          const double ct = Ct[k], bk = w.b[k];
          auto xval = [&](long kk) -> double {
            const double x0 = __ldcg(xc + kk);
            return add_fd ? fma((double)__ldcg(FD + kk), (double)w.fs[kk], x0) : x0;
          };
          auto xv = [&](long kk) -> double {
            const double cc = Ct[kk];
            return (elim && cc < 0) ? w.b[kk] / (-cc) : xval(kk);
          };
          const double xk = xval(k);
          if (add_fd) xn[k] = xk;
          double r;
          if (ct > 0) {
            const double ax = ct * xk - (Gx[k] * xv(k + 1) + Gx[k - 1] * xv(k - 1) +
                                         Gy[k] * xv(k + pitch) + Gy[k - pitch] * xv(k - pitch));
            r = bk - ax;
          } else {
            r = bk - (-ct) * xk;
          }
          const float rs = (float)(r / sqrt(fabs(ct)));
          acc[0] += (double)rs * (double)rs;
          acc[1] += r * r;
          acc[2] += bk * bk;
          w.fr0[k] = rs;
          w.fp0[k] = 0.0f;
        }
      }
    }
    if (!grid_allreduce<3, kRedStride>(acc, sc, partials, totals, nb, rank)) return 0;
    if (add_fd) {  // the corrected x is in the other buffer now
      double *t = xc;
      xc = xn;
      xn = t;
    }
    rr = acc[1];
    if (outer == 0) bnorm = sqrt(acc[2]);
    if (converged(rr, bnorm)) {
      done = 1;
      break;
    }
    if (outer > 0 && rr > 1e-2 * rr_prev) break;  // no tenfold gain: FP64 takes over
    rr_prev = rr;

    // ---- inner FP32 solve of A~ d~ = r~ until (r~, r~) fell by eps_inner^2
    const double g0 = acc[0];
    double gamma = g0, delta;
    {
      double d0[1] = {first_delta<float, kTallTH>(w.fr0, w.fhx, w.fhy, g, ti2, rank, nb, smem)};
      if (!grid_allreduce<1, kRedStride>(d0, sc, partials, totals, nb, rank)) return 0;
      delta = d0[0];
    }
    double gamma_old = 1.0, e1 = 0.0, e2 = 0.0, e3 = 0.0;
    int cur = 0, it = 0;
    const double stop = p.eps_inner * p.eps_inner * g0;
    while (gamma > stop && it < p.maxIter) {
      const double beta = it == 0 ? 0.0 : gamma / gamma_old;
      const double alpha = gamma / (delta + beta * (e1 + e2) + beta * beta * e3);
      ++it;
      float *rn_out = cur ? w.fr0 : w.fr1, *pn_out = cur ? w.fp0 : w.fp1;
      double red[6] = {0, 0, 0, 0, 0, 0};
      const SweepMaps sm{&m->tfr[cur], &m->tfp[cur], &m->tfhx, &m->tfhy};
      // d~ starts from zero at the inner solve's first sweep
      if (!sweep<float, false, float, kTallTH>(sm, rn_out, pn_out, FD, Ct, g, ti2, rank, nb,
                                               (float)alpha, (float)beta, red, smem, bars, seq, sc,
                                               it == 1))
        return 0;
      if (!grid_allreduce<6, kRedStride>(red, sc, partials, totals, nb, rank)) return 0;
      gamma_old = gamma;
      gamma = red[0];
      delta = red[1];
      e1 = red[2];
      e2 = red[3];
      e3 = red[4];
      cur ^= 1;
    }
    it_all += it;
    add_fd = it > 0;  // the next residual pass applies this solve's correction
  }
  if (!done) return 2;
  if (xc != X) {  // the solution in w.x, where the step reads it (own cells; no barrier after)
    for (int tile = rank; tile < ti.ntiles; tile += nb) {
      int i0, j0;
      tile_origin(ti, tile, &i0, &j0);
      const int j = j0 + ty;
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        const int i = i0 + c * 32 + tx;
        if (i < nx && j < ny) {
          const long k = g.at(i, j);
          X[k] = xc[k];
        }
      }
    }
  }
  if (rank == 0 && threadIdx.x == 0) {
    sc->cg_iters = it_all;
    sc->cg_fallback = 0;
    sc->cg_noconv = 0;
    sc->cg_rr = rr;
    sc->cg_bb = bnorm * bnorm;
  }
  return 1;
}

// The domain's solve in its configured precision.
// kMix: the kernel carries the mixed-precision path too (its FP32 tall-tile
// sweeps cost registers that the FP64-only kernels do not pay).
template <bool kMix>
static __device__ __forceinline__ bool cg1_solve(const View &w, const Cg1Maps *__restrict__ m,
                                                 int x0_surface, int eliminate, unsigned rank,
                                                 unsigned nb, unsigned char *smem,
                                                 unsigned long long *bars, unsigned &seq) {
  if (test_skip_barrier(w.sc, rank)) {  // a lone CTA has no partner whose wait could run out
    if (nb == 1 && threadIdx.x == 0) set_status(w.sc, FREHD_ERR_TIMEOUT);
    return false;
  }
  if (kMix && w.p.mixed) {
    const int r = cg1_mixed(w, m, x0_surface, eliminate, rank, nb, smem, bars, seq);
    if (r != 2) return r == 1;
    const bool ok = cg1_fp64(w, m, x0_surface, eliminate, rank, nb, smem, bars, seq);
    if (ok && rank == 0 && threadIdx.x == 0) w.sc->cg_fallback = 2;
    return ok;
  }
  return cg1_fp64(w, m, x0_surface, eliminate, rank, nb, smem, bars, seq);
}

// Dynamic shared memory of one CTA: two stages and two mbarriers, the base
// rounded up to 128 bytes (the region after the static shared data is only
// 16-byte aligned; the launch requests 128 bytes of slack).  False if an
// alignment the TMA needs does not hold.
static __device__ __forceinline__ bool cg1_smem(unsigned char *smem_raw, unsigned char **smem,
                                                unsigned long long **bars) {
  *smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  *bars = reinterpret_cast<unsigned long long *>(*smem + kSmemStages);
  if ((smem_u32(*smem) & 127u) || (smem_u32(*bars) & 7u)) return false;
  if (threadIdx.x == 0) {
    mbar_init(&(*bars)[0], 1);
    mbar_init(&(*bars)[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  return true;
}

template <bool kMix>
__global__ void __launch_bounds__(kCgThreads, kCg1MinBlocks)
    k_cg1(View w, const Cg1Maps *__restrict__ m, int x0_surface, int eliminate) {
  if (*(volatile int *)&w.sc->status != FREHD_OK) return;
  extern __shared__ unsigned char smem_raw[];
  unsigned char *smem;
  unsigned long long *bars;
  // TMA destinations 128-byte aligned, mbarriers 8-byte aligned, tensor maps
  // 64-byte aligned: refuse (every block alike) otherwise
  if (!cg1_smem(smem_raw, &smem, &bars) || (reinterpret_cast<unsigned long long>(m) & 63ull)) {
    if (threadIdx.x == 0) set_status(w.sc, FREHD_ERR_CUDA);
    return;
  }
  // the solve reads the view from shared memory
  __shared__ View s_view;
  {
    const unsigned long long *src = reinterpret_cast<const unsigned long long *>(&w);
    unsigned long long *dst = reinterpret_cast<unsigned long long *>(&s_view);
    for (int e = threadIdx.x; e < (int)(sizeof(View) / 8); e += blockDim.x) dst[e] = src[e];
  }
  __syncthreads();
  unsigned seq = 0;
  cg1_solve<kMix>(s_view, m, x0_surface, eliminate, blockIdx.x, gridDim.x, smem, bars, seq);
}

// Batched solve: CTA c first runs jobs[job_start[c] .. job_start[c+1]) in
// order (its share of a multi-CTA domain's solve: rank `rank` of a group of
// `nb` CTAs, all co-resident in this cooperative launch), then takes
// single-CTA solves from the shared list `singles` (largest first; *taken
// counts the entries handed out, zero at the launch) until none is left, so
// that the CTAs which finish early carry the rest.  A single-CTA domain's solve
// is the same whichever CTA runs it.  Each domain's view is taken at its
// current parity.
template <bool kMix>
__global__ void __launch_bounds__(kCgThreads, kCg1MinBlocks)
    k_cg1_batch(const View *__restrict__ views2, const Cg1Maps *const *__restrict__ maps,
                const int *__restrict__ job_start, const CgJob *__restrict__ jobs,
                const CgJob *__restrict__ singles, int nsingles, int *taken) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ View s_view;
  __shared__ int s_cur, s_next;
  unsigned char *smem;
  unsigned long long *bars;
  const int q0 = job_start[blockIdx.x], q1 = job_start[blockIdx.x + 1];
  const bool aligned = cg1_smem(smem_raw, &smem, &bars);
  unsigned seq = 0;
  const int nstatic = q1 - q0;
  for (int n = 0;; ++n) {
    CgJob jb;
    if (n < nstatic) {
      jb = jobs[q0 + n];
    } else {
      __syncthreads();  // every thread read the previous s_next
      if (threadIdx.x == 0) s_next = atomicAdd(taken, 1);
      __syncthreads();
      if (s_next >= nsingles) break;
      jb = singles[s_next];
    }
    __syncthreads();  // the previous job is done with s_view
    if (threadIdx.x == 0) s_cur = *(volatile int *)&views2[2 * jb.d].sc->cur;
    __syncthreads();
    {
      const unsigned long long *src =
          reinterpret_cast<const unsigned long long *>(views2 + 2 * jb.d + s_cur);
      unsigned long long *dst = reinterpret_cast<unsigned long long *>(&s_view);
      for (int e = threadIdx.x; e < (int)(sizeof(View) / 8); e += blockDim.x) dst[e] = src[e];
    }
    __syncthreads();
    if (*(volatile int *)&s_view.sc->status != FREHD_OK) continue;
    if (!aligned || (reinterpret_cast<unsigned long long>(maps[jb.d]) & 63ull)) {
      if (threadIdx.x == 0) set_status(s_view.sc, FREHD_ERR_CUDA);
      continue;
    }
    if (!cg1_solve<kMix>(s_view, maps[jb.d], jb.flags & 1, (jb.flags >> 1) & 1, jb.rank, jb.nb, smem,
                         bars, seq)) {
      // this CTA's later static jobs are not run: mark their domains failed (the
      // shared list's remaining entries go to the other CTAs)
      for (int r = q0 + n + 1; r < q1; ++r)
        if (threadIdx.x == 0) set_status(views2[2 * jobs[r].d].sc, FREHD_ERR_TIMEOUT);
      return;
    }
  }
}

// ================================================================ batched solve, one tile list
//
// Every domain of a batch is solved by one cooperative launch of all co-resident
// CTAs.  The domains' CG tiles form one list (domain after domain, each in its
// own tile order) and CTA c works on entries c, c + C, c + 2C, ... (C CTAs), so
// that every domain's work, large or small, is spread over the whole GPU.  The
// solve runs in rounds: in a round every tile takes one step of its domain's
// state machine (a set-up pass, one CG sweep, the final scaling; or the mixed
// form's residual, inner sweep and correction passes), and writes the sums that
// step needs to the tile's own slot of `part`; after a grid barrier, domain k's
// slots are added up in tile order by CTA k mod C, which advances the domain's
// state (the scalars of the next sweep, convergence, the stall and precision
// fall-backs); a second barrier publishes the states.  A domain's arithmetic
// thus depends on its own tiles only: its result is the same alone, in any mix
// and for any number of CTAs.  The steps are those of cg1_fp64 and cg1_mixed
// (same passes, same stopping rules, same fall-backs); only the order in which
// the partial sums are added differs.
// Arguments of k_cg1_tiles (the host's tables of the batch composition).
struct TilesArgs {
  const View *views2;
  const Cg1Maps *const *maps;
  const BDom *doms;
  BState *states;
  const BTile *tiles;
  int ndom, ntiles;
  double *part;
  Scratch *bsync;
  double *bpart;
};

namespace {

enum : int {
  kPhSetup1 = 0, kPhSetup2, kPhDelta0, kPhSweep, kPhFinal,
  kPhMSetup, kPhMResid, kPhMDelta0, kPhMSweep, kPhMXupd, kPhDone
};
constexpr int kMaxAcqDomains = 4096;  // domains whose tensor maps a CTA tracks as acquired
constexpr int kTlMaxDoms = 512;       // domains whose round parameters a CTA keeps in shared memory
constexpr int kTlMaxLocal = 1024;     // a CTA's list entries kept in shared memory

// What a tile of domain k needs in a round: its state's phase and sweep
// scalars, and the domain's place (copied to shared memory at each round's start).
struct TlDom {
  double alpha, beta;
  int phase, cur, vpar, elim, slot, ntx, ntiles, flags;
};
constexpr unsigned kStageStride = kSmemStages / 2;  // one stage of either element type

// A domain's state as published by the last round (L2: written by another CTA).
__device__ __forceinline__ BState load_state(const BState *p) {
  static_assert(sizeof(BState) % 8 == 0, "BState is copied in 8-byte words");
  BState st;
  const unsigned long long *src = reinterpret_cast<const unsigned long long *>(p);
  unsigned long long *dst = reinterpret_cast<unsigned long long *>(&st);
#pragma unroll
  for (int q = 0; q < (int)(sizeof(BState) / 8); ++q) dst[q] = __ldcg(src + q);
  return st;
}
__device__ __forceinline__ int load_phase(const BState *p) { return __ldcg(&p->phase); }

__device__ __forceinline__ bool is_sweep(int ph) { return ph == kPhSweep || ph == kPhMSweep; }

// sums a phase's tiles produce
__device__ __forceinline__ int phase_sums(int ph) {
  switch (ph) {
    case kPhSetup2: case kPhMResid: return 3;
    case kPhDelta0: case kPhMDelta0: return 1;
    case kPhSweep: case kPhMSweep: return 6;
    default: return 0;
  }
}

// A~ v at padded index k read from global memory: apply() on the arrays
// themselves (zeros outside the interior), the same products and order.
template <typename T>
__device__ __forceinline__ T apply_g(const T *V, const T *HX, const T *HY, long k, long pitch) {
  const T he = __ldcg(HX + k);
  const T off = fabs(he) * __ldcg(V + k + 1) + fabs(__ldcg(HX + k - 1)) * __ldcg(V + k - 1) +
                __ldcg(HY + k) * __ldcg(V + k + pitch) + __ldcg(HY + k - pitch) * __ldcg(V + k - pitch);
  return signbit(he) ? __ldcg(V + k) : __ldcg(V + k) - off;
}

// ---- plain passes of one tile (cg1_fp64 / cg1_mixed, per tile)
__device__ __forceinline__ void t_setup1(const View &w, int i0, int j0, int elim, int x0s) {
  const Grid g = w.gr;
  const long pitch = g.pitch;
  const int tx = threadIdx.x & 31, j = j0 + (threadIdx.x >> 5);
  const double *Ct = w.Ct, *Gx = w.Gx, *Gy = w.Gy;
#pragma unroll
  for (int c = 0; c < CPT; ++c) {
    const int i = i0 + c * 32 + tx;
    if (i < g.nx && j < g.ny) {
      const long k = g.at(i, j);
      const double ct = Ct[k], ce = Ct[k + 1], cn = Ct[k + pitch];
      const double d = sqrt(fabs(ct));
      double hx = Gx[k] / (d * sqrt(fabs(ce))), hy = Gy[k] / (d * sqrt(fabs(cn)));
      if (elim) {
        if (!(ct > 0 && ce > 0)) hx = 0.0;
        if (!(ct > 0 && cn > 0)) hy = 0.0;
      }
      w.Hx[k] = ct < 0 ? -fabs(hx) : fabs(hx);
      w.Hy[k] = hy;
      w.x[k] = x0s ? d * w.surf_cur[k] : 0.0;
      w.p0[k] = 0.0;
    }
  }
}

__device__ __forceinline__ void t_setup2(const View &w, int i0, int j0, int elim, int x0s,
                                         double (&acc)[6]) {
  const Grid g = w.gr;
  const long pitch = g.pitch;
  const int tx = threadIdx.x & 31, j = j0 + (threadIdx.x >> 5);
  const double *Ct = w.Ct, *Gx = w.Gx, *Gy = w.Gy;
#pragma unroll
  for (int c = 0; c < CPT; ++c) {
    const int i = i0 + c * 32 + tx;
    if (i < g.nx && j < g.ny) {
      const long k = g.at(i, j);
      const double ct = Ct[k], bk = w.b[k];
      auto x0 = [&](long kk) -> double { return x0s ? w.surf_cur[kk] : 0.0; };
      auto xv = [&](long kk) -> double {
        const double cc = Ct[kk];
        return (elim && cc < 0) ? w.b[kk] / (-cc) : x0(kk);
      };
      double r;
      if (ct > 0) {
        const double ax = ct * x0(k) - (Gx[k] * xv(k + 1) + Gx[k - 1] * xv(k - 1) +
                                        Gy[k] * xv(k + pitch) + Gy[k - pitch] * xv(k - pitch));
        r = bk - ax;
      } else {
        r = bk - (-ct) * x0(k);
      }
      const double rs = r / sqrt(fabs(ct));
      acc[0] += rs * rs;
      acc[1] += r * r;
      acc[2] += bk * bk;
      w.r[k] = rs;
    }
  }
}

template <typename T>
__device__ __forceinline__ void t_delta0(const Grid &g, const T *V, const T *HX, const T *HY, int i0,
                                         int j0, double (&acc)[6]) {
  const int tx = threadIdx.x & 31, j = j0 + (threadIdx.x >> 5);
#pragma unroll
  for (int c = 0; c < CPT; ++c) {
    const int i = i0 + c * 32 + tx;
    if (i < g.nx && j < g.ny) {
      const long k = g.at(i, j);
      acc[0] += (double)apply_g<T>(V, HX, HY, k, g.pitch) * (double)__ldcg(V + k);
    }
  }
}

__device__ __forceinline__ void t_final(const View &w, int i0, int j0) {
  const Grid g = w.gr;
  const int tx = threadIdx.x & 31, j = j0 + (threadIdx.x >> 5);
#pragma unroll
  for (int c = 0; c < CPT; ++c) {
    const int i = i0 + c * 32 + tx;
    if (i < g.nx && j < g.ny) {
      const long k = g.at(i, j);
      w.x[k] = w.x[k] / sqrt(fabs(w.Ct[k]));
    }
  }
}

__device__ __forceinline__ void t_msetup(const View &w, int i0, int j0, int elim, int x0s) {
  const Grid g = w.gr;
  const long pitch = g.pitch;
  const int tx = threadIdx.x & 31, j = j0 + (threadIdx.x >> 5);
  const double *Ct = w.Ct, *Gx = w.Gx, *Gy = w.Gy;
#pragma unroll
  for (int c = 0; c < CPT; ++c) {
    const int i = i0 + c * 32 + tx;
    if (i < g.nx && j < g.ny) {
      const long k = g.at(i, j);
      const double ct = Ct[k], ce = Ct[k + 1], cn = Ct[k + pitch];
      const double d = sqrt(fabs(ct));
      double hx = Gx[k] / (d * sqrt(fabs(ce))), hy = Gy[k] / (d * sqrt(fabs(cn)));
      if (elim) {
        if (!(ct > 0 && ce > 0)) hx = 0.0;
        if (!(ct > 0 && cn > 0)) hy = 0.0;
      }
      const float hxf = fabsf((float)hx);
      w.fhx[k] = ct < 0 ? -hxf : hxf;
      w.fhy[k] = (float)hy;
      w.x[k] = x0s ? w.surf_cur[k] : 0.0;
    }
  }
}

__device__ __forceinline__ void t_mresid(const View &w, int i0, int j0, int elim, double (&acc)[6]) {
  const Grid g = w.gr;
  const long pitch = g.pitch;
  const int tx = threadIdx.x & 31, j = j0 + (threadIdx.x >> 5);
  const double *Ct = w.Ct, *Gx = w.Gx, *Gy = w.Gy;
  double *const X = w.x;
#pragma unroll
  for (int c = 0; c < CPT; ++c) {
    const int i = i0 + c * 32 + tx;
    if (i < g.nx && j < g.ny) {
      const long k = g.at(i, j);
      const double ct = Ct[k], bk = w.b[k];
      auto xv = [&](long kk) -> double {
        const double cc = Ct[kk];
        return (elim && cc < 0) ? w.b[kk] / (-cc) : __ldcg(X + kk);
      };
      double r;
      if (ct > 0) {
        const double ax = ct * __ldcg(X + k) - (Gx[k] * xv(k + 1) + Gx[k - 1] * xv(k - 1) +
                                                Gy[k] * xv(k + pitch) + Gy[k - pitch] * xv(k - pitch));
        r = bk - ax;
      } else {
        r = bk - (-ct) * __ldcg(X + k);
      }
      const float rs = (float)(r / sqrt(fabs(ct)));
      acc[0] += (double)rs * (double)rs;
      acc[1] += r * r;
      acc[2] += bk * bk;
      w.fr0[k] = rs;
      w.fp0[k] = 0.0f;
      w.fd[k] = 0.0f;
    }
  }
}

__device__ __forceinline__ void t_xupd(const View &w, int i0, int j0) {
  const Grid g = w.gr;
  const int tx = threadIdx.x & 31, j = j0 + (threadIdx.x >> 5);
#pragma unroll
  for (int c = 0; c < CPT; ++c) {
    const int i = i0 + c * 32 + tx;
    if (i < g.nx && j < g.ny) {
      const long k = g.at(i, j);
      w.x[k] = w.x[k] + (double)__ldcg(w.fd + k) / sqrt(fabs(w.Ct[k]));
    }
  }
}

// One CG sweep of one tile whose boxes are in stage `s` (sweep()'s passes A-C):
// p = r~ + beta p_old, s = A~ p, r~' = r~ - alpha s, w = A~ r~', X += alpha p;
// r~' and p stored to rn_out / pn_out; red gets the tile's six sums.
template <typename T, bool kUnscaled, typename XT>
__device__ __forceinline__ void sweep_tile(const Stage<T> &s, const Grid &g, int i0, int j0,
                                           const XT (&xs)[CPT], const double (&ds)[CPT], XT *X,
                                           T *rn_out, T *pn_out, T alpha, T beta, double (&red)[6]) {
  using B = Box<T>;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int j = j0 + ty;
  {
    using P2 = typename Pair<T>::type;
    P2 *pp = reinterpret_cast<P2 *>(s.P);
    const P2 *rp = reinterpret_cast<const P2 *>(s.R);
#pragma unroll
    for (int e = threadIdx.x; e < B::kBox / 2; e += kCgThreads) {
      const P2 rv = rp[e];
      P2 pv = pp[e];
      pv.x = rv.x + beta * pv.x;
      pv.y = rv.y + beta * pv.y;
      pp[e] = pv;
    }
  }
  __syncthreads();
  {
    T rb[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      const int q = B::q(c * 32 + tx, ty);
      const T sv = apply<T>(s.P, s.HX, s.HY, q);
      rb[c] = s.R[q] - alpha * sv;
      if (i0 + c * 32 + tx < g.nx && j < g.ny) {
        red[2] += (double)rb[c] * (double)sv;
        red[4] += (double)s.P[q] * (double)sv;
      }
    }
    T rring[B::kRingPer];
    int qr[B::kRingPer];
#pragma unroll
    for (int t = 0; t < B::kRingPer; ++t) {
      const int e = threadIdx.x + t * kCgThreads;
      qr[t] = e < B::kRing ? B::ring(e) : 0;
      rring[t] = e < B::kRing ? s.R[qr[t]] - alpha * apply<T>(s.P, s.HX, s.HY, qr[t]) : T(0);
    }
#pragma unroll
    for (int c = 0; c < CPT; ++c) s.R[B::q(c * 32 + tx, ty)] = rb[c];
#pragma unroll
    for (int t = 0; t < B::kRingPer; ++t)
      if (threadIdx.x + t * kCgThreads < B::kRing) s.R[qr[t]] = rring[t];
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < CPT; ++c) {
    const int i = i0 + c * 32 + tx;
    if (i < g.nx && j < g.ny) {
      const int q = B::q(c * 32 + tx, ty);
      const T u = s.R[q], pc = s.P[q];
      const T wv = apply<T>(s.R, s.HX, s.HY, q);
      const double ud = u;
      red[0] += ud * ud;
      red[1] += (double)wv * ud;
      red[3] += (double)pc * (double)wv;
      red[5] += kUnscaled ? ds[c] * (ud * ud) : ud * ud;
      const long k = g.at(i, j);
      X[k] = xs[c] + alpha * pc;
      rn_out[k] = u;
      pn_out[k] = pc;
    }
  }
}

__device__ __forceinline__ const View &tile_view(const TilesArgs &a, const BDom &dm, int vpar) {
  return a.views2[2 * dm.slot + vpar];
}

// Mark every domain of the launch failed (a wait that gave up strands them all).
__device__ __forceinline__ void fail_all(const TilesArgs &a, int code) {
  if (threadIdx.x != 0) return;
  for (int k = 0; k < a.ndom; ++k) set_status(a.views2[2 * a.doms[k].slot].sc, code);
}

// The round parameters of domain k from its published state.
__device__ __forceinline__ TlDom load_tldom(const TilesArgs &a, int k) {
  const BState st = load_state(a.states + k);
  const BDom dm = a.doms[k];
  TlDom t;
  t.alpha = st.alpha;
  t.beta = st.beta;
  t.phase = st.phase;
  t.cur = st.cur;
  t.vpar = st.vpar;
  t.elim = st.elim;
  t.slot = dm.slot;
  t.ntx = dm.ntx;
  t.ntiles = dm.ntiles;
  t.flags = dm.flags;
  return t;
}

// The CTA's shared copies: round parameters of the first kTlMaxDoms domains and
// its first kTlMaxLocal list entries; the rest is read from global memory.
struct TlCache {
  const TlDom *dom;
  const BTile *loc;
  __device__ __forceinline__ TlDom get_dom(const TilesArgs &a, int k) const {
    return k < kTlMaxDoms ? dom[k] : load_tldom(a, k);
  }
  __device__ __forceinline__ BTile get_tile(const TilesArgs &a, int idx, unsigned c, unsigned C) const {
    return idx < kTlMaxLocal ? loc[idx] : a.tiles[(long)c + (long)idx * C];
  }
};

// Issue the boxes of the sweep tile (list entry t of domain parameters dm) into
// stage buffer `stage` (thread 0).
__device__ __forceinline__ void issue_sweep(const TilesArgs &a, const BTile &t, const TlDom &dm,
                                            unsigned char *stage, unsigned long long *bar,
                                            unsigned *acq) {
  const Cg1Maps *m = a.maps[dm.slot];
  const bool fp32 = dm.phase == kPhMSweep;
  // the maps were written by host copies: acquire them once per domain and precision
  const int bit = 2 * t.dom + (fp32 ? 1 : 0);
  if (t.dom >= kMaxAcqDomains || !((acq[bit >> 5] >> (bit & 31)) & 1u)) {
    acquire_maps(fp32 ? &m->fr[0] : &m->r[0], 6);
    if (t.dom < kMaxAcqDomains) acq[bit >> 5] |= 1u << (bit & 31);
  }
  TileIt ti;
  ti.ntx = dm.ntx;
  ti.ntiles = dm.ntiles;
  ti.nty = dm.ntiles / dm.ntx;
  if (fp32) {
    const SweepMaps sm{&m->fr[dm.cur], &m->fp[dm.cur], &m->fhx, &m->fhy};
    issue_tile<float>(sm, ti, t.tile, stage, bar);
  } else {
    const SweepMaps sm{&m->r[dm.cur], &m->p[dm.cur], &m->hx, &m->hy};
    issue_tile<double>(sm, ti, t.tile, stage, bar);
  }
}

// The CTA's next local list index at or after idx whose domain sweeps this round
// (n: the CTA's entry count).
__device__ __forceinline__ int next_sweep(const TilesArgs &a, const TlCache &tc, int idx, int n,
                                          unsigned c, unsigned C) {
  for (; idx < n; ++idx)
    if (is_sweep(tc.get_dom(a, tc.get_tile(a, idx, c, C).dom).phase)) return idx;
  return n;
}

// Advance domain k's state after its sums `tot` of this round (thread 0).
__device__ void advance(const TilesArgs &a, int k, BState &st, const double (&tot)[6]) {
  const BDom dm = a.doms[k];
  const View &w = tile_view(a, dm, st.vpar);
  const Params &p = w.p;
  Scratch *sc = w.sc;
  auto converged = [&](double rr_, double bn) {
    const double rn = sqrt(rr_);
    return rn < p.eps * bn || (bn == 0.0 && 1.0 + rn == 1.0);
  };
  auto finish = [&](int iters, int fallback, int noconv) {
    sc->cg_iters = iters;
    sc->cg_fallback = fallback;
    sc->cg_noconv = noconv;
    sc->cg_rr = st.rr;
    sc->cg_bb = st.bnorm * st.bnorm;
    st.phase = kPhDone;
    atomicAdd(&a.bsync->n_done, 1);
  };
  // the next FP64 sweep, or the end of the solve (cg1_fp64's loop condition)
  auto next_fp64 = [&]() {
    if (!converged(st.rr, st.bnorm) && st.it < p.maxIter) {
      st.beta = st.it == 0 ? 0.0 : st.gamma / st.gamma_old;
      st.alpha = st.gamma / (st.delta + st.beta * (st.e1 + st.e2) + st.beta * st.beta * st.e3);
      ++st.it;
      st.phase = kPhSweep;
    } else {
      st.it_all += st.it;
      st.noconv = !converged(st.rr, st.bnorm);
      st.phase = kPhFinal;
    }
  };
  // the next FP32 inner sweep, or the correction pass (cg1_mixed's inner loop)
  auto next_inner = [&]() {
    if (st.gamma > st.stop && st.it < p.maxIter) {
      st.beta = st.it == 0 ? 0.0 : st.gamma / st.gamma_old;
      st.alpha = st.gamma / (st.delta + st.beta * (st.e1 + st.e2) + st.beta * st.beta * st.e3);
      ++st.it;
      st.phase = kPhMSweep;
    } else {
      st.it_all += st.it;
      st.phase = kPhMXupd;
    }
  };
  // the mixed refinement hands the solve to the FP64 path (cg1_solve)
  auto take_over = [&]() {
    st.takeover = 1;
    st.attempt = 0;
    st.elim = (dm.flags >> 1) & 1;
    st.it_all = 0;
    st.fallback = 0;
    st.phase = kPhSetup1;
  };
  switch (st.phase) {
    case kPhSetup1:
      st.phase = kPhSetup2;
      break;
    case kPhSetup2:
      st.gamma = tot[0];
      st.rr = tot[1];
      st.bnorm = sqrt(tot[2]);
      st.phase = kPhDelta0;
      break;
    case kPhDelta0:
      st.delta = tot[0];
      st.gamma_old = 1.0;
      st.e1 = st.e2 = st.e3 = 0.0;
      st.best = st.rr;
      st.best_it = 0;
      st.cur = 0;
      st.it = 0;
      next_fp64();
      break;
    case kPhSweep:
      st.gamma_old = st.gamma;
      st.gamma = tot[0];
      st.delta = tot[1];
      st.e1 = tot[2];
      st.e2 = tot[3];
      st.e3 = tot[4];
      st.rr = tot[5];
      st.cur ^= 1;
      if (st.rr < 0.25 * st.best) {
        st.best = st.rr;
        st.best_it = st.it;
      } else if (!st.elim && st.it - st.best_it >= kStallIters) {
        // stalled on the assembled matrix: start again in the eliminated form
        st.it_all += st.it;
        st.attempt += 1;
        st.elim = 1;
        st.fallback = 1;
        st.phase = kPhSetup1;
        break;
      }
      next_fp64();
      break;
    case kPhFinal:
      finish(st.it_all, st.takeover ? 2 : st.fallback, st.noconv);
      break;
    case kPhMSetup:
      st.outer = 0;
      st.phase = kPhMResid;
      break;
    case kPhMResid:
      st.rr = tot[1];
      if (st.outer == 0) st.bnorm = sqrt(tot[2]);
      if (converged(st.rr, st.bnorm)) {
        finish(st.it_all, 0, 0);
      } else if (st.outer > 0 && st.rr > 1e-2 * st.rr_prev) {
        take_over();  // no tenfold gain
      } else {
        st.rr_prev = st.rr;
        st.gamma = tot[0];  // g0 of the inner solve
        st.stop = p.eps_inner * p.eps_inner * tot[0];
        st.phase = kPhMDelta0;
      }
      break;
    case kPhMDelta0:
      st.delta = tot[0];
      st.gamma_old = 1.0;
      st.e1 = st.e2 = st.e3 = 0.0;
      st.cur = 0;
      st.it = 0;
      next_inner();
      break;
    case kPhMSweep:
      st.gamma_old = st.gamma;
      st.gamma = tot[0];
      st.delta = tot[1];
      st.e1 = tot[2];
      st.e2 = tot[3];
      st.e3 = tot[4];
      st.cur ^= 1;
      next_inner();
      break;
    case kPhMXupd:
      st.outer += 1;
      if (st.outer < kMaxOuter) st.phase = kPhMResid;
      else take_over();
      break;
    default:
      break;
  }
}

}  // namespace

__global__ void __launch_bounds__(kCgThreads, kCg1MinBlocks) k_cg1_tiles(TilesArgs a) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ double sh_red[2][6][NWARP];
  __shared__ unsigned s_acq[2 * kMaxAcqDomains / 32];
  __shared__ TlDom s_dom[kTlMaxDoms];
  __shared__ BTile s_loc[kTlMaxLocal];
  __shared__ int s_ok, s_next;
  unsigned char *smem;
  unsigned long long *bars;
  const unsigned C = gridDim.x, c = blockIdx.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (!cg1_smem(smem_raw, &smem, &bars)) {  // every CTA alike: nobody reaches a barrier
    if (c == 0) fail_all(a, FREHD_ERR_CUDA);
    return;
  }
  const TlCache tc{s_dom, s_loc};
  // this CTA's list entries: c, c + C, c + 2C, ...
  const int nloc = a.ntiles > (int)c ? (a.ntiles - (int)c + (int)C - 1) / (int)C : 0;
  for (int q = threadIdx.x; q < 2 * kMaxAcqDomains / 32; q += blockDim.x) s_acq[q] = 0;
  for (int q = threadIdx.x; q < nloc && q < kTlMaxLocal; q += blockDim.x)
    s_loc[q] = a.tiles[(long)c + (long)q * C];
  // ---- prologue: each CTA starts the solves of its domains
  if (threadIdx.x == 0) {
    for (int k = (int)c; k < a.ndom; k += (int)C) {
      const BDom dm = a.doms[k];
      Scratch *sc = a.views2[2 * dm.slot].sc;
      BState st;
      memset(&st, 0, sizeof(st));
      st.vpar = *(volatile int *)&sc->cur & 1;
      const View &w = a.views2[2 * dm.slot + st.vpar];
      st.elim = (dm.flags >> 1) & 1;
      if (*(volatile int *)&sc->status != FREHD_OK || (reinterpret_cast<unsigned long long>(a.maps[dm.slot]) & 63ull)) {
        if (*(volatile int *)&sc->status == FREHD_OK) set_status(sc, FREHD_ERR_CUDA);
        st.phase = kPhDone;
        atomicAdd(&a.bsync->n_done, 1);
      } else if (test_skip_barrier(sc, 0)) {  // the test hook of frehd_domain_set_wait_test
        set_status(sc, FREHD_ERR_TIMEOUT);
        st.phase = kPhDone;
        atomicAdd(&a.bsync->n_done, 1);
      } else {
        st.phase = w.p.mixed ? kPhMSetup : kPhSetup1;
      }
      a.states[k] = st;
    }
  }
  {
    double none[1] = {0};
    if (!grid_allreduce<1, kRedStride>(none, a.bsync, a.bpart, a.bpart + kRedStride * (long)C, C, c)) {
      fail_all(a, FREHD_ERR_TIMEOUT);
      return;
    }
  }
  unsigned seq = 0;
  int rbuf = 0;
  for (;;) {
    // ---- this round's parameters of every domain, then one step of every tile
    for (int k = threadIdx.x; k < a.ndom && k < kTlMaxDoms; k += blockDim.x) s_dom[k] = load_tldom(a, k);
    __syncthreads();
    if (threadIdx.x == 0) {
      asm volatile("fence.proxy.async.global;" ::: "memory");
      s_next = next_sweep(a, tc, 0, nloc, c, C);
      if (s_next < nloc) {
        const BTile t = tc.get_tile(a, s_next, c, C);
        issue_sweep(a, t, tc.get_dom(a, t.dom), smem + (seq & 1) * kStageStride, &bars[seq & 1], s_acq);
      }
    }
    __syncthreads();
    for (int idx = 0; idx < nloc; ++idx) {
      const long g = (long)c + (long)idx * C;
      const BTile t = tc.get_tile(a, idx, c, C);
      const TlDom dm = tc.get_dom(a, t.dom);  // the same in every thread this round
      const int ph = dm.phase;
      if (ph == kPhDone) continue;
      const View &w = a.views2[2 * dm.slot + dm.vpar];
      const int i0 = (t.tile % dm.ntx) * CTX, j0 = (t.tile / dm.ntx) * CTY;
      double acc[6] = {0, 0, 0, 0, 0, 0};
      const int nv = phase_sums(ph);
      if (is_sweep(ph)) {
        const int st_idx = seq & 1;
        unsigned char *stage = smem + st_idx * kStageStride;
        const Grid gr = w.gr;
        const int tx = threadIdx.x & 31, j = j0 + (threadIdx.x >> 5);
        const bool fp32 = ph == kPhMSweep;
        if (threadIdx.x == 0) {  // the next sweep tile's boxes, into the other stage
          const int i2 = next_sweep(a, tc, idx + 1, nloc, c, C);
          s_next = i2;
          if (i2 < nloc) {
            const BTile t2 = tc.get_tile(a, i2, c, C);
            issue_sweep(a, t2, tc.get_dom(a, t2.dom), smem + (st_idx ^ 1) * kStageStride,
                        &bars[st_idx ^ 1], s_acq);
          }
        }
        // X and |Ct| of the owned cells: in flight while the boxes arrive
        double xs[CPT], ds[CPT];
        float fxs[CPT];
#pragma unroll
        for (int cc = 0; cc < CPT; ++cc) {
          const int i = i0 + cc * 32 + tx;
          const bool in = i < gr.nx && j < gr.ny;
          const long k = gr.at(in ? i : 0, in ? j : 0);
          if (fp32) {
            fxs[cc] = w.fd[k];
            xs[cc] = 0.0;
            ds[cc] = 0.0;
          } else {
            xs[cc] = w.x[k];
            ds[cc] = fabs(w.Ct[k]);
            fxs[cc] = 0.0f;
          }
        }
        if (threadIdx.x == 0) s_ok = mbar_wait(&bars[st_idx], (seq >> 1) & 1, kBarrierTimeoutNs);
        __syncthreads();
        if (!s_ok) {
          if (threadIdx.x == 0) {
            fail_all(a, FREHD_ERR_TIMEOUT);
            if (s_next < nloc) mbar_wait(&bars[st_idx ^ 1], ((seq + 1) >> 1) & 1, kBarrierTimeoutNs);
          }
          return;
        }
        mbar_wait(&bars[st_idx], (seq >> 1) & 1, kBarrierTimeoutNs);  // acquire in every thread
        if (fp32) {
          float *rn_out = dm.cur ? w.fr0 : w.fr1, *pn_out = dm.cur ? w.fp0 : w.fp1;
          sweep_tile<float, false, float>(Stage<float>(stage), gr, i0, j0, fxs, ds, w.fd, rn_out,
                                          pn_out, (float)dm.alpha, (float)dm.beta, acc);
        } else {
          double *rn_out = dm.cur ? w.r : w.q, *pn_out = dm.cur ? w.p0 : w.p1;
          sweep_tile<double, true, double>(Stage<double>(stage), gr, i0, j0, xs, ds, w.x, rn_out,
                                           pn_out, dm.alpha, dm.beta, acc);
        }
        ++seq;
      } else {
        const int x0s = dm.flags & 1;
        switch (ph) {
          case kPhSetup1: t_setup1(w, i0, j0, dm.elim, x0s); break;
          case kPhSetup2: t_setup2(w, i0, j0, dm.elim, x0s, acc); break;
          case kPhDelta0: t_delta0<double>(w.gr, w.r, w.Hx, w.Hy, i0, j0, acc); break;
          case kPhFinal: t_final(w, i0, j0); break;
          case kPhMSetup: t_msetup(w, i0, j0, dm.elim, x0s); break;
          case kPhMResid: t_mresid(w, i0, j0, dm.elim, acc); break;
          case kPhMDelta0: t_delta0<float>(w.gr, w.fr0, w.fhx, w.fhy, i0, j0, acc); break;
          case kPhMXupd: t_xupd(w, i0, j0); break;
          default: break;
        }
      }
      if (nv) {  // the tile's sums, added in a fixed order, into its slot
#pragma unroll
        for (int m = 0; m < 6; ++m)
          if (m < nv) {
            const double v = warp_sum(acc[m]);
            if (lane == 0) sh_red[rbuf][m][wid] = v;
          }
        __syncthreads();
        if (threadIdx.x < nv) {
          double sum = 0;
          for (int q = 0; q < NWARP; ++q) sum += sh_red[rbuf][threadIdx.x][q];
          a.part[g * kTilePartStride + threadIdx.x] = sum;
        }
        rbuf ^= 1;
      } else if (is_sweep(ph)) {
        __syncthreads();  // the stage is free for the tile after next
      }
    }
    // this thread's global writes before the next round's TMA reads (other CTAs)
    asm volatile("fence.proxy.async.global;" ::: "memory");
    {
      double none[1] = {0};
      if (!grid_allreduce<1, kRedStride>(none, a.bsync, a.bpart, a.bpart + kRedStride * (long)C, C, c)) {
        fail_all(a, FREHD_ERR_TIMEOUT);
        return;
      }
    }
    // ---- reduce: domain k by CTA k mod C, its tiles' sums in tile order
    for (int k = (int)c; k < a.ndom; k += (int)C) {
      BState st = load_state(a.states + k);
      __syncthreads();  // every thread read the state before thread 0 may replace it
      if (st.phase == kPhDone) continue;
      const BDom dm = a.doms[k];
      const int nv = phase_sums(st.phase);
      double tot[6] = {0, 0, 0, 0, 0, 0};
      if (nv) {
        double v[6] = {0, 0, 0, 0, 0, 0};
        for (int q = threadIdx.x; q < dm.ntiles; q += blockDim.x)
#pragma unroll
          for (int m = 0; m < 6; ++m)
            if (m < nv) v[m] += __ldcg(a.part + (long)(dm.tile0 + q) * kTilePartStride + m);
#pragma unroll
        for (int m = 0; m < 6; ++m)
          if (m < nv) {
            const double sum = warp_sum(v[m]);
            if (lane == 0) sh_red[0][m][wid] = sum;
          }
        __syncthreads();
        if (threadIdx.x == 0)
#pragma unroll
          for (int m = 0; m < 6; ++m)
            if (m < nv)
              for (int q = 0; q < NWARP; ++q) tot[m] += sh_red[0][m][q];
      }
      if (threadIdx.x == 0) {
        advance(a, k, st, tot);
        a.states[k] = st;
      }
      __syncthreads();
    }
    rbuf = 0;
    {
      double none[1] = {0};
      if (!grid_allreduce<1, kRedStride>(none, a.bsync, a.bpart, a.bpart + kRedStride * (long)C, C, c)) {
        fail_all(a, FREHD_ERR_TIMEOUT);
        return;
      }
    }
    if (*(volatile int *)&a.bsync->n_done >= a.ndom) break;
  }
}

// ---------------------------------------------------------------- host side

namespace {

// Looked up once; the initialisation of a function-local static is thread-safe,
// so domains may be set up on several host threads (the server's callers).
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
  }();
  return fn;
}

template <typename T, int TH = kTH>
int encode(const Grid &g, T *base, CUtensorMap *out) {
  auto fn = encode_fn();
  if (!fn) return fail(FREHD_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  const cuuint64_t dims[2] = {(cuuint64_t)g.pitch, (cuuint64_t)(g.ny + 2)};
  const cuuint64_t strides[1] = {(cuuint64_t)g.pitch * sizeof(T)};
  const cuuint32_t box[2] = {(cuuint32_t)Box<T, TH>::kBW, (cuuint32_t)Box<T, TH>::kBH};
  const cuuint32_t estr[2] = {1, 1};
  const CUtensorMapDataType dt =
      sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  CUresult e = fn(out, dt, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (e != CUDA_SUCCESS) return fail(FREHD_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)e);
  return FREHD_OK;
}

}  // namespace

int cg1_make_maps(const Grid &g, double *r0, double *r1, double *p0, double *p1, double *hx,
                  double *hy, Cg1Maps *m) {
  std::memset(m, 0, sizeof(*m));
  int rc = 0;
  rc = rc ? rc : encode(g, r0, &m->r[0]);
  rc = rc ? rc : encode(g, r1, &m->r[1]);
  rc = rc ? rc : encode(g, p0, &m->p[0]);
  rc = rc ? rc : encode(g, p1, &m->p[1]);
  rc = rc ? rc : encode(g, hx, &m->hx);
  rc = rc ? rc : encode(g, hy, &m->hy);
  return rc;
}

int cg1_make_maps_f32(const Grid &g, float *r0, float *r1, float *p0, float *p1, float *hx,
                      float *hy, Cg1Maps *m) {
  int rc = 0;
  rc = rc ? rc : encode(g, r0, &m->fr[0]);
  rc = rc ? rc : encode(g, r1, &m->fr[1]);
  rc = rc ? rc : encode(g, p0, &m->fp[0]);
  rc = rc ? rc : encode(g, p1, &m->fp[1]);
  rc = rc ? rc : encode(g, hx, &m->fhx);
  rc = rc ? rc : encode(g, hy, &m->fhy);
  // the same arrays as the mixed solve's tall inner-sweep boxes
  rc = rc ? rc : encode<float, kTallTH>(g, r0, &m->tfr[0]);
  rc = rc ? rc : encode<float, kTallTH>(g, r1, &m->tfr[1]);
  rc = rc ? rc : encode<float, kTallTH>(g, p0, &m->tfp[0]);
  rc = rc ? rc : encode<float, kTallTH>(g, p1, &m->tfp[1]);
  rc = rc ? rc : encode<float, kTallTH>(g, hx, &m->tfhx);
  rc = rc ? rc : encode<float, kTallTH>(g, hy, &m->tfhy);
  return rc;
}

// two stages, two mbarriers, and slack to align the base to 128 bytes
size_t cg1_smem_bytes() { return (size_t)kSmemStages + 2 * sizeof(unsigned long long) + 128; }

int cg1_blocks(int device, const Grid &g, int *blocks) {
  static const size_t smem = cg1_smem_bytes();
  cudaError_t e = cudaFuncSetAttribute(k_cg1<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_cg1<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return fail(FREHD_ERR_CUDA, "k_cg1 shared memory: %s", cudaGetErrorString(e));
  int nsm = 0, per = 0;
  e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_cg1<true>, kCgThreads, smem);
  if (e != cudaSuccess) return fail(FREHD_ERR_CUDA, "k_cg1 occupancy: %s", cudaGetErrorString(e));
  if (per < 1) return fail(FREHD_ERR_CUDA, "k_cg1 does not fit on an SM");
  const long ntiles = (long)((g.nx + CTX - 1) / CTX) * ((g.ny + CTY - 1) / CTY);
  const long cap = (long)nsm * per;
  *blocks = (int)(ntiles < cap ? ntiles : cap);
  return FREHD_OK;
}

int cg1_batch_capacity(int device, int *ctas) {
  static const size_t smem = cg1_smem_bytes();
  cudaError_t e = cudaFuncSetAttribute(k_cg1_batch<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_cg1_batch<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return fail(FREHD_ERR_CUDA, "k_cg1_batch shared memory: %s", cudaGetErrorString(e));
  int nsm = 0, per = 0;
  e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_cg1_batch<true>, kCgThreads, smem);
  if (e != cudaSuccess) return fail(FREHD_ERR_CUDA, "k_cg1_batch occupancy: %s", cudaGetErrorString(e));
  *ctas = nsm * (per > 0 ? per : 0);
  return *ctas > 0 ? FREHD_OK : fail(FREHD_ERR_CUDA, "k_cg1_batch does not fit on an SM");
}

int cg1_launch_batch(const View *views2, const Cg1Maps *const *maps, const int *job_start,
                     const CgJob *jobs, const CgJob *singles, int nsingles, int *taken, int nctas,
                     int any_mixed, cudaStream_t stream) {
  void *args[] = {&views2, &maps, &job_start, &jobs, &singles, &nsingles, &taken};
  void *fn = any_mixed ? (void *)k_cg1_batch<true> : (void *)k_cg1_batch<false>;
  cudaError_t e = cudaLaunchCooperativeKernel(fn, dim3(nctas), dim3(kCgThreads), args,
                                              cg1_smem_bytes(), stream);
  if (e != cudaSuccess) return fail(FREHD_ERR_CUDA, "k_cg1_batch launch: %s", cudaGetErrorString(e));
  return FREHD_OK;
}

int cg1_launch(const View &w, const Cg1Maps *m_dev, int blocks, int x0_surface, int eliminate,
               cudaStream_t stream) {
  View wv = w;
  const Cg1Maps *mp = m_dev;
  int x0 = x0_surface, el = eliminate;
  void *args[] = {&wv, &mp, &x0, &el};
  void *fn = w.p.mixed ? (void *)k_cg1<true> : (void *)k_cg1<false>;
  cudaError_t e = cudaLaunchCooperativeKernel(fn, dim3(blocks), dim3(kCgThreads), args,
                                              cg1_smem_bytes(), stream);
  if (e != cudaSuccess) return fail(FREHD_ERR_CUDA, "k_cg1 launch: %s", cudaGetErrorString(e));
  return FREHD_OK;
}

int cg1_tiles_capacity(int device, int *ctas) {
  static const size_t smem = cg1_smem_bytes();
  cudaError_t e = cudaFuncSetAttribute(k_cg1_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return fail(FREHD_ERR_CUDA, "k_cg1_tiles shared memory: %s", cudaGetErrorString(e));
  int nsm = 0, per = 0;
  e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_cg1_tiles, kCgThreads, smem);
  if (e != cudaSuccess) return fail(FREHD_ERR_CUDA, "k_cg1_tiles occupancy: %s", cudaGetErrorString(e));
  *ctas = nsm * (per > 0 ? per : 0);
  return *ctas > 0 ? FREHD_OK : fail(FREHD_ERR_CUDA, "k_cg1_tiles does not fit on an SM");
}

int cg1_launch_tiles(const View *views2, const Cg1Maps *const *maps, const BDom *doms,
                     BState *states, const BTile *tiles, int ndom, int ntiles, double *part,
                     Scratch *bsync, double *bpart, int nctas, cudaStream_t stream) {
  TilesArgs a{views2, maps, doms, states, tiles, ndom, ntiles, part, bsync, bpart};
  void *args[] = {&a};
  cudaError_t e = cudaLaunchCooperativeKernel((void *)k_cg1_tiles, dim3(nctas), dim3(kCgThreads), args,
                                              cg1_smem_bytes(), stream);
  if (e != cudaSuccess) return fail(FREHD_ERR_CUDA, "k_cg1_tiles launch: %s", cudaGetErrorString(e));
  return FREHD_OK;
}

}  // namespace frehd

// Persistent Jacobi-preconditioned CG for the 5-point free-surface system.
//
// The reference assembles a laspack QMatrix every step and calls CGIter with an
// SSOR preconditioner from x = 0 (nsfunctions.c:927-1017, itersolv.c:355-456).
// Here the system stays matrix-free in the padded layout written by k_explicit:
// one face coefficient per east face (Gx) and north face (Gy) and the row
// diagonal Ct.  Rows the reference decouples -- tidal rows (Ct = 1) and closed
// dry cells (Ct = dx*dy) -- carry a negative Ct.  The reference runs CG on the
// non-symmetric full matrix; both stop when ||r||_2 < eps*||b||_2 (rtc.c:53)
// with ||b|| taken over the full right-hand side.
//
// A decoupled row has no off-diagonal entries, so inside the reference's CG it
// is a lone eigen-component (lambda = 1 after Jacobi/SSOR scaling) and ends at
// x = (b/Ct)(1 - P(1)), P the CG residual polynomial: within the tolerance of
// b/Ct but on a side the CG picks.  That side decides later branches (a closed
// dry cell with x a hair above its bed triggers limiterCFL's velocity removal,
// nsfunctions.c:461-476).  So decoupled rows are iterated here too, as lambda = 1
// components with their own residual.  Their neighbours' rows keep the coupling
// to them, as in the reference's assembled matrix, which is then non-symmetric
// (FREHD_DECOUPLED_AS_ASSEMBLED, default: the neighbours see the decoupled
// row's current iterate, exactly as laspack iterates it); or the couplings are
// moved into the right-hand side at the exact value b/|Ct|
// (FREHD_DECOUPLED_ELIMINATED: the iterated system is symmetric).
//
// One cooperative launch runs the whole solve.  Each block owns a fixed list of
// 128 x 16 cell tiles for the whole solve.  Per iteration:
//   phase 1  the block loads r, p_old and Ct of a tile plus a one-cell halo into
//            shared memory (L2-coherent loads: other blocks wrote them), forms
//            p = r/|Ct| + beta p_old there once, writes its own p and q = A p
//   phase 2  x += alpha p, r -= alpha q, partial (r, M^-1 r) and ||r||^2
// Each phase ends in grid_allreduce: blocks publish partial sums, the last block
// to arrive sums them in a fixed order and releases the others, which then read
// the totals -- one barrier per reduction, identical totals in every block,
// bit-reproducible runs.  Waits are bounded (kBarrierTimeoutNs); a timeout
// records FREHD_ERR_TIMEOUT and every block leaves.
#include <cmath>

#include "cg_common.cuh"
#include "domain.cuh"
#include "kernels.cuh"

namespace frehd {

__global__ void __launch_bounds__(kCgThreads, 1) k_cg(View w, int x0_surface, int eliminate) {
  Scratch *sc = w.sc;
  if (*(volatile int *)&sc->status != FREHD_OK) return;
  if (test_skip_barrier(sc, blockIdx.x)) {  // a lone CTA has no partner whose wait could run out
    if (gridDim.x == 1 && threadIdx.x == 0) set_status(sc, FREHD_ERR_TIMEOUT);
    return;
  }
  const Grid g = w.gr;
  const Params &p = w.p;
  const int nx = g.nx, ny = g.ny;
  const long pitch = g.pitch;
  const unsigned nb = gridDim.x;
  TileIt ti;
  ti.ntx = (nx + CTX - 1) / CTX;
  ti.nty = (ny + CTY - 1) / CTY;
  ti.ntiles = ti.ntx * ti.nty;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  double *partials = w.partials, *totals = w.partials + 4 * (long)nb;
  const double *Ct = w.Ct, *Gx = w.Gx, *Gy = w.Gy;
  __shared__ double s_p[HY][HX], s_c[HY][HX];

  // A solve of the assembled (non-symmetric) matrix can stall: ||r|| stops
  // falling above eps*||b|| and laspack's CGIter runs on to maxIter.  When ||r||
  // has not halved for kStallIters iterations the solve starts again in the
  // eliminated (symmetric positive definite) form, and the step reports it.
  int it = 0, it_all = 0, fallback = 0, noconv = 0;
  double rr = 0.0, bnorm = 0.0;
  for (int attempt = 0;; ++attempt) {
    const int elim = eliminate | (attempt > 0);
    // ---- setup 1: x0 and the p buffers
    for (int tile = blockIdx.x; tile < ti.ntiles; tile += nb) {
      int i0, j0;
      tile_origin(ti, tile, &i0, &j0);
      const int j = j0 + ty;
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        const int i = i0 + c * 32 + tx;
        if (i < nx && j < ny) {
          const long k = g.at(i, j);
          w.x[k] = x0_surface ? w.surf_cur[k] : 0.0;
          w.p0[k] = 0.0;
          w.p1[k] = 0.0;
        }
      }
    }
    {
      double none[1] = {0};
      if (!grid_allreduce<1>(none, sc, partials, totals, nb)) return;
    }

    // ---- setup 2: r = b - A x (eliminated: decoupled neighbours at their exact b/|Ct|)
    double acc[3] = {0, 0, 0};
    for (int tile = blockIdx.x; tile < ti.ntiles; tile += nb) {
      int i0, j0;
      tile_origin(ti, tile, &i0, &j0);
      const int j = j0 + ty;
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        const int i = i0 + c * 32 + tx;
        if (i < nx && j < ny) {
          const long k = g.at(i, j);
          const double ct = Ct[k], bk = w.b[k];
          auto xv = [&](long kk) -> double {
            const double cc = Ct[kk];
            return (elim && cc < 0) ? w.b[kk] / (-cc) : ld(w.x, kk);
          };
          double r;
          if (ct > 0) {
            const double ax = ct * ld(w.x, k) - (Gx[k] * xv(k + 1) + Gx[k - 1] * xv(k - 1) +
                                                 Gy[k] * xv(k + pitch) + Gy[k - pitch] * xv(k - pitch));
            r = bk - ax;
          } else {
            r = bk - (-ct) * ld(w.x, k);
          }
          acc[0] += r * (r / fabs(ct));
          acc[1] += r * r;
          acc[2] += bk * bk;
          w.r[k] = r;
        }
      }
    }
    if (!grid_allreduce<3>(acc, sc, partials, totals, nb)) return;
    double rho = acc[0], rho_old = 1.0;
    rr = acc[1];
    bnorm = sqrt(acc[2]);
    double best = rr;
    int best_it = 0, cur = 0;
    bool stalled = false;
    it = 0;
    auto converged = [&](double rr_) {
      const double rn = sqrt(rr_);
      return rn < p.eps * bnorm || (bnorm == 0.0 && 1.0 + rn == 1.0);
    };
    while (!converged(rr) && it < p.maxIter) {
      ++it;
      const double beta = it == 1 ? 0.0 : rho / rho_old;
      const double *pold = cur ? w.p1 : w.p0;
      double *pnew = cur ? w.p0 : w.p1;
      // ---- phase 1: p = M^-1 r + beta p_old on tile + halo, q = A p
      double pq[1] = {0};
      for (int tile = blockIdx.x; tile < ti.ntiles; tile += nb) {
        int i0, j0;
        tile_origin(ti, tile, &i0, &j0);
        __syncthreads();  // the previous tile's shared data is consumed
        for (int e = threadIdx.x; e < HX * HY; e += kCgThreads) {
          const int ey = e / HX, ex = e - ey * HX;
          const int i = i0 - 1 + ex, j = j0 - 1 + ey;
          double pv = 0.0, cv = -1.0;
          if (i <= nx && j <= ny) {
            const long k = g.at(i, j);
            cv = Ct[k];
            const double rv = ld(w.r, k), po = ld(pold, k);
            pv = rv / fabs(cv) + beta * po;
          }
          s_p[ey][ex] = pv;
          s_c[ey][ex] = cv;
        }
        __syncthreads();
        const int j = j0 + ty, ly = ty + 1;
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          const int lx = c * 32 + tx + 1;
          const int i = i0 + lx - 1;
          if (i < nx && j < ny) {
            const long k = g.at(i, j);
            const double ct = s_c[ly][lx], pc = s_p[ly][lx];
            // eliminated: decoupled neighbours contribute nothing (their coupling is in b)
            auto nb_p = [&](int yy, int xx) -> double {
              return (elim && s_c[yy][xx] < 0) ? 0.0 : s_p[yy][xx];
            };
            double qv;
            if (ct > 0)
              qv = ct * pc - (Gx[k] * nb_p(ly, lx + 1) + Gx[k - 1] * nb_p(ly, lx - 1) +
                              Gy[k] * nb_p(ly + 1, lx) + Gy[k - pitch] * nb_p(ly - 1, lx));
            else
              qv = (-ct) * pc;  // decoupled row: lambda = 1 component
            pnew[k] = pc;
            w.q[k] = qv;
            pq[0] += pc * qv;
          }
        }
      }
      if (!grid_allreduce<1>(pq, sc, partials, totals, nb)) return;
      const double alpha = rho / pq[0];
      // ---- phase 2: x, r update and the preconditioned residual norms
      double a2[2] = {0, 0};
      for (int tile = blockIdx.x; tile < ti.ntiles; tile += nb) {
        int i0, j0;
        tile_origin(ti, tile, &i0, &j0);
        const int j = j0 + ty;
        double xs[CPT], rs[CPT], ps[CPT], qs[CPT], cs[CPT];
        long ks[CPT];
        bool ok[CPT];
#pragma unroll
        for (int c = 0; c < CPT; ++c) {  // issue every load of the tile row first
          const int i = i0 + c * 32 + tx;
          ok[c] = i < nx && j < ny;
          ks[c] = ok[c] ? g.at(i, j) : g.at(0, 0);
          cs[c] = Ct[ks[c]];
          ps[c] = ld(pnew, ks[c]);
          qs[c] = ld(w.q, ks[c]);
          rs[c] = ld(w.r, ks[c]);
          xs[c] = ld(w.x, ks[c]);
        }
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          if (!ok[c]) continue;
          const double rv = rs[c] - alpha * qs[c];
          w.x[ks[c]] = xs[c] + alpha * ps[c];
          w.r[ks[c]] = rv;
          a2[0] += rv * (rv / fabs(cs[c]));
          a2[1] += rv * rv;
        }
      }
      if (!grid_allreduce<2>(a2, sc, partials, totals, nb)) return;
      rho_old = rho;
      rho = a2[0];
      rr = a2[1];
      cur ^= 1;
      // identical totals in every block: every block takes the same decision
      if (rr < 0.25 * best) {
        best = rr;
        best_it = it;
      } else if (!elim && it - best_it >= kStallIters) {
        stalled = true;
        break;
      }
    }
    it_all += it;
    // maxIter reached first: laspack's CGIter stops there silently; the step reports it
    noconv = !stalled && !converged(rr);
    if (!stalled) break;
    fallback = 1;
  }  // attempt
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->cg_iters = it_all;
    sc->cg_fallback = fallback;
    sc->cg_noconv = noconv;
    sc->cg_rr = rr;
    sc->cg_bb = bnorm * bnorm;
  }
}

}  // namespace frehd

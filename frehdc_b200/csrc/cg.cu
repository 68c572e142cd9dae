// Persistent Jacobi-preconditioned CG for the 5-point free-surface system.
//
// The reference assembles a laspack QMatrix every step and calls CGIter with an
// SSOR preconditioner from x = 0 (nsfunctions.c:927-1017, itersolv.c:355-456).
// Here the system stays matrix-free in the padded layout written by k_explicit:
// one face coefficient per east face (Gx) and north face (Gy) and the row
// diagonal Ct.  Rows the reference decouples -- tidal rows (Ct = 1) and closed
// dry cells (Ct = dx*dy) -- carry a negative Ct.  Their unknowns are known
// exactly (x = b/|Ct|) and are eliminated: their couplings move to the
// right-hand side of the neighbouring rows, which leaves a symmetric positive
// definite system over the remaining rows.  The reference runs CG on the
// non-symmetric full matrix; both stop when ||r||_2 < eps*||b||_2 (rtc.c:53)
// with ||b|| taken over the full right-hand side, so both solve the same system
// to the same residual tolerance.
//
// One cooperative launch runs the whole solve: all blocks are co-resident and
// meet at a grid barrier twice per iteration.  The barrier waits are bounded
// (kBarrierTimeoutNs); a timeout records FREHD_ERR_TIMEOUT and every block
// leaves.  Dot products are reduced in a fixed order (per-block partials, then
// every block sums all partials in the same order), so every block computes the
// same alpha/beta and runs are bit-reproducible.
#include <cmath>

#include "domain.cuh"
#include "kernels.cuh"

namespace frehd {

constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;  // 2 s per wait

__device__ __forceinline__ unsigned long long gtimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ double ld(const double *a, long k) { return __ldcg(a + k); }

__device__ bool grid_barrier(Scratch *sc, unsigned nblocks) {
  __shared__ int s_ok;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned *gen = &sc->bar_gen;
    const unsigned my = *gen;
    __threadfence();
    const unsigned arrived = atomicAdd(&sc->bar_count, 1u);
    int ok = 1;
    if (arrived == nblocks - 1) {
      atomicExch(&sc->bar_count, 0u);
      __threadfence();
      atomicAdd(&sc->bar_gen, 1u);
    } else {
      const unsigned long long t0 = gtimer_ns();
      while (*gen == my) {
        if (gtimer_ns() - t0 > kBarrierTimeoutNs) {
          set_status(sc, FREHD_ERR_TIMEOUT);
          ok = 0;
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
    if (*(volatile int *)&sc->status == FREHD_ERR_TIMEOUT) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Write this block's partial sums of NV values (fixed reduction order).
template <int NV>
__device__ void block_partials(double (&v)[NV], double *out) {
  __shared__ double sh[NV][kCgThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int m = 0; m < NV; ++m) {
    const double s = warp_sum(v[m]);
    if (lane == 0) sh[m][wid] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int m = 0; m < NV; ++m) {
      double a = 0;
      for (int q = 0; q < kCgThreads / 32; ++q) a += sh[m][q];
      out[m] = a;
    }
  }
}

// Sum of all blocks' partials, identical in every block.
template <int NV>
__device__ void grid_total(const double *partials, unsigned nblocks, double (&tot)[NV]) {
  __shared__ double sh[NV][kCgThreads / 32];
  double a[NV];
#pragma unroll
  for (int m = 0; m < NV; ++m) a[m] = 0;
  for (unsigned q = threadIdx.x; q < nblocks; q += blockDim.x) {
#pragma unroll
    for (int m = 0; m < NV; ++m) a[m] += ld(partials, (long)q * 4 + m);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int m = 0; m < NV; ++m) {
    const double s = warp_sum(a[m]);
    if (lane == 0) sh[m][wid] = s;
  }
  __syncthreads();
#pragma unroll
  for (int m = 0; m < NV; ++m) {
    double t = 0;
    for (int q = 0; q < kCgThreads / 32; ++q) t += sh[m][q];
    tot[m] = t;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kCgThreads) k_cg(View w, int x0_surface) {
  Scratch *sc = w.sc;
  if (*(volatile int *)&sc->status != FREHD_OK) return;
  const Grid g = w.gr;
  const Params &p = w.p;
  const unsigned nx = g.nx, N = (unsigned)g.nx * g.ny;
  const unsigned nb = gridDim.x;
  const unsigned gtid = blockIdx.x * blockDim.x + threadIdx.x, gs = nb * blockDim.x;
  // two partial buffers, alternating per reduction, so a fast block never
  // overwrites partials a slow block is still summing
  double *part[2] = {w.partials, w.partials + 4 * (long)nb};
  int pb = 0;
  const double *Ct = w.Ct, *Gx = w.Gx, *Gy = w.Gy;

  for (unsigned t = gtid; t < N; t += gs) {
    const int i = t % nx, j = t / nx;
    const long k = g.at(i, j);
    const double ct = Ct[k];
    w.x[k] = ct < 0 ? w.b[k] / (-ct) : (x0_surface ? w.surf_cur[k] : 0.0);
    w.p0[k] = 0.0;
    w.p1[k] = 0.0;
  }
  if (!grid_barrier(sc, nb)) return;

  double acc[3] = {0, 0, 0};
  for (unsigned t = gtid; t < N; t += gs) {
    const int i = t % nx, j = t / nx;
    const long k = g.at(i, j), kE = k + 1, kW = k - 1, kN = k + g.pitch, kS = k - g.pitch;
    const double ct = Ct[k], bk = w.b[k];
    double r = 0;
    if (ct > 0) {
      const double ax = ct * ld(w.x, k) -
                        (Gx[k] * ld(w.x, kE) + Gx[kW] * ld(w.x, kW) + Gy[k] * ld(w.x, kN) +
                         Gy[kS] * ld(w.x, kS));
      r = bk - ax;
      acc[0] += r * (r / ct);
      acc[1] += r * r;
    }
    w.r[k] = r;
    acc[2] += bk * bk;
  }
  block_partials<3>(acc, part[pb] + 4 * blockIdx.x);
  if (!grid_barrier(sc, nb)) return;
  double tot3[3];
  grid_total<3>(part[pb], nb, tot3);
  pb ^= 1;
  double rho = tot3[0], rr = tot3[1], rho_old = 1.0;
  const double bnorm = sqrt(tot3[2]);
  int it = 0, cur = 0;
  auto converged = [&](double rr_) {
    const double rn = sqrt(rr_);
    return rn < p.eps * bnorm || (bnorm == 0.0 && 1.0 + rn == 1.0);
  };
  while (!converged(rr) && it < p.maxIter) {
    ++it;
    const double beta = it == 1 ? 0.0 : rho / rho_old;
    const double *pold = cur ? w.p1 : w.p0;
    double *pnew = cur ? w.p0 : w.p1;
    // p = M^-1 r + beta p (neighbours recomputed, no extra barrier); q = A p
    double pq = 0;
    for (unsigned t = gtid; t < N; t += gs) {
      const int i = t % nx, j = t / nx;
      const long k = g.at(i, j);
      const double ct = Ct[k];
      if (ct < 0) {
        pnew[k] = 0.0;
        w.q[k] = 0.0;
        continue;
      }
      const long kE = k + 1, kW = k - 1, kN = k + g.pitch, kS = k - g.pitch;
      auto pn = [&](long kk) -> double {
        const double c = Ct[kk];
        return c < 0 ? 0.0 : ld(w.r, kk) / c + beta * ld(pold, kk);
      };
      const double pc = ld(w.r, k) / ct + beta * ld(pold, k);
      const double qv = ct * pc - (Gx[k] * pn(kE) + Gx[kW] * pn(kW) + Gy[k] * pn(kN) + Gy[kS] * pn(kS));
      pnew[k] = pc;
      w.q[k] = qv;
      pq += pc * qv;
    }
    double a1[1] = {pq};
    block_partials<1>(a1, part[pb] + 4 * blockIdx.x);
    if (!grid_barrier(sc, nb)) return;
    double t1[1];
    grid_total<1>(part[pb], nb, t1);
    pb ^= 1;
    const double alpha = rho / t1[0];
    double a2[2] = {0, 0};
    for (unsigned t = gtid; t < N; t += gs) {
      const int i = t % nx, j = t / nx;
      const long k = g.at(i, j);
      const double ct = Ct[k];
      if (ct < 0) continue;
      const double pc = ld(pnew, k), qv = ld(w.q, k);
      const double rv = ld(w.r, k) - alpha * qv;
      w.x[k] = ld(w.x, k) + alpha * pc;
      w.r[k] = rv;
      a2[0] += rv * (rv / ct);
      a2[1] += rv * rv;
    }
    block_partials<2>(a2, part[pb] + 4 * blockIdx.x);
    if (!grid_barrier(sc, nb)) return;
    double t2[2];
    grid_total<2>(part[pb], nb, t2);
    pb ^= 1;
    rho_old = rho;
    rho = t2[0];
    rr = t2[1];
    cur ^= 1;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->cg_iters = it;
    sc->cg_rr = rr;
    sc->cg_bb = bnorm * bnorm;
  }
}

}  // namespace frehd

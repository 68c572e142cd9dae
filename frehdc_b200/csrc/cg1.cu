// Single-sweep Jacobi-PCG for the 5-point free-surface system (default solver).
//
// Same system, preconditioner, start and stopping rule as k_cg (cg.cu): Jacobi
// M = diag|Ct|, x0 = 0 (or the surface), stop when ||r||_2 < eps*||b||_2
// checked before each iteration (rtc.c:53, itersolv.c:355-456), decoupled rows
// iterated as lambda = 1 components whose couplings sit in b.  What changes is
// the schedule: the Chronopoulos-Gear form of CG (Chronopoulos & Gear, "s-step
// iterative methods for symmetric linear systems", J. Comput. Appl. Math. 25,
// 1989) takes alpha_i from the previous iteration's two dot products,
//   beta_i  = gamma_i / gamma_{i-1}
//   alpha_i = gamma_i / (delta_i - beta_i * gamma_i / alpha_{i-1}),
//   gamma_i = (r_i, u_i), delta_i = (A u_i, u_i), u_i = M^-1 r_i,
// so one sweep over the grid does a whole iteration and ends in ONE grid
// reduction of (gamma, delta, ||r||^2) instead of two.  A p_i is computed
// explicitly from p_i (not by a recurrence), so r follows the same update as
// in standard CG.
//
// One sweep per tile of 128 x 16 cells, with a two-cell halo loaded by TMA:
//   A  p_i = r_i/|Ct| + beta p_{i-1}            tile + 2 halo (in place)
//   B  s = A p_i; r_{i+1} = r_i - alpha s;
//      u_{i+1} = r_{i+1}/|Ct|                   tile + 1 halo (in place)
//   C  w = A u_{i+1}; x += alpha p_i            tile
// DRAM traffic per cell and iteration: read r, p, Ct, Gx, Gy, x; write r, p, x
// = 72 bytes.  r and p ping-pong between two buffers (neighbouring blocks read
// the old halo while a block writes its new tile); x is updated in place.
// Boxes of r, p, Ct, Gx, Gy (132 x 20 doubles each) are double-buffered in
// shared memory behind one mbarrier per stage: the next tile's loads are in
// flight while the current tile computes.  All waits are bounded.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstring>

#include "cg1.h"
#include "cg_common.cuh"
#include "frehd_internal.h"

namespace frehd {

namespace {

constexpr int kTW = CTX, kTH = CTY;              // owned cells of a tile (128 x 16)
constexpr int kBW = kTW + 4, kBH = kTH + 4;      // tile + two-cell halo: 132 x 20
constexpr int kBox = kBW * kBH;                  // doubles per array per stage
constexpr int kIW = kBW - 2, kIH = kBH - 2;      // tile + one-cell halo: 130 x 18
constexpr int kNArr = 5;                         // r, p, Ct, Gx, Gy
constexpr unsigned kArrBytes = kBox * 8u;        // 21120, a multiple of 128
constexpr unsigned kStageBytes = kNArr * kArrBytes;
static_assert(kArrBytes % 128 == 0, "TMA destinations must stay 128-byte aligned");
static_assert((kBW * 8) % 16 == 0, "TMA box rows must be a multiple of 16 bytes");
static_assert(kTH == kCgThreads / 32, "one warp per tile row in pass C");

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_test(unsigned long long *bar, unsigned parity) {
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
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity,
                                          unsigned long long limit_ns) {
  if (mbar_test(bar, parity)) return true;
  const unsigned long long t0 = gtimer_ns();
  while (!mbar_test(bar, parity)) {
    if (gtimer_ns() - t0 > limit_ns) return false;
  }
  return true;
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map,
                                            unsigned long long *bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// Shared-memory arrays of one stage.
struct Stage {
  double *R, *P, *C, *GX, *GY;
  __device__ Stage(unsigned char *base) {
    R = reinterpret_cast<double *>(base);
    P = R + kBox;
    C = P + kBox;
    GX = C + kBox;
    GY = GX + kBox;
  }
};

// Issue the five box loads of tile `tile` into stage `st` (one thread).
__device__ __forceinline__ void issue_tile(const Cg1Maps *m, int cur, const TileIt &ti, int tile,
                                           unsigned char *stage_base, unsigned long long *bar) {
  int i0, j0;
  tile_origin(ti, tile, &i0, &j0);
  // box origin: cell (i0-2, j0-2) = padded column i0+2 (even: 16-byte aligned), row j0-1
  const int x = i0 - 2 + kXOff, y = j0 - 2 + 1;
  Stage s(stage_base);
  // generic-proxy writes to this stage (the in-place passes) come before the TMA writes
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  mbar_expect_tx(bar, kStageBytes);
  tma_load_2d(s.R, &m->r[cur], bar, x, y);
  tma_load_2d(s.P, &m->p[cur], bar, x, y);
  tma_load_2d(s.C, &m->ct, bar, x, y);
  tma_load_2d(s.GX, &m->gx, bar, x, y);
  tma_load_2d(s.GY, &m->gy, bar, x, y);
}

}  // namespace

__global__ void __launch_bounds__(kCgThreads, 1)
    k_cg1(View w, const Cg1Maps *__restrict__ m, int x0_surface) {
  Scratch *sc = w.sc;
  if (*(volatile int *)&sc->status != FREHD_OK) return;
  // The dynamic region starts after the static shared data (this kernel's and
  // grid_allreduce's), which only guarantees 16-byte alignment: round the base
  // up to 128 bytes at run time (the launch requests 128 bytes of slack).
  extern __shared__ unsigned char smem_raw[];
  unsigned char *smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  unsigned long long *bars = reinterpret_cast<unsigned long long *>(smem + 2 * kStageBytes);
  __shared__ int s_ok;
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

  // TMA destinations 128-byte aligned, mbarriers 8-byte aligned, tensor maps
  // 64-byte aligned: refuse (every block alike) otherwise
  if ((smem_u32(smem) & 127u) || (smem_u32(bars) & 7u) ||
      (reinterpret_cast<unsigned long long>(m) & 63ull)) {
    if (threadIdx.x == 0) set_status(sc, FREHD_ERR_CUDA);
    return;
  }
  if (threadIdx.x == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    // the maps were written to global memory by a host copy: make them visible to the TMA unit
    const CUtensorMap *maps = &m->r[0];
    for (int q = 0; q < 7; ++q)
      asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(maps + q) : "memory");
  }
  __syncthreads();

  // ---- setup 1: x0 and p_{-1} = 0
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
      }
    }
  }
  {
    double none[1] = {0};
    if (!grid_allreduce<1>(none, sc, partials, totals, nb)) return;
  }

  // ---- setup 2: r0 = b - A x0 (decoupled neighbours at their exact b/|Ct|)
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
          return cc < 0 ? w.b[kk] / (-cc) : ld(w.x, kk);
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
  double gamma = acc[0], rr = acc[1];
  const double bnorm = sqrt(acc[2]);

  // ---- setup 3: delta0 = (A u0, u0), u0 = r0/|Ct| (plain halo loads into stage 0)
  double delta;
  {
    double d0[1] = {0};
    Stage s(smem);
    for (int tile = blockIdx.x; tile < ti.ntiles; tile += nb) {
      int i0, j0;
      tile_origin(ti, tile, &i0, &j0);
      __syncthreads();
      for (int e = threadIdx.x; e < kIW * kIH; e += kCgThreads) {
        const int ly = 1 + e / kIW, lx = 1 + e % kIW;
        const int i = i0 - 2 + lx, j = j0 - 2 + ly;
        double u = 0.0, cv = -1.0;
        if ((unsigned)i < (unsigned)nx && (unsigned)j < (unsigned)ny) {
          const long k = g.at(i, j);
          cv = Ct[k];
          u = ld(w.r, k) / fabs(cv);
        }
        s.R[ly * kBW + lx] = u;
        s.C[ly * kBW + lx] = cv;
      }
      __syncthreads();
      const int j = j0 + ty;
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        const int i = i0 + c * 32 + tx;
        if (i < nx && j < ny) {
          const long k = g.at(i, j);
          const int cc = (ty + 2) * kBW + c * 32 + tx + 2;
          const double ct = s.C[cc], u = s.R[cc];
          auto vis = [&](int q) -> double { return s.C[q] > 0 ? s.R[q] : 0.0; };
          const double au = ct > 0 ? ct * u - (Gx[k] * vis(cc + 1) + Gx[k - 1] * vis(cc - 1) +
                                               Gy[k] * vis(cc + kBW) + Gy[k - pitch] * vis(cc - kBW))
                                   : (-ct) * u;
          d0[0] += au * u;
        }
      }
    }
    __syncthreads();
    if (!grid_allreduce<1>(d0, sc, partials, totals, nb)) return;
    delta = d0[0];
  }

  auto converged = [&](double rr_) {
    const double rn = sqrt(rr_);
    return rn < p.eps * bnorm || (bnorm == 0.0 && 1.0 + rn == 1.0);
  };
  double gamma_old = 1.0, alpha_old = 1.0;
  int it = 0, cur = 0;
  unsigned seq = 0;  // tiles consumed by this block: stage = seq & 1, phase parity = (seq >> 1) & 1
  while (!converged(rr) && it < p.maxIter) {
    const double beta = it == 0 ? 0.0 : gamma / gamma_old;
    const double alpha = it == 0 ? gamma / delta : gamma / (delta - beta * gamma / alpha_old);
    ++it;
    double *rn_out = cur ? w.r : w.q, *pn_out = cur ? w.p0 : w.p1;
    double red[3] = {0, 0, 0};  // gamma, delta, rr of the new residual
    // generic writes of the previous sweep (all blocks) come before this sweep's TMA reads
    if (threadIdx.x == 0) {
      asm volatile("fence.proxy.async.global;" ::: "memory");
      issue_tile(m, cur, ti, blockIdx.x, smem + (seq & 1) * kStageBytes, &bars[seq & 1]);
    }
    for (int tile = blockIdx.x; tile < ti.ntiles; tile += nb, ++seq) {
      const int st = seq & 1;
      const int next = tile + (int)nb;
      if (threadIdx.x == 0 && next < ti.ntiles)
        issue_tile(m, cur, ti, next, smem + (st ^ 1) * kStageBytes, &bars[st ^ 1]);
      int i0, j0;
      tile_origin(ti, tile, &i0, &j0);
      // x of the owned cells: in flight while the boxes arrive
      double xs[CPT];
      {
        const int j = j0 + ty;
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          const int i = i0 + c * 32 + tx;
          xs[c] = (i < nx && j < ny) ? w.x[g.at(i, j)] : 0.0;
        }
      }
      if (threadIdx.x == 0) s_ok = mbar_wait(&bars[st], (seq >> 1) & 1, kBarrierTimeoutNs);
      __syncthreads();
      if (!s_ok) {
        // the other stage may hold a load issued for the next tile: let it land
        if (threadIdx.x == 0) {
          set_status(sc, FREHD_ERR_TIMEOUT);
          if (next < ti.ntiles) mbar_wait(&bars[st ^ 1], ((seq + 1) >> 1) & 1, kBarrierTimeoutNs);
        }
        return;
      }
      mbar_wait(&bars[st], (seq >> 1) & 1, kBarrierTimeoutNs);  // completed: acquire in every thread
      Stage s(smem + st * kStageBytes);

      // pass A: p_i = r_i/|Ct| + beta p_{i-1} on tile + 2 halo; outside the domain p = r = 0
      for (int e = threadIdx.x; e < kBox; e += kCgThreads) {
        const int ly = e / kBW, lx = e - ly * kBW;
        const int i = i0 - 2 + lx, j = j0 - 2 + ly;
        if ((unsigned)i < (unsigned)nx && (unsigned)j < (unsigned)ny) {
          s.P[e] = s.R[e] / fabs(s.C[e]) + beta * s.P[e];
        } else {
          s.P[e] = 0.0;
          s.R[e] = 0.0;
          s.C[e] = -1.0;
        }
      }
      __syncthreads();

      // pass B: s = A p_i, r_{i+1} = r_i - alpha s, u_{i+1} = r_{i+1}/|Ct| on tile + 1 halo
      for (int e = threadIdx.x; e < kIW * kIH; e += kCgThreads) {
        const int ly = 1 + e / kIW, lx = 1 + e % kIW;
        const int q = ly * kBW + lx;
        const double ct = s.C[q], pc = s.P[q];
        auto vis = [&](int qq) -> double { return s.C[qq] > 0 ? s.P[qq] : 0.0; };
        const double ap = ct > 0 ? ct * pc - (s.GX[q] * vis(q + 1) + s.GX[q - 1] * vis(q - 1) +
                                              s.GY[q] * vis(q + kBW) + s.GY[q - kBW] * vis(q - kBW))
                                 : (-ct) * pc;
        const double rnew = s.R[q] - alpha * ap;
        const double unew = rnew / fabs(ct);
        s.R[q] = unew;
        const int li = lx - 2, lj = ly - 2;
        if ((unsigned)li < (unsigned)kTW && (unsigned)lj < (unsigned)kTH) {
          const int i = i0 + li, j = j0 + lj;
          if (i < nx && j < ny) {
            rn_out[g.at(i, j)] = rnew;
            red[0] += rnew * unew;
            red[2] += rnew * rnew;
          }
        }
      }
      __syncthreads();

      // pass C: w = A u_{i+1}, delta partial; x_{i+1} = x_i + alpha p_i; store p_i
      {
        const int j = j0 + ty;
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          const int i = i0 + c * 32 + tx;
          if (i < nx && j < ny) {
            const int q = (ty + 2) * kBW + c * 32 + tx + 2;
            const double ct = s.C[q], u = s.R[q];
            auto vis = [&](int qq) -> double { return s.C[qq] > 0 ? s.R[qq] : 0.0; };
            const double au = ct > 0 ? ct * u - (s.GX[q] * vis(q + 1) + s.GX[q - 1] * vis(q - 1) +
                                                 s.GY[q] * vis(q + kBW) + s.GY[q - kBW] * vis(q - kBW))
                                     : (-ct) * u;
            red[1] += au * u;
            const long k = g.at(i, j);
            const double pc = s.P[q];
            w.x[k] = xs[c] + alpha * pc;
            pn_out[k] = pc;
          }
        }
      }
      __syncthreads();  // stage st is free for the tile after next
    }
    // this thread's global writes before the next sweep's TMA reads (other blocks)
    asm volatile("fence.proxy.async.global;" ::: "memory");
    if (!grid_allreduce<3>(red, sc, partials, totals, nb)) return;
    gamma_old = gamma;
    alpha_old = alpha;
    gamma = red[0];
    delta = red[1];
    rr = red[2];
    cur ^= 1;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->cg_iters = it;
    sc->cg_rr = rr;
    sc->cg_bb = bnorm * bnorm;
  }
}

// ---------------------------------------------------------------- host side

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }
  return fn;
}

int encode(const Grid &g, double *base, CUtensorMap *out) {
  auto fn = encode_fn();
  if (!fn) return fail(FREHD_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  const cuuint64_t dims[2] = {(cuuint64_t)g.pitch, (cuuint64_t)(g.ny + 2)};
  const cuuint64_t strides[1] = {(cuuint64_t)g.pitch * sizeof(double)};
  const cuuint32_t box[2] = {(cuuint32_t)kBW, (cuuint32_t)kBH};
  const cuuint32_t estr[2] = {1, 1};
  CUresult e = fn(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, base, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (e != CUDA_SUCCESS) return fail(FREHD_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)e);
  return FREHD_OK;
}

}  // namespace

int cg1_make_maps(const Grid &g, double *r0, double *r1, double *p0, double *p1, double *ct,
                  double *gx, double *gy, Cg1Maps *m) {
  std::memset(m, 0, sizeof(*m));
  int rc = 0;
  rc = rc ? rc : encode(g, r0, &m->r[0]);
  rc = rc ? rc : encode(g, r1, &m->r[1]);
  rc = rc ? rc : encode(g, p0, &m->p[0]);
  rc = rc ? rc : encode(g, p1, &m->p[1]);
  rc = rc ? rc : encode(g, ct, &m->ct);
  rc = rc ? rc : encode(g, gx, &m->gx);
  rc = rc ? rc : encode(g, gy, &m->gy);
  return rc;
}

// two stages, two mbarriers, and slack to align the base to 128 bytes
size_t cg1_smem_bytes() { return 2 * (size_t)kStageBytes + 2 * sizeof(unsigned long long) + 128; }

int cg1_blocks(int device, const Grid &g, int *blocks) {
  static const size_t smem = cg1_smem_bytes();
  cudaError_t e = cudaFuncSetAttribute(k_cg1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return fail(FREHD_ERR_CUDA, "k_cg1 shared memory: %s", cudaGetErrorString(e));
  int nsm = 0, per = 0;
  e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_cg1, kCgThreads, smem);
  if (e != cudaSuccess) return fail(FREHD_ERR_CUDA, "k_cg1 occupancy: %s", cudaGetErrorString(e));
  if (per < 1) return fail(FREHD_ERR_CUDA, "k_cg1 does not fit on an SM");
  const long ntiles = (long)((g.nx + CTX - 1) / CTX) * ((g.ny + CTY - 1) / CTY);
  const long cap = (long)nsm * per;
  *blocks = (int)(ntiles < cap ? ntiles : cap);
  return FREHD_OK;
}

int cg1_launch(const View &w, const Cg1Maps *m_dev, int blocks, int x0_surface, cudaStream_t stream) {
  View wv = w;
  const Cg1Maps *mp = m_dev;
  int x0 = x0_surface;
  void *args[] = {&wv, &mp, &x0};
  cudaError_t e = cudaLaunchCooperativeKernel((void *)k_cg1, dim3(blocks), dim3(kCgThreads), args,
                                              cg1_smem_bytes(), stream);
  if (e != cudaSuccess) return fail(FREHD_ERR_CUDA, "k_cg1 launch: %s", cudaGetErrorString(e));
  return FREHD_OK;
}

}  // namespace frehd

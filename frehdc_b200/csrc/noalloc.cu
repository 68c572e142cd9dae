// frehd_cg_solve_noalloc: the free-surface CG solve for callers that cannot
// allocate device memory.
//
// Who needs it: a host whose device memory belongs to another runtime's pool
// (the pool reserves the GPU up front, so a cudaMalloc from a library either
// fails or breaks the host's accounting), and hosts whose time loop must not
// allocate after start-up (cudaMalloc/cudaFree synchronise the device and add
// unbounded latency).  Such a caller owns every buffer it passes; the solve's
// own work vectors live in this file's static device array instead of in
// memory the library would otherwise allocate per domain.
//
// The scratch array is part of the library image: every GPU that loads the
// library holds kNoAllocScratchDoubles doubles (about 8.4 MB) until the process
// exits.  Every call shares it and it keeps the last call's contents; each call
// first clears the counters that must start at zero (stream-ordered, no host
// synchronisation).  Two calls that overlap on the GPU (different streams, or
// different host threads without ordering) use the same scratch and race.
//
// The kernel is the persistent Jacobi-PCG of cg.cu over caller-provided
// row-major arrays (no ghost ring): identical tile decomposition, arithmetic
// and fixed-order reductions.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "cg_common.cuh"
#include "frehd_internal.h"

namespace {

using namespace frehd;

constexpr long kNoAllocMaxCells = 512L * 512L;  // largest nx*ny accepted
constexpr int kNoAllocMaxBlocks = 1024;         // largest cooperative grid
constexpr long kHeaderDoubles = 32;             // Scratch (barrier, status, CG counters)
constexpr long kPartialDoubles = 4L * kNoAllocMaxBlocks + 32;
constexpr long kNoAllocScratchDoubles = kHeaderDoubles + kPartialDoubles + 4 * kNoAllocMaxCells;
static_assert(sizeof(Scratch) <= kHeaderDoubles * sizeof(double), "scratch header too small");

// The scratch: header | per-block partials + totals | r | p0 | p1 | q.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

struct NoAllocArgs {
  int nx, ny;
  const double *Ct, *Gx, *Gy, *b;
  double *x;
  double eps;
  int max_iter, x0_from_x;
  double *scratch;  // device address of g_noalloc_scratch (from cudaGetSymbolAddress)
};

__global__ void k_noalloc_reset(double *scratch) {
  Scratch *sc = reinterpret_cast<Scratch *>(scratch);
  sc->bar_count = 0;
  sc->status = FREHD_OK;
  sc->cg_iters = 0;
  sc->cg_rr = 0;
  sc->cg_bb = 0;
}

__global__ void __launch_bounds__(kCgThreads, 1) k_cg_noalloc(NoAllocArgs a) {
  Scratch *sc = reinterpret_cast<Scratch *>(a.scratch);
  const int nx = a.nx, ny = a.ny;
  const long N = (long)nx * ny;
  const unsigned nb = gridDim.x;
  double *partials = a.scratch + kHeaderDoubles, *totals = partials + 4 * (long)nb;
  double *r = a.scratch + kHeaderDoubles + kPartialDoubles;
  double *p0 = r + kNoAllocMaxCells, *p1 = p0 + kNoAllocMaxCells, *q = p1 + kNoAllocMaxCells;
  const double *Ct = a.Ct, *Gx = a.Gx, *Gy = a.Gy, *b = a.b;
  double *x = a.x;
  TileIt ti;
  ti.ntx = (nx + CTX - 1) / CTX;
  ti.nty = (ny + CTY - 1) / CTY;
  ti.ntiles = ti.ntx * ti.nty;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  __shared__ double s_p[HY][HX], s_c[HY][HX];
  (void)N;

  for (int tile = blockIdx.x; tile < ti.ntiles; tile += nb) {
    int i0, j0;
    tile_origin(ti, tile, &i0, &j0);
    const int j = j0 + ty;
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      const int i = i0 + c * 32 + tx;
      if (i < nx && j < ny) {
        const long k = (long)j * nx + i;
        if (!a.x0_from_x) x[k] = 0.0;
        p0[k] = 0.0;
        p1[k] = 0.0;
      }
    }
  }
  {
    double none[1] = {0};
    if (!grid_allreduce<1>(none, sc, partials, totals, nb)) return;
  }

  double acc[3] = {0, 0, 0};
  for (int tile = blockIdx.x; tile < ti.ntiles; tile += nb) {
    int i0, j0;
    tile_origin(ti, tile, &i0, &j0);
    const int j = j0 + ty;
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      const int i = i0 + c * 32 + tx;
      if (i < nx && j < ny) {
        const long k = (long)j * nx + i;
        const double ct = Ct[k], bk = b[k];
        // a decoupled neighbour enters at its exact b/|Ct|; outside the domain: 0
        auto xv = [&](int ii, int jj) -> double {
          if (ii < 0 || ii >= nx || jj < 0 || jj >= ny) return 0.0;
          const long kk = (long)jj * nx + ii;
          const double cc = Ct[kk];
          return cc < 0 ? b[kk] / (-cc) : ld(x, kk);
        };
        double rv;
        if (ct > 0) {
          const double gw = i > 0 ? Gx[k - 1] : 0.0, gs = j > 0 ? Gy[k - nx] : 0.0;
          const double ax = ct * ld(x, k) - (Gx[k] * xv(i + 1, j) + gw * xv(i - 1, j) +
                                             Gy[k] * xv(i, j + 1) + gs * xv(i, j - 1));
          rv = bk - ax;
        } else {
          rv = bk - (-ct) * ld(x, k);
        }
        acc[0] += rv * (rv / fabs(ct));
        acc[1] += rv * rv;
        acc[2] += bk * bk;
        r[k] = rv;
      }
    }
  }
  if (!grid_allreduce<3>(acc, sc, partials, totals, nb)) return;
  double rho = acc[0], rr = acc[1], rho_old = 1.0;
  const double bnorm = sqrt(acc[2]);
  int it = 0, cur = 0;
  auto converged = [&](double rr_) {
    const double rn = sqrt(rr_);
    return rn < a.eps * bnorm || (bnorm == 0.0 && 1.0 + rn == 1.0);
  };
  while (!converged(rr) && it < a.max_iter) {
    ++it;
    const double beta = it == 1 ? 0.0 : rho / rho_old;
    const double *pold = cur ? p1 : p0;
    double *pnew = cur ? p0 : p1;
    double pq[1] = {0};
    for (int tile = blockIdx.x; tile < ti.ntiles; tile += nb) {
      int i0, j0;
      tile_origin(ti, tile, &i0, &j0);
      __syncthreads();
      for (int e = threadIdx.x; e < HX * HY; e += kCgThreads) {
        const int ey = e / HX, ex = e - ey * HX;
        const int i = i0 - 1 + ex, j = j0 - 1 + ey;
        double pv = 0.0, cv = -1.0;
        if (i >= 0 && i < nx && j >= 0 && j < ny) {
          const long k = (long)j * nx + i;
          cv = Ct[k];
          pv = ld(r, k) / fabs(cv) + beta * ld(pold, k);
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
          const long k = (long)j * nx + i;
          const double ct = s_c[ly][lx], pc = s_p[ly][lx];
          auto nb_p = [&](int yy, int xx) -> double { return s_c[yy][xx] < 0 ? 0.0 : s_p[yy][xx]; };
          double qv;
          if (ct > 0) {
            const double gw = i > 0 ? Gx[k - 1] : 0.0, gs = j > 0 ? Gy[k - nx] : 0.0;
            qv = ct * pc - (Gx[k] * nb_p(ly, lx + 1) + gw * nb_p(ly, lx - 1) +
                            Gy[k] * nb_p(ly + 1, lx) + gs * nb_p(ly - 1, lx));
          } else {
            qv = (-ct) * pc;
          }
          pnew[k] = pc;
          q[k] = qv;
          pq[0] += pc * qv;
        }
      }
    }
    if (!grid_allreduce<1>(pq, sc, partials, totals, nb)) return;
    const double alpha = rho / pq[0];
    double a2[2] = {0, 0};
    for (int tile = blockIdx.x; tile < ti.ntiles; tile += nb) {
      int i0, j0;
      tile_origin(ti, tile, &i0, &j0);
      const int j = j0 + ty;
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        const int i = i0 + c * 32 + tx;
        if (i < nx && j < ny) {
          const long k = (long)j * nx + i;
          const double rv = ld(r, k) - alpha * ld(q, k);
          x[k] = ld(x, k) + alpha * ld(pnew, k);
          r[k] = rv;
          a2[0] += rv * (rv / fabs(Ct[k]));
          a2[1] += rv * rv;
        }
      }
    }
    if (!grid_allreduce<2>(a2, sc, partials, totals, nb)) return;
    rho_old = rho;
    rho = a2[0];
    rr = a2[1];
    cur ^= 1;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->cg_iters = it;
    sc->cg_rr = rr;
    sc->cg_bb = bnorm * bnorm;
  }
}

// Per-device set-up: the device address of the scratch array and the
// cooperative grid size, found once per device with that device current.
struct DeviceSetup {
  bool done = false;
  double *scratch = nullptr;
  int max_blocks = 0;
};
constexpr int kMaxDevices = 64;
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mu;

int setup_current_device(DeviceSetup **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(FREHD_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(FREHD_ERR_INVALID, "device %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_setup_mu);
  DeviceSetup &s = g_setup[dev];
  if (!s.done) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      return fail(FREHD_ERR_CUDA, "cudaGetSymbolAddress(g_noalloc_scratch): %s", cudaGetErrorString(e));
    int nsm = 0, per = 0;
    e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return fail(FREHD_ERR_CUDA, "device attribute: %s", cudaGetErrorString(e));
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_cg_noalloc, kCgThreads, 0);
    if (e != cudaSuccess) return fail(FREHD_ERR_CUDA, "occupancy: %s", cudaGetErrorString(e));
    s.scratch = static_cast<double *>(p);
    s.max_blocks = nsm * (per > 0 ? per : 1);
    if (s.max_blocks > kNoAllocMaxBlocks) s.max_blocks = kNoAllocMaxBlocks;
    s.done = true;
  }
  *out = &s;
  return FREHD_OK;
}

}  // namespace

extern "C" int frehd_cg_solve_noalloc(int nx, int ny, const double *Ct, const double *Gx,
                                      const double *Gy, const double *b, double *x, double eps,
                                      int max_iter, int x0_from_x, void *stream, int *iters,
                                      double *rel_residual) {
  clear_error();
  if (nx < 1 || ny < 1) return fail(FREHD_ERR_INVALID, "frehd_cg_solve_noalloc: bad size %d x %d", nx, ny);
  if ((long)nx * ny > kNoAllocMaxCells)
    return fail(FREHD_ERR_INVALID,
                "frehd_cg_solve_noalloc: %d x %d = %ld cells exceeds the no-allocation maximum "
                "of %ld cells",
                nx, ny, (long)nx * ny, kNoAllocMaxCells);
  if (!Ct || !Gx || !Gy || !b || !x) return fail(FREHD_ERR_INVALID, "frehd_cg_solve_noalloc: null array");
  if (!(eps > 0) || max_iter < 0) return fail(FREHD_ERR_INVALID, "frehd_cg_solve_noalloc: bad eps/max_iter");
  DeviceSetup *s = nullptr;
  int rc = setup_current_device(&s);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_noalloc_reset<<<1, 1, 0, st>>>(s->scratch);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(FREHD_ERR_CUDA, "reset launch: %s", cudaGetErrorString(e));
  const long ntiles = (long)((nx + CTX - 1) / CTX) * ((ny + CTY - 1) / CTY);
  const int grid = (int)(ntiles < s->max_blocks ? ntiles : s->max_blocks);
  NoAllocArgs a{nx, ny, Ct, Gx, Gy, b, x, eps, max_iter, x0_from_x, s->scratch};
  void *args[] = {&a};
  e = cudaLaunchCooperativeKernel((void *)k_cg_noalloc, dim3(grid), dim3(kCgThreads), args, 0, st);
  if (e != cudaSuccess) return fail(FREHD_ERR_CUDA, "cooperative launch: %s", cudaGetErrorString(e));
  if (!iters && !rel_residual) return FREHD_OK;  // asynchronous: results land in x
  Scratch h;
  e = cudaMemcpyAsync(&h, s->scratch, sizeof(Scratch), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(FREHD_ERR_CUDA, "reading the solve status: %s", cudaGetErrorString(e));
  if (iters) *iters = h.cg_iters;
  if (rel_residual) *rel_residual = h.cg_bb > 0 ? std::sqrt(h.cg_rr) / std::sqrt(h.cg_bb) : 0.0;
  if (h.status != FREHD_OK) return fail(h.status, "frehd_cg_solve_noalloc: %s", frehd_status_string(h.status));
  return FREHD_OK;
}

// C ABI of one domain (include/frehd_b200.h): device allocation, layout
// conversion, the host-side initialisation sequence and the step driver.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <set>
#include <vector>

#include "cg1.h"
#include "domain.cuh"
#include "domain_host.h"
#include "frehd_internal.h"
#include "kernels.cuh"

using namespace frehd;

#define CUDA_TRY(expr)                                                                 \
  do {                                                                                 \
    cudaError_t e_ = (expr);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail(FREHD_ERR_CUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_),     \
                  __FILE__, __LINE__);                                                 \
  } while (0)


namespace {

// A domain's device memory comes from the device's stream-ordered pool on the
// domain's own stream and goes back the same way.  cudaFree synchronises the
// whole device, so a server destroying finished requests' domains would stall
// the batch it steps for everyone else; cudaFreeAsync waits for nothing.  The
// pool keeps what is freed (release threshold: everything), so the next
// domain's arrays reuse it.
void pool_setup(int device) {
  static std::mutex mu;
  static std::set<int> done;
  std::lock_guard<std::mutex> lk(mu);
  if (done.count(device)) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    unsigned long long keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaGetLastError();
  done.insert(device);
}

cudaError_t dev_alloc(frehd_domain *d, void **p, size_t bytes) {
  return cudaMallocAsync(p, std::max<size_t>(bytes, 1), d->stream);
}

void dev_free(frehd_domain *d, void *p) {
  if (p) cudaFreeAsync(p, d->stream);
}

// Pinned step-statistics blocks, reused across domains (cudaFreeHost
// synchronises the device too).
std::mutex g_out_mu;
std::vector<StepOut *> g_out_free;

StepOut *take_out_host() {
  {
    std::lock_guard<std::mutex> lk(g_out_mu);
    if (!g_out_free.empty()) {
      StepOut *o = g_out_free.back();
      g_out_free.pop_back();
      return o;
    }
  }
  StepOut *o = nullptr;
  if (cudaMallocHost((void **)&o, sizeof(StepOut)) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return o;
}

void give_out_host(StepOut *o) {
  if (!o) return;
  std::lock_guard<std::mutex> lk(g_out_mu);
  g_out_free.push_back(o);
}

template <class T>
int dalloc(frehd_domain *d, T **p, long n) {
  void *q = nullptr;
  cudaError_t e = dev_alloc(d, &q, sizeof(T) * (size_t)std::max(n, 1L));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(FREHD_ERR_NOMEM, "device allocation of %ld bytes: %s", (long)(sizeof(T) * n),
                cudaGetErrorString(e));
  }
  cudaMemsetAsync(q, 0, sizeof(T) * (size_t)std::max(n, 1L), d->stream);
  d->allocs.push_back(q);
  d->bytes += (long long)(sizeof(T) * (size_t)std::max(n, 1L));
  *p = (T *)q;
  return FREHD_OK;
}

int check_config(const frehd_config *c) {
  if (c->nx < 2 || c->ny < 2) return fail(FREHD_ERR_INVALID, "grid %d x %d too small", c->nx, c->ny);
  if ((long)c->nx * c->ny > 2000000000L) return fail(FREHD_ERR_INVALID, "grid too large");
  if (c->useSubgrid != 1) return fail(FREHD_ERR_UNSUPPORTED, "useSubgrid=%d (only 1)", c->useSubgrid);
  if (c->staggeredV != 1) return fail(FREHD_ERR_UNSUPPORTED, "staggeredV=%d (only 1)", c->staggeredV);
  if (c->useSubDrag != 0) return fail(FREHD_ERR_UNSUPPORTED, "useSubDrag=%d (only 0)", c->useSubDrag);
  if (c->CDnotN != 0) return fail(FREHD_ERR_UNSUPPORTED, "CDnotN=%d (only 0)", c->CDnotN);
  if (c->useminA != 0) return fail(FREHD_ERR_UNSUPPORTED, "useminA=%d (only 0)", c->useminA);
  if (c->useminV == 1 || c->useminV == 2)
    return fail(FREHD_ERR_UNSUPPORTED, "useminV=%d (1 and 2 not implemented)", c->useminV);
  if (c->bcType != 1) return fail(FREHD_ERR_UNSUPPORTED, "bcType=%d (only 1)", c->bcType);
  // ReadUserSettings never assigns useEvap, useRain, useSubStep or
  // checkConservation (configuration.c:18-159): the reference never runs them
  if (c->useEvap || c->useRain || c->useSubStep || c->checkConservation)
    return fail(FREHD_ERR_UNSUPPORTED, "evaporation/rain/sub-stepping/conservation output");
  if (c->useWind != 0 && c->useWind != 1) return fail(FREHD_ERR_INVALID, "useWind=%d", c->useWind);
  if (c->inflowLocLength < 0 ||
      (c->inflowLocLength > 0 &&
       (c->inflowI0 < 0 || c->inflowJ0 < 0 || c->inflowI1 > c->nx || c->inflowJ1 > c->ny ||
        (long)(c->inflowI1 - c->inflowI0) * (c->inflowJ1 - c->inflowJ0) != c->inflowLocLength)))
    return fail(FREHD_ERR_INVALID, "inflow cells must be the rectangle of inflowLocLength interior cells");
  if (c->useScalar && ((c->scalarAdv != 1 && c->scalarAdv != 2) || c->useConstTidePS != 1))
    return fail(FREHD_ERR_UNSUPPORTED, "scalar: scalarAdv 1 or 2 with a constant tidal scalar");
  if (c->nscalar < 0 || c->nscalar > FREHD_MAX_SCALARS)
    return fail(FREHD_ERR_INVALID, "nscalar=%d (0 .. %d)", c->nscalar, FREHD_MAX_SCALARS);
  if (c->tideLocFirstP < 0 || c->tideLocLengthP < 0 || c->tideLocFirstP + c->tideLocLengthP > c->nx)
    return fail(FREHD_ERR_INVALID, "tidal cells outside the YP row");
  if (!(c->dsurf > 0) || !(c->dx > 0) || !(c->dy > 0) || !(c->dt > 0))
    return fail(FREHD_ERR_INVALID, "dx, dy, dt and dsurf must be positive");
  return FREHD_OK;
}

View make_view_at(const frehd_domain *d, int cur) {
  View w;
  w.p = d->p;
  w.gr = d->gr;
  const int c = cur, n = cur ^ 1;
  w.surf_cur = d->surf[c]; w.surf_nxt = d->surf[n];
  w.depth_cur = d->depth[c]; w.depth_nxt = d->depth[n];
  w.S_cur = d->S[c]; w.S_nxt = d->S[n];
  for (int s = 0; s < FREHD_MAX_SCALARS - 1; ++s) { w.Tr_cur[s] = d->Tr[s][c]; w.Tr_nxt[s] = d->Tr[s][n]; }
  w.ind_cur = d->ind[c]; w.ind_nxt = d->ind[n];
  w.u = d->u; w.v = d->v; w.CDXP = d->CDXP; w.CDYP = d->CDYP; w.CFLx = d->CFLx; w.CFLy = d->CFLy;
  w.V = d->V; w.Z = d->Z; w.Nx = d->Nx; w.Oy = d->Oy; w.Vx = d->Vx; w.Vy = d->Vy; w.Zx = d->Zx;
  w.Zy = d->Zy;
  w.bottomZ = d->bottomZ; w.bottomXP = d->bottomXP; w.bottomYP = d->bottomYP;
  w.EnXP = d->EnXP; w.EnYP = d->EnYP; w.Gx = d->Gx; w.Gy = d->Gy; w.Ct = d->Ct; w.b = d->b;
  w.Hx = d->Hx; w.Hy = d->Hy;
  w.fr0 = d->fr0; w.fr1 = d->fr1; w.fp0 = d->fp0; w.fp1 = d->fp1; w.fd = d->fd;
  w.fhx = d->fhx; w.fhy = d->fhy; w.fs = d->fs;
  w.x = d->x; w.r = d->r; w.p0 = d->p0; w.p1 = d->p1; w.q = d->q;
  w.cellV = d->cellV; w.Sm = d->Sm; w.Fuu = d->Fuu; w.Fvv = d->Fvv;
  w.rmv = d->rmv; w.fix_list = d->fix_list; w.partials = d->partials;
  w.tide = d->tide; w.ntide = d->ntide;
  w.inflow = d->inflow; w.ninflow = d->ninflow;
  w.wspd = d->wspd; w.nwspd = d->nwspd; w.wcos = d->wcos; w.wsin = d->wsin; w.nwdir = d->nwdir;
  w.dXP = d->dXP; w.dYP = d->dYP;
  w.lvc = d->lvc;
  w.lvi = d->lvi;
  w.sc = d->sc;
  return w;
}

View make_view(const frehd_domain *d) { return make_view_at(d, d->cur); }

dim3 tile_grid(const frehd_domain *d) {
  return dim3((d->gr.nx + 31) / 32, (d->gr.ny + 7) / 8);
}

__global__ void k_set_tt(Scratch *sc, int tt) { sc->tt = tt; }

// A new state clears what a stopped step left behind: the device status (after
// CFL > 20 or a wait that gave up), a half-counted grid barrier, the per-step
// counters and the failure-path test settings.
__global__ void k_reset_scratch(Scratch *sc) {
  sc->status = FREHD_OK;
  sc->bar_count = 0;
  sc->n_fix = 0;
  sc->n_cfl_warn = 0;
  sc->max_cflx_bits = 0;
  sc->max_cfly_bits = 0;
  sc->cg_noconv = 0;
  sc->skip_barrier_rank1 = 0;
  sc->wait_limit_ns = 0;
}

__global__ void k_set_wait_test(Scratch *sc, unsigned long long limit_ns, int skip_rank1) {
  sc->wait_limit_ns = limit_ns;
  sc->skip_barrier_rank1 = skip_rank1;
}

// host copies in the reference layout: index helpers (map.c:45-143)
struct RefMap {
  int nx, ny;
  long N, T;
  long jPbd(int i) const { return N - nx + i; }
  long jPgt(int i) const { return N + i; }
  long jMbd(int i) const { return i; }
  long jMgt(int i) const { return N + nx + i; }
  long iPbd(int j) const { return (long)(j + 1) * nx - 1; }
  long iPgt(int j) const { return N + 2L * nx + j; }
  long iMbd(int j) const { return (long)j * nx; }
  long iMgt(int j) const { return N + 2L * nx + ny + j; }
  long iPjc(long ii) const { return ii % nx == nx - 1 ? N + 2L * nx + ii / nx : ii + 1; }
  long icjP(long ii) const { return ii / nx == ny - 1 ? N + ii % nx : ii + nx; }
  long iMjP() const { return T - 4; }
  long iPjP() const { return T - 3; }
  long iPjM() const { return T - 2; }
  long iMjM() const { return T - 1; }
};

int upload_ref(frehd_domain *d, double *dst_padded, const double *host, long n) {
  CUDA_TRY(cudaMemcpyAsync(d->stage, host, sizeof(double) * n, cudaMemcpyHostToDevice, d->stream));
  k_ref_to_padded<<<(unsigned)((n + 255) / 256), 256, 0, d->stream>>>(dst_padded, d->stage, n,
                                                                      d->gr.nx, d->gr.ny, d->gr.pitch);
  CUDA_TRY(cudaGetLastError());
  return FREHD_OK;
}

int download_ref(frehd_domain *d, double *host, const double *src_padded, long n) {
  k_padded_to_ref<<<(unsigned)((n + 255) / 256), 256, 0, d->stream>>>(d->stage, src_padded, n,
                                                                      d->gr.nx, d->gr.ny, d->gr.pitch);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemcpyAsync(host, d->stage, sizeof(double) * n, cudaMemcpyDeviceToHost, d->stream));
  CUDA_TRY(cudaStreamSynchronize(d->stream));
  return FREHD_OK;
}

int read_stats(frehd_domain *d) {
  CUDA_TRY(cudaMemcpyAsync(d->out_host, d->out, sizeof(StepOut), cudaMemcpyDeviceToHost, d->stream));
  CUDA_TRY(cudaStreamSynchronize(d->stream));
  const StepOut &o = *d->out_host;
  d->last.step = o.step;
  d->last.cg_iters = o.cg_iters;
  d->last.cg_fallback = o.cg_fallback;
  d->last.status = o.status;
  d->last.cg_rel_residual = o.cg_bb > 0 ? std::sqrt(o.cg_rr) / std::sqrt(o.cg_bb) : 0.0;
  d->last.max_cflx = o.max_cflx;
  d->last.max_cfly = o.max_cfly;
  d->last.n_cfl_warn = o.n_cfl_warn;
  d->last.volume = o.volume;
  d->last.cg_noconverge = o.cg_noconv;
  return FREHD_OK;
}

long long take_noconv(frehd_domain *d) {
  const long long n = d->out_host->cg_noconv_steps - d->noconv_seen;
  d->noconv_seen = d->out_host->cg_noconv_steps;
  return n;
}

int launch_cg(frehd_domain *d, const View &w) {
  if (d->cg_schedule == FREHD_CG_SINGLE_SWEEP)
    return cg1_launch(w, d->cg1_maps_dev, d->cg1_blocks_n, d->x0_mode, d->eliminate, d->stream);
  View wv = w;
  int x0 = d->x0_mode, el = d->eliminate;
  void *args[] = {&wv, &x0, &el};
  CUDA_TRY(cudaLaunchCooperativeKernel((void *)k_cg, dim3(d->cg_blocks), dim3(kCgThreads), args, 0,
                                       d->stream));
  return FREHD_OK;
}

// Event slots of step s (6 per step: before explicit, cg, geo, vel, finish, after).
cudaEvent_t *step_events(frehd_domain *d, int s) {
  if (!d->profiling) return nullptr;
  const size_t need = (size_t)(s + 1) * 6;
  while (d->ev.size() < need) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    d->ev.push_back(e);
  }
  return &d->ev[(size_t)s * 6];
}

void mark(cudaEvent_t *ev, int slot, cudaStream_t st) {
  if (ev) cudaEventRecord(ev[slot], st);
}

int launch_update(frehd_domain *d, const View &w, cudaEvent_t *ev = nullptr) {
  const dim3 gb = tile_grid(d), bb(32, 8);
  mark(ev, 2, d->stream);
  k_update_geo<<<gb, bb, 0, d->stream>>>(w);
  mark(ev, 3, d->stream);
  if (d->p.scalarAdv == 2)
    k_update_vel_tvd<<<gb, bb, 0, d->stream>>>(w);
  else
    k_update_vel<<<gb, bb, 0, d->stream>>>(w);
  mark(ev, 4, d->stream);
  k_finish<<<1, 256, 0, d->stream>>>(w, (int)(gb.x * gb.y), d->out);
  mark(ev, 5, d->stream);
  CUDA_TRY(cudaGetLastError());
  return FREHD_OK;
}

}  // namespace

View frehd::domain_view(const frehd_domain *d, int cur) { return make_view_at(d, cur); }
int frehd::domain_read_stats(frehd_domain *d) { return read_stats(d); }
long long frehd::domain_take_noconv(frehd_domain *d) { return take_noconv(d); }

// ---------------------------------------------------------------- lifecycle
extern "C" int frehd_device_count(int *count) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    cudaGetLastError();
    n = 0;
  }
  if (count) *count = n;
  return FREHD_OK;
}

extern "C" int frehd_domain_create(const frehd_config *cfg, int device, frehd_domain **out) {
  clear_error();
  if (!cfg || !out) return fail(FREHD_ERR_INVALID, "null argument");
  *out = nullptr;
  int rc = check_config(cfg);
  if (rc) return rc;
  CUDA_TRY(cudaSetDevice(device));
  pool_setup(device);
  frehd_domain *d = new frehd_domain();
  d->cfg = *cfg;
  d->device = device;
  if (cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete d;
    return fail(FREHD_ERR_CUDA, "cudaStreamCreate failed");
  }
  d->gr = Grid::make(cfg->nx, cfg->ny);
  d->N = (long)cfg->nx * cfg->ny;
  d->T = (long)(cfg->nx + 2) * (cfg->ny + 2);
  Params &p = d->p;
  std::memset(&p, 0, sizeof(p));
  p.nx = cfg->nx; p.ny = cfg->ny; p.pitch = d->gr.pitch;
  p.dx = cfg->dx; p.dy = cfg->dy; p.dt = cfg->dt; p.g = cfg->g; p.NUx = cfg->NUx; p.NUy = cfg->NUy;
  p.Kx = cfg->Kx; p.Ky = cfg->Ky; p.manningN = cfg->manningN; p.hD = cfg->hD;
  p.minDepth = cfg->minDepth; p.wtfh = cfg->wtfh; p.CFLl = cfg->CFLl; p.CFLh = cfg->CFLh;
  p.offset = cfg->offset; p.surfmin = cfg->surfmin; p.dsurf = cfg->dsurf; p.tidePS = cfg->tidePS;
  p.subR = cfg->subR; p.dxf = cfg->dxf; p.dyf = cfg->dyf; p.eps = cfg->eps;
  p.Ne = (int)std::lround((cfg->surfmax - cfg->surfmin) / cfg->dsurf);  // subgrid.c:2115
  p.useThinLayer = cfg->useThinLayer; p.useScalar = cfg->useScalar; p.scalarAdv = cfg->scalarAdv;
  p.nscalar = cfg->useScalar ? std::max(cfg->nscalar, 1) : 0;
  p.tideFirst = cfg->tideLocFirstP; p.tideLen = cfg->tideLocLengthP; p.maxIter = cfg->maxIter;
  p.inflowLen = cfg->inflowLocLength;
  p.inflowI0 = cfg->inflowI0; p.inflowI1 = cfg->inflowI1;
  p.inflowJ0 = cfg->inflowJ0; p.inflowJ1 = cfg->inflowJ1;
  p.inflowS = cfg->inflowS;
  p.useWind = cfg->useWind; p.rhoa = cfg->rhoa; p.Cw = cfg->Cw; p.CwT = cfg->CwT;
  p.mixed = 0;
  p.eps_inner = 1e-5;
  const long tot = d->gr.total;
  int r = 0;
  for (int a = 0; a < 2 && !r; ++a) {
    r |= dalloc(d, &d->surf[a], tot);
    r |= dalloc(d, &d->depth[a], tot);
    r |= dalloc(d, &d->S[a], tot);
    r |= dalloc(d, &d->ind[a], tot);
    for (int s = 0; s + 1 < p.nscalar && !r; ++s) r |= dalloc(d, &d->Tr[s][a], tot);
  }
  double **arrs[] = {&d->u, &d->v, &d->CDXP, &d->CDYP, &d->CFLx, &d->CFLy, &d->V, &d->Z, &d->Nx,
                     &d->Oy, &d->Vx, &d->Vy, &d->Zx, &d->Zy, &d->bottomZ, &d->bottomXP,
                     &d->bottomYP, &d->EnXP, &d->EnYP, &d->Gx, &d->Gy, &d->Hx, &d->Hy, &d->Ct, &d->b, &d->x, &d->r,
                     &d->p0, &d->p1, &d->q, &d->cellV, &d->Sm, &d->Fuu, &d->Fvv};
  for (auto a : arrs)
    if (!r) r |= dalloc(d, a, tot);
  if (!r) r |= dalloc(d, &d->rmv, tot);
  if (!r && cfg->useWind) {  // face depths the wind term reads (zero until set)
    r |= dalloc(d, &d->dXP, tot);
    if (!r) r |= dalloc(d, &d->dYP, tot);
  }
  if (!r) r |= dalloc(d, &d->fix_list, d->N);
  if (!r) r |= dalloc(d, &d->stage, d->T);
  if (!r) r |= dalloc(d, &d->stage2, d->T);
  if (!r) r |= dalloc(d, &d->sc, 1);
  if (!r) r |= dalloc(d, &d->out, 1);
  // CG launch size: all blocks co-resident (cooperative launch), no more blocks
  // than 256-cell chunks
  int nsm = 0, per = 0;
  if (!r) {
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_cg, kCgThreads, 0);
    long want = (long)((d->gr.nx + 127) / 128) * ((d->gr.ny + kCgThreads / 32 - 1) / (kCgThreads / 32));
    long cap = (long)nsm * std::max(per, 1);
    d->cg_blocks = (int)std::max(1L, std::min(want, cap));
    r |= cg1_blocks(device, d->gr, &d->cg1_blocks_n);
  }
  if (!r) {
    const long nvel = (long)((d->gr.nx + 31) / 32) * ((d->gr.ny + 7) / 8);
    d->npartials = std::max(nvel, std::max(4L * d->cg_blocks, (long)kCg1PartialStride * d->cg1_blocks_n) + 8);
    r |= dalloc(d, &d->partials, d->npartials);
  }
  // the single-sweep CG reads r/q and p0/p1 alternately, Hx and Hy as TMA boxes
  if (!r)
    r |= cg1_make_maps(d->gr, d->r, d->q, d->p0, d->p1, d->Hx, d->Hy, &d->cg1_maps);
  if (!r) r |= dalloc(d, &d->cg1_maps_dev, 1);
  if (!r && cudaMemcpyAsync(d->cg1_maps_dev, &d->cg1_maps, sizeof(Cg1Maps), cudaMemcpyHostToDevice,
                            d->stream) != cudaSuccess)
    r = fail(FREHD_ERR_CUDA, "copying the CG tensor maps to the device failed");
  if (!r && !(d->out_host = take_out_host())) r = fail(FREHD_ERR_NOMEM, "pinned host allocation failed");
  if (r) {
    frehd_domain_destroy(d);
    return r;
  }
  // Ct ghosts mark "no unknown" (negative) so the CG treats them as decoupled
  k_fill<<<(unsigned)((tot + 255) / 256), 256, 0, d->stream>>>(d->Ct, tot, -1.0);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(d->stream));
  if (cfg->useWind) {  // the direction before any series is set: zero plus northAngle
    const int rc = frehd_domain_set_series(d, FREHD_SERIES_WIND_DIR, 0, nullptr);
    if (rc) {
      frehd_domain_destroy(d);
      return rc;
    }
  }
  *out = d;
  return FREHD_OK;
}

extern "C" int frehd_domain_destroy(frehd_domain *d) {
  if (!d) return FREHD_OK;
  // an admitted domain's arrays are referenced by its batch's tables and graph
  if (d->in_batch) return fail(FREHD_ERR_STATE, "domain is in a batch: release it first");
  cudaSetDevice(d->device);
  if (d->stream) cudaStreamSynchronize(d->stream);
  if (d->stream) {  // the pool takes the memory back in the domain's stream order
    for (void *p : d->allocs) dev_free(d, p);
    for (void *p : {(void *)d->tables, (void *)d->zf, (void *)d->lvc, (void *)d->lvi, (void *)d->tide,
                    (void *)d->inflow, (void *)d->wspd, (void *)d->wcos, (void *)d->wsin})
      dev_free(d, p);
  }
  give_out_host(d->out_host);
  for (cudaEvent_t e : d->ev) cudaEventDestroy(e);
  if (d->stream) cudaStreamDestroy(d->stream);
  delete d;
  return FREHD_OK;
}

extern "C" int frehd_domain_set_tables(frehd_domain *d, int Ne, const double *tables) {
  if (!d || !tables) return fail(FREHD_ERR_INVALID, "null argument");
  if (Ne != d->p.Ne)
    return fail(FREHD_ERR_INVALID, "tables hold %d levels, the config implies Ne=%d", Ne, d->p.Ne);
  CUDA_TRY(cudaSetDevice(d->device));
  const size_t bytes = sizeof(double) * 10 * (size_t)Ne * d->N;
  dev_free(d, d->tables);
  d->tables = nullptr;
  d->bytes -= d->tables_bytes;
  d->tables_bytes = 0;
  if (dev_alloc(d, (void **)&d->tables, bytes) != cudaSuccess) {
    cudaGetLastError();
    d->tables = nullptr;
    return fail(FREHD_ERR_NOMEM, "tables: %zu bytes", bytes);
  }
  CUDA_TRY(cudaMemcpyAsync(d->tables, tables, bytes, cudaMemcpyHostToDevice, d->stream));
  d->p.geom_fine = 0;
  d->p.tab = d->tables;
  d->tables_bytes = (long long)bytes;
  d->bytes += d->tables_bytes;
  d->geom_set = 1;
  return FREHD_OK;
}

extern "C" int frehd_domain_set_fine_bottoms(frehd_domain *d, int r, const double *zf, long fpitch) {
  return frehd_domain_set_fine_bottoms_ex(d, r, zf, fpitch, 0);
}

extern "C" int frehd_domain_set_fine_bottoms_ex(frehd_domain *d, int r, const double *zf, long fpitch,
                                                int flags) {
  if (!d || !zf || r <= 0 || (flags & ~FREHD_GEOM_BLOCK_CHECK))
    return fail(FREHD_ERR_INVALID, "bad argument");
  const int check_block = (flags & FREHD_GEOM_BLOCK_CHECK) && r > 1;
  if (check_block && r > 8) return fail(FREHD_ERR_UNSUPPORTED, "block check needs r <= 8 (r = %d)", r);
  if (fpitch < (long)d->gr.nx * r) return fail(FREHD_ERR_INVALID, "fine pitch too small");
  if (std::fabs(d->cfg.dx / d->cfg.dxf - r) > 1e-9 * r)
    return fail(FREHD_ERR_INVALID, "r=%d does not match dx/dxf", r);
  CUDA_TRY(cudaSetDevice(d->device));
  const long rows = (long)d->gr.ny * r, cols = (long)d->gr.nx * r;
  dev_free(d, d->zf);
  d->zf = nullptr;
  if (dev_alloc(d, (void **)&d->zf, sizeof(double) * rows * cols) != cudaSuccess) {
    cudaGetLastError();
    d->zf = nullptr;
    return fail(FREHD_ERR_NOMEM, "fine bottoms: %ld bytes", (long)(sizeof(double) * rows * cols));
  }
  CUDA_TRY(cudaMemcpy2DAsync(d->zf, sizeof(double) * cols, zf, sizeof(double) * fpitch,
                             sizeof(double) * cols, rows, cudaMemcpyHostToDevice, d->stream));
  d->p.geom_fine = 1;
  d->p.zf = d->zf;
  d->bytes += (long long)(sizeof(double) * rows * cols) - d->zf_bytes;
  d->zf_bytes = (long long)(sizeof(double) * rows * cols);
  d->p.fpitch = cols;
  d->p.r = r;
  d->p.check_block = check_block;
  // the level-value cache: allocated once, emptied for every new set of bottoms
  const long tot = d->gr.total;
  if (!d->lvc) {
    const size_t vb = sizeof(double) * 20 * (size_t)tot, ib = sizeof(int) * 2 * (size_t)tot;
    if (dev_alloc(d, (void **)&d->lvc, vb) != cudaSuccess || dev_alloc(d, (void **)&d->lvi, ib) != cudaSuccess) {
      cudaGetLastError();
      dev_free(d, d->lvc);
      d->lvc = nullptr;
      d->lvi = nullptr;
      return fail(FREHD_ERR_NOMEM, "level-value cache: %zu bytes", vb + ib);
    }
    d->lvc_bytes = (long long)(vb + ib);
    d->bytes += d->lvc_bytes;
  }
  CUDA_TRY(cudaMemsetAsync(d->lvi, 0xff, sizeof(int) * 2 * (size_t)tot, d->stream));  // -1: empty
  d->geom_set = 1;
  return FREHD_OK;
}

extern "C" int frehd_domain_set_tide(frehd_domain *d, int n, const double *tideP) {
  if (!d || (n > 0 && !tideP) || n < 0) return fail(FREHD_ERR_INVALID, "bad argument");
  CUDA_TRY(cudaSetDevice(d->device));
  dev_free(d, d->tide);
  d->tide = nullptr;
  CUDA_TRY(dev_alloc(d, (void **)&d->tide, sizeof(double) * std::max(n, 1)));
  if (n) CUDA_TRY(cudaMemcpyAsync(d->tide, tideP, sizeof(double) * n, cudaMemcpyHostToDevice, d->stream));
  d->ntide = n;
  return FREHD_OK;
}

namespace {
int upload_series(frehd_domain *d, double **dst, const std::vector<double> &h) {
  dev_free(d, *dst);
  *dst = nullptr;
  CUDA_TRY(dev_alloc(d, (void **)dst, sizeof(double) * std::max<size_t>(h.size(), 1)));
  if (!h.empty()) {  // h is the caller's temporary: the copy completes before it goes
    CUDA_TRY(cudaMemcpyAsync(*dst, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice,
                             d->stream));
    CUDA_TRY(cudaStreamSynchronize(d->stream));
  }
  return FREHD_OK;
}
}  // namespace

extern "C" int frehd_domain_set_series(frehd_domain *d, int kind, int n, const double *values) {
  if (!d || n < 0 || (n > 0 && !values)) return fail(FREHD_ERR_INVALID, "bad argument");
  if (d->in_batch) return fail(FREHD_ERR_STATE, "the domain is stepped by a batch (release it first)");
  CUDA_TRY(cudaSetDevice(d->device));
  CUDA_TRY(cudaStreamSynchronize(d->stream));
  std::vector<double> h(values, values + n);
  int rc;
  switch (kind) {
    case FREHD_SERIES_INFLOW:
      rc = upload_series(d, &d->inflow, h);
      if (!rc) d->ninflow = n;
      return rc;
    case FREHD_SERIES_WIND_SPEED:
      rc = upload_series(d, &d->wspd, h);
      if (!rc) d->nwspd = n;
      return rc;
    case FREHD_SERIES_WIND_DIR: {
      // omega = (winddir[tt] + northAngle) * pi / 180 with the reference's pi
      // (nsfunctions.c:611-617), its cosine and sine taken here by the host's
      // libm as the reference takes them; entry n serves the steps past the
      // series, where the reference reads a zero direction
      const double pi = 3.1415926;
      std::vector<double> c(n + 1), s(n + 1);
      for (int t = 0; t <= n; ++t) {
        const double phi = (t < n ? h[t] : 0.0) + d->cfg.northAngle;
        const double omega = phi * pi / 180.0;
        c[t] = std::cos(omega);
        s[t] = std::sin(omega);
      }
      rc = upload_series(d, &d->wcos, c);
      if (!rc) rc = upload_series(d, &d->wsin, s);
      if (!rc) d->nwdir = n;
      return rc;
    }
    default:
      return fail(FREHD_ERR_INVALID, "unknown series kind %d", kind);
  }
}

extern "C" int frehd_domain_update_series(frehd_domain *d, int kind, int t0, int n,
                                          const double *values) {
  if (!d || t0 < 0 || n < 0 || (n > 0 && !values)) return fail(FREHD_ERR_INVALID, "bad argument");
  if (n == 0) return FREHD_OK;
  double *dst = nullptr;
  int len = 0;
  switch (kind) {
    case FREHD_SERIES_TIDE: dst = d->tide; len = d->ntide; break;
    case FREHD_SERIES_INFLOW: dst = d->inflow; len = d->ninflow; break;
    case FREHD_SERIES_WIND_SPEED: dst = d->wspd; len = d->nwspd; break;
    case FREHD_SERIES_WIND_DIR: len = d->nwdir; break;
    default: return fail(FREHD_ERR_INVALID, "unknown series kind %d", kind);
  }
  if ((long)t0 + n > len)
    return fail(FREHD_ERR_INVALID, "entries %d..%d past the series' %d (set it first)", t0,
                t0 + n - 1, len);
  CUDA_TRY(cudaSetDevice(d->device));
  if (kind != FREHD_SERIES_WIND_DIR) {
    CUDA_TRY(cudaMemcpyAsync(dst + t0, values, sizeof(double) * n, cudaMemcpyHostToDevice, d->stream));
    return FREHD_OK;
  }
  const double pi = 3.1415926;  // as in frehd_domain_set_series
  std::vector<double> c(n), s(n);
  for (int t = 0; t < n; ++t) {
    const double omega = (values[t] + d->cfg.northAngle) * pi / 180.0;
    c[t] = std::cos(omega);
    s[t] = std::sin(omega);
  }
  CUDA_TRY(cudaMemcpyAsync(d->wcos + t0, c.data(), sizeof(double) * n, cudaMemcpyHostToDevice, d->stream));
  CUDA_TRY(cudaMemcpyAsync(d->wsin + t0, s.data(), sizeof(double) * n, cudaMemcpyHostToDevice, d->stream));
  CUDA_TRY(cudaStreamSynchronize(d->stream));
  return FREHD_OK;
}

extern "C" int frehd_domain_set_solver(frehd_domain *d, int x0_mode) {
  if (!d || (x0_mode != FREHD_X0_ZERO && x0_mode != FREHD_X0_SURFACE))
    return fail(FREHD_ERR_INVALID, "bad solver option");
  d->x0_mode = x0_mode;
  return FREHD_OK;
}

extern "C" int frehd_domain_set_precision(frehd_domain *d, int mode, double eps_inner) {
  if (!d || (mode != FREHD_PRECISION_FP64 && mode != FREHD_PRECISION_MIXED))
    return fail(FREHD_ERR_INVALID, "bad precision mode");
  if (mode == FREHD_PRECISION_MIXED && !(eps_inner > 0 && eps_inner < 1))
    return fail(FREHD_ERR_INVALID, "eps_inner must lie in (0, 1)");
  if (d->in_batch) return fail(FREHD_ERR_STATE, "the domain is stepped by a batch (release it first)");
  CUDA_TRY(cudaSetDevice(d->device));
  if (mode == FREHD_PRECISION_MIXED && !d->fr0) {
    const long tot = d->gr.total;
    int r = 0;
    float **arrs[] = {&d->fr0, &d->fr1, &d->fp0, &d->fp1, &d->fd, &d->fhx, &d->fhy, &d->fs};
    for (auto a : arrs)
      if (!r) r |= dalloc(d, a, tot);
    if (!r) r |= cg1_make_maps_f32(d->gr, d->fr0, d->fr1, d->fp0, d->fp1, d->fhx, d->fhy, &d->cg1_maps);
    if (r) return r;
    CUDA_TRY(cudaMemcpyAsync(d->cg1_maps_dev, &d->cg1_maps, sizeof(Cg1Maps), cudaMemcpyHostToDevice,
                             d->stream));
    CUDA_TRY(cudaStreamSynchronize(d->stream));
  }
  d->p.mixed = mode == FREHD_PRECISION_MIXED;
  if (d->p.mixed) d->p.eps_inner = eps_inner;
  return FREHD_OK;
}

extern "C" int frehd_domain_set_decoupled(frehd_domain *d, int mode) {
  if (!d || (mode != FREHD_DECOUPLED_AS_ASSEMBLED && mode != FREHD_DECOUPLED_ELIMINATED))
    return fail(FREHD_ERR_INVALID, "bad decoupled-row mode");
  d->eliminate = mode == FREHD_DECOUPLED_ELIMINATED;
  return FREHD_OK;
}

extern "C" int frehd_domain_set_cg_schedule(frehd_domain *d, int schedule) {
  if (!d || (schedule != FREHD_CG_SINGLE_SWEEP && schedule != FREHD_CG_TWO_PHASE))
    return fail(FREHD_ERR_INVALID, "bad CG schedule");
  d->cg_schedule = schedule;
  return FREHD_OK;
}

// ---------------------------------------------------------------- state I/O
extern "C" int frehd_domain_upload_state(frehd_domain *d, const frehd_state *st) {
  if (d && d->in_batch) return fail(FREHD_ERR_STATE, "the domain is stepped by a batch (release it first)");
  if (!d || !st) return fail(FREHD_ERR_INVALID, "null argument");
  CUDA_TRY(cudaSetDevice(d->device));
  const long N = d->N, T = d->T;
  const int c = d->cur;
  k_reset_scratch<<<1, 1, 0, d->stream>>>(d->sc);
  CUDA_TRY(cudaGetLastError());
  struct Item {
    const double *h;
    double *dv;
    long n;
  } items[] = {
      {st->surf, d->surf[c], T}, {st->uuXP, d->u, T}, {st->vvYP, d->v, T}, {st->S, d->S[c], T},
      {st->depth, d->depth[c], N}, {st->CDXP, d->CDXP, T}, {st->CDYP, d->CDYP, T},
      {st->CFLx, d->CFLx, T}, {st->CFLy, d->CFLy, T}, {st->V, d->V, T}, {st->Z, d->Z, T},
      {st->Nx, d->Nx, T}, {st->Oy, d->Oy, T}, {st->Vx, d->Vx, T}, {st->Vy, d->Vy, T},
      {st->Zx, d->Zx, T}, {st->Zy, d->Zy, T}, {st->bottomZ, d->bottomZ, T},
      {st->bottomXP, d->bottomXP, T}, {st->bottomYP, d->bottomYP, T},
      {st->depthXP, d->dXP, T}, {st->depthYP, d->dYP, T},
  };
  for (auto &it : items)
    if (it.h && it.dv) {
      int rc = upload_ref(d, it.dv, it.h, it.n);
      if (rc) return rc;
    }
  // ping-pong state goes into both buffers, so ghost entries that no kernel
  // rewrites keep the uploaded values whichever buffer is current
  const int o = c ^ 1;
  struct Item2 {
    const double *h;
    double *dv;
    long n;
  } twins[] = {{st->surf, d->surf[o], T}, {st->S, d->S[o], T}, {st->depth, d->depth[o], N}};
  for (auto &it : twins)
    if (it.h) {
      int rc = upload_ref(d, it.dv, it.h, it.n);
      if (rc) return rc;
    }
  if (st->ind) {
    CUDA_TRY(cudaMemcpyAsync(d->stage, st->ind, sizeof(int) * T, cudaMemcpyHostToDevice, d->stream));
    for (int a = 0; a < 2; ++a)
      k_ref_to_padded_int<<<(unsigned)((T + 255) / 256), 256, 0, d->stream>>>(
          d->ind[a], (const int *)d->stage, T, d->gr.nx, d->gr.ny, d->gr.pitch);
    CUDA_TRY(cudaGetLastError());
  }
  CUDA_TRY(cudaStreamSynchronize(d->stream));
  d->ready = 1;
  return FREHD_OK;
}

extern "C" int frehd_domain_download_state(frehd_domain *d, frehd_state *st) {
  if (d && d->in_batch) return fail(FREHD_ERR_STATE, "the domain is stepped by a batch (release it first)");
  if (!d || !st) return fail(FREHD_ERR_INVALID, "null argument");
  CUDA_TRY(cudaSetDevice(d->device));
  const long N = d->N, T = d->T;
  const int c = d->cur, o = d->cur ^ 1;
  struct Item {
    double *h;
    const double *dv;
    long n;
  } items[] = {
      {st->surf, d->surf[c], T}, {st->uuXP, d->u, T}, {st->vvYP, d->v, T}, {st->S, d->S[c], T},
      {st->depth, d->depth[c], N}, {st->CDXP, d->CDXP, T}, {st->CDYP, d->CDYP, T},
      {st->CFLx, d->CFLx, T}, {st->CFLy, d->CFLy, T}, {st->V, d->V, T}, {st->Z, d->Z, T},
      {st->Nx, d->Nx, T}, {st->Oy, d->Oy, T}, {st->Vx, d->Vx, T}, {st->Vy, d->Vy, T},
      {st->Zx, d->Zx, T}, {st->Zy, d->Zy, T}, {st->bottomZ, d->bottomZ, T},
      {st->bottomXP, d->bottomXP, T}, {st->bottomYP, d->bottomYP, T},
      {st->surfOld, d->surf[o], T}, {st->EnXP, d->EnXP, T}, {st->EnYP, d->EnYP, T},
      {st->cellV, d->cellV, N}, {st->Sm, d->Sm, N}, {st->Fuu, d->Fuu, T}, {st->Fvv, d->Fvv, T},
      {st->depthXP, d->dXP, T}, {st->depthYP, d->dYP, T},
  };
  for (auto &it : items)
    if (it.h && it.dv) {
      int rc = download_ref(d, it.h, it.dv, it.n);
      if (rc) return rc;
    }
  if (st->ind) {
    k_padded_to_ref_int<<<(unsigned)((T + 255) / 256), 256, 0, d->stream>>>(
        (int *)d->stage, d->ind[c], T, d->gr.nx, d->gr.ny, d->gr.pitch);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(st->ind, d->stage, sizeof(int) * T, cudaMemcpyDeviceToHost, d->stream));
  }
  if (st->uuYP || st->vvXP) {
    View w = make_view(d);
    k_interp_velocity<<<(unsigned)((N + 255) / 256), 256, 0, d->stream>>>(w, d->stage, d->stage2);
    CUDA_TRY(cudaGetLastError());
    if (st->uuYP)
      CUDA_TRY(cudaMemcpyAsync(st->uuYP, d->stage, sizeof(double) * N, cudaMemcpyDeviceToHost, d->stream));
    if (st->vvXP)
      CUDA_TRY(cudaMemcpyAsync(st->vvXP, d->stage2, sizeof(double) * N, cudaMemcpyDeviceToHost, d->stream));
  }
  CUDA_TRY(cudaStreamSynchronize(d->stream));
  return FREHD_OK;
}

// Device buffers of scalar s at the current half (h = 0) or the other one (h = 1).
static double *scalar_buf(frehd_domain *d, int s, int h) {
  const int half = d->cur ^ h;
  return s == 0 ? d->S[half] : d->Tr[s - 1][half];
}

static int check_scalar(const frehd_domain *d, int s) {
  if (d->in_batch) return fail(FREHD_ERR_STATE, "the domain is stepped by a batch (release it first)");
  if (!d->p.useScalar || s < 0 || s >= d->p.nscalar)
    return fail(FREHD_ERR_INVALID, "scalar %d of a domain with %d", s, d->p.nscalar);
  return FREHD_OK;
}

extern "C" int frehd_domain_upload_scalar(frehd_domain *d, int s, const double *values) {
  if (!d || !values) return fail(FREHD_ERR_INVALID, "null argument");
  int rc = check_scalar(d, s);
  if (rc) return rc;
  CUDA_TRY(cudaSetDevice(d->device));
  // both halves, as frehd_domain_upload_state does for S
  for (int h = 0; h < 2 && !rc; ++h) rc = upload_ref(d, scalar_buf(d, s, h), values, d->T);
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(d->stream));
  return FREHD_OK;
}

extern "C" int frehd_domain_download_scalar(frehd_domain *d, int s, double *values) {
  if (!d || !values) return fail(FREHD_ERR_INVALID, "null argument");
  int rc = check_scalar(d, s);
  if (rc) return rc;
  CUDA_TRY(cudaSetDevice(d->device));
  rc = download_ref(d, values, scalar_buf(d, s, 0), d->T);
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(d->stream));
  return FREHD_OK;
}

extern "C" int frehd_domain_init_scalar(frehd_domain *d, int s, const double *S0) {
  if (!d) return fail(FREHD_ERR_INVALID, "null argument");
  int rc = check_scalar(d, s);
  if (rc) return rc;
  if (!d->ready) return fail(FREHD_ERR_STATE, "domain has no state (frehd_domain_init first)");
  CUDA_TRY(cudaSetDevice(d->device));
  const long N = d->N;
  std::vector<double> dep(N), S(d->T, 0.0);
  rc = download_ref(d, dep.data(), d->depth[d->cur], N);
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(d->stream));
  // initFieldValues (initialize.c:410-430), then the dry-cell zeroing of Init
  // (initialize.c:149); the ghost ring stays zero
  for (long ii = 0; ii < N; ++ii) S[ii] = (S0 && dep[ii] > 0) ? S0[ii] : 0.0;
  return frehd_domain_upload_scalar(d, s, S.data());
}

// ---------------------------------------------------------------- init
// Init (initialize.c:40-155) for the subgrid path, restated on the host in the
// reference layout; the subgrid evaluation (computeSubArea + combineSubArea) runs
// on the device with the step's own kernel.
extern "C" int frehd_domain_init(frehd_domain *d, const double *bottom, const double *bxp,
                                 const double *byp, const double *surf0, const double *u0,
                                 const double *v0, const double *S0, int round_trip_output) {
  if (!d || !bottom || !bxp || !byp || !surf0) return fail(FREHD_ERR_INVALID, "null argument");
  if (!d->geom_set) return fail(FREHD_ERR_STATE, "set tables or fine bottoms before init");
  CUDA_TRY(cudaSetDevice(d->device));
  const frehd_config &c = d->cfg;
  RefMap m{c.nx, c.ny, d->N, d->T};
  const long N = d->N, T = d->T;
  const double off = c.offset;
  std::vector<double> bz(T, 0.0), bx(T, 0.0), by(T, 0.0), s(T, 0.0), u(T, 0.0), v(T, 0.0),
      S(T, 0.0), cdx(T, c.CDx), cdy(T, c.CDy), dep(N, 0.0), hx(T, 0.0), hy(T, 0.0);
  std::vector<double> ex(N), ey(N);
  for (long ii = 0; ii < N; ++ii) {  // InitBathymetry (bathymetry.c:104-121)
    bz[ii] = bottom[ii] + off;
    ex[ii] = bxp[ii] + off;
    ey[ii] = byp[ii] + off;
  }
  for (int i = 0; i < c.nx; ++i) { bz[m.jMgt(i)] = bz[m.jMbd(i)]; bz[m.jPgt(i)] = bz[m.jPbd(i)]; }
  for (int j = 0; j < c.ny; ++j) { bz[m.iMgt(j)] = bz[m.iMbd(j)]; bz[m.iPgt(j)] = bz[m.iPbd(j)]; }
  // updateAllFaceElev, subgrid branch (nsfunctions.c:76-140)
  for (long ii = 0; ii < N; ++ii) bx[ii] = ex[ii];
  for (int j = 0; j < c.ny; ++j) { bx[m.iMgt(j)] = bz[m.iMbd(j)]; bx[m.iPgt(j)] = bx[m.iPbd(j)]; }
  for (int i = 0; i < c.nx; ++i) { bx[m.jMgt(i)] = bx[m.jMbd(i)]; bx[m.jPgt(i)] = bx[m.jPbd(i)]; }
  for (long ii = 0; ii < N; ++ii) by[ii] = ey[ii];
  for (int i = 0; i < c.nx; ++i) {
    const long gi = m.jMgt(i);
    by[gi] = bz[gi] > bz[i] ? bz[gi] : bz[i];
    by[m.jPgt(i)] = by[m.jPbd(i)];
  }
  for (int j = 0; j < c.ny; ++j) { by[m.iMgt(j)] = by[m.iMbd(j)]; by[m.iPgt(j)] = by[m.iPbd(j)]; }
  // initFieldValues (initialize.c:393-443)
  for (long ii = 0; ii < N; ++ii) {
    s[ii] = surf0[ii] + off;
    u[ii] = u0 ? u0[ii] : 0.0;
    v[ii] = v0 ? v0[ii] : 0.0;
    if (c.useScalar) S[ii] = S0 ? S0[ii] : 0.0;
  }
  for (long ii = 0; ii < N; ++ii)  // zeroNegSurf
    if (s[ii] < bz[ii]) s[ii] = bz[ii];
  // enforceFreeSurfaceBC / enforceVelocityBC with corners (nsfunctions.c:289-334)
  for (int i = 0; i < c.nx; ++i) {
    s[m.jPgt(i)] = s[m.jPbd(i)]; s[m.jMgt(i)] = s[m.jMbd(i)];
    u[m.jPgt(i)] = u[m.jPbd(i)]; u[m.jMgt(i)] = u[m.jMbd(i)];
    v[m.jPgt(i)] = v[m.jPbd(i)]; v[m.jMgt(i)] = v[m.jMbd(i)];
  }
  for (int j = 0; j < c.ny; ++j) {
    s[m.iPgt(j)] = s[m.iPbd(j)]; s[m.iMgt(j)] = s[m.iMbd(j)];
    u[m.iPgt(j)] = u[m.iPbd(j)]; u[m.iMgt(j)] = u[m.iMbd(j)];
    v[m.iPgt(j)] = v[m.iPbd(j)]; v[m.iMgt(j)] = v[m.iMbd(j)];
  }
  s[m.iPjP()] = s[m.iPgt(c.ny - 1)]; s[m.iPjM()] = s[m.iMgt(c.ny - 1)];
  s[m.iMjP()] = s[m.iPgt(0)]; s[m.iMjM()] = s[m.iMgt(0)];
  u[m.iPjP()] = u[m.jPgt(c.nx - 1)]; u[m.iPjM()] = u[m.jMgt(c.nx - 1)];
  u[m.iMjP()] = u[m.jPgt(0)]; u[m.iMjM()] = u[m.jMgt(0)];
  v[m.iPjP()] = v[m.iPgt(c.ny - 1)]; v[m.iPjM()] = v[m.iMgt(c.ny - 1)];
  v[m.iMjP()] = v[m.iPgt(0)]; v[m.iMjM()] = v[m.iMgt(0)];
  // enforceTidalBC at tt = 0
  std::vector<double> tide0(1, 0.0);
  if (d->ntide > 0) {
    CUDA_TRY(cudaMemcpyAsync(tide0.data(), d->tide, sizeof(double), cudaMemcpyDeviceToHost, d->stream));
    CUDA_TRY(cudaStreamSynchronize(d->stream));
  }
  for (int k = 0; k < c.tideLocLengthP; ++k) {
    const long cc = c.tideLocFirstP + k + (long)c.nx * (c.ny - 1);
    if (tide0[0] + off > bz[cc]) s[cc] = tide0[0] + off;
  }
  for (long ii = 0; ii < N; ++ii) {  // updateDepth
    dep[ii] = s[ii] - bz[ii];
    if (dep[ii] < 0) dep[ii] = 0;
  }
  // updateAllFaceDepth (nsfunctions.c:143-236): only the interior face depths
  // feed thinLayerDrag and the wind term
  for (long ii = 0; ii < N; ++ii) {
    const double a = s[ii], bE = s[m.iPjc(ii)], bN = s[m.icjP(ii)];
    hx[ii] = (a > bE ? a : bE) - bx[ii];
    hy[ii] = (a > bN ? a : bN) - by[ii];
  }
  for (int j = 0; j < c.ny; ++j) hx[m.iPbd(j)] = 0;
  for (int i = 0; i < c.nx; ++i) hy[m.jPbd(i)] = 0;
  for (long ii = 0; ii < N; ++ii) {
    if (hx[ii] < 0) hx[ii] = 0;
    if (hy[ii] < 0) hy[ii] = 0;
  }
  // thinLayerDrag, called unconditionally by Init (initialize.c:140), CDnotN = 0
  const double coeff = c.g * c.manningN * c.manningN;
  for (long ii = 0; ii < N; ++ii)
    if (dep[ii] > 0) {
      if (hx[ii] <= c.hD) cdx[ii] = coeff / std::pow(dep[ii], 2.0 / 3.0);
      if (hy[ii] <= c.hD) cdy[ii] = coeff / std::pow(dep[ii], 2.0 / 3.0);
    }
  if (c.useScalar)
    for (long ii = 0; ii < N; ++ii)
      if (dep[ii] <= 0) S[ii] = 0;
  std::vector<int> ind(T, d->p.Ne / 2);  // subgrid.c:2268-2270
  // upload and evaluate the subgrid geometry
  frehd_state st;
  std::memset(&st, 0, sizeof(st));
  st.surf = s.data(); st.uuXP = u.data(); st.vvYP = v.data(); st.S = S.data();
  st.depth = dep.data(); st.CDXP = cdx.data(); st.CDYP = cdy.data();
  st.bottomZ = bz.data(); st.bottomXP = bx.data(); st.bottomYP = by.data(); st.ind = ind.data();
  st.depthXP = hx.data(); st.depthYP = hy.data();  // held for the wind term only
  // no previous step: the advection limiter's CFL numbers start at zero (the
  // reference reads its never-written arrays), also on a domain set up again
  std::vector<double> zeros(T, 0.0);
  st.CFLx = zeros.data(); st.CFLy = zeros.data();
  int rc = frehd_domain_upload_state(d, &st);
  if (rc) return rc;
  {
    View w = make_view(d);
    k_update_geo_init<<<tile_grid(d), dim3(32, 8), 0, d->stream>>>(w);
    CUDA_TRY(cudaGetLastError());
    std::swap(d->ind[0], d->ind[1]);  // the evaluated indices become current
  }
  if (round_trip_output) {  // DataOutput at tt = 0 (fileio.c:65-66,120-121)
    for (long ii = 0; ii < N; ++ii) s[ii] = s[ii] - off;
    for (long ii = 0; ii < N; ++ii) s[ii] = s[ii] + off;
    rc = upload_ref(d, d->surf[d->cur], s.data(), T);
    if (rc) return rc;
  }
  CUDA_TRY(cudaStreamSynchronize(d->stream));
  d->ready = 1;
  return FREHD_OK;
}

// ---------------------------------------------------------------- stepping
extern "C" int frehd_domain_phase(frehd_domain *d, int phase, int tt, const double *x_ext) {
  if (d && d->in_batch) return fail(FREHD_ERR_STATE, "the domain is stepped by a batch (release it first)");
  if (!d) return fail(FREHD_ERR_INVALID, "null domain");
  if (!d->ready) return fail(FREHD_ERR_STATE, "domain has no state (init or upload first)");
  CUDA_TRY(cudaSetDevice(d->device));
  View w = make_view(d);
  if (phase == FREHD_PHASE_EXPLICIT) {
    k_set_tt<<<1, 1, 0, d->stream>>>(d->sc, tt);
    k_explicit<<<tile_grid(d), dim3(32, 8), 0, d->stream>>>(w);
    CUDA_TRY(cudaGetLastError());
  } else if (phase == FREHD_PHASE_SOLVE) {
    int rc = launch_cg(d, w);
    if (rc) return rc;
  } else if (phase == FREHD_PHASE_UPDATE) {
    k_set_tt<<<1, 1, 0, d->stream>>>(d->sc, tt);
    if (x_ext) {
      CUDA_TRY(cudaMemcpyAsync(d->stage, x_ext, sizeof(double) * d->N, cudaMemcpyHostToDevice, d->stream));
      k_solution_from_ref<<<(unsigned)((d->N + 255) / 256), 256, 0, d->stream>>>(w, d->stage);
      CUDA_TRY(cudaGetLastError());
    }
    int rc = launch_update(d, w);
    if (rc) return rc;
    d->cur ^= 1;
    rc = read_stats(d);
    if (rc) return rc;
    return d->last.status == FREHD_ERR_CFL ? FREHD_ERR_CFL : FREHD_OK;
  } else {
    return fail(FREHD_ERR_INVALID, "unknown phase %d", phase);
  }
  CUDA_TRY(cudaStreamSynchronize(d->stream));
  return FREHD_OK;
}

extern "C" int frehd_domain_run(frehd_domain *d, int t0, int nsteps) {
  if (d && d->in_batch) return fail(FREHD_ERR_STATE, "the domain is stepped by a batch (release it first)");
  if (!d) return fail(FREHD_ERR_INVALID, "null domain");
  if (!d->ready) return fail(FREHD_ERR_STATE, "domain has no state (init or upload first)");
  if (nsteps <= 0) return FREHD_OK;
  CUDA_TRY(cudaSetDevice(d->device));
  const int cur0 = d->cur;
  k_set_tt<<<1, 1, 0, d->stream>>>(d->sc, t0);
  for (int s = 0; s < nsteps; ++s) {
    View w = make_view(d);
    cudaEvent_t *ev = step_events(d, s);
    mark(ev, 0, d->stream);
    k_explicit<<<tile_grid(d), dim3(32, 8), 0, d->stream>>>(w);
    mark(ev, 1, d->stream);
    int rc = launch_cg(d, w);
    if (rc) return rc;
    rc = launch_update(d, w, ev);
    if (rc) return rc;
    d->cur ^= 1;
  }
  int rc = read_stats(d);
  if (rc) return rc;
  if (d->profiling) {
    for (int s = 0; s < nsteps; ++s) {
      cudaEvent_t *ev = &d->ev[(size_t)s * 6];
      float ms[5];
      for (int k = 0; k < 5; ++k) cudaEventElapsedTime(&ms[k], ev[k], ev[k + 1]);
      d->times.explicit_ms += ms[0];
      d->times.cg_ms += ms[1];
      d->times.update_geo_ms += ms[2];
      d->times.update_vel_ms += ms[3];
      d->times.finish_ms += ms[4];
    }
    d->times.steps += nsteps;
    d->times.cg_iters = d->out_host->cg_iters_total - d->iters_at_prof_start;
  }
  // after a fatal step the later steps are skipped on the device; recover the
  // buffer parity from the last completed step
  const int done = d->last.step - t0 + 1;
  if (done != nsteps) d->cur = cur0 ^ (done & 1);
  const long long noconv = take_noconv(d);
  if (d->last.status == FREHD_ERR_CFL) return fail(FREHD_ERR_CFL, "max CFL > 20 at step %d", d->last.step);
  if (d->last.status != FREHD_OK)
    return fail(d->last.status, "step %d: %s", d->last.step, frehd_status_string(d->last.status));
  if (noconv > 0)  // reported, not fatal: the steps ran on, as laspack's CGIter does
    return fail(FREHD_ERR_CG_NOCONVERGE, "CG reached maxIter = %d in %lld of steps %d..%d",
                d->p.maxIter, noconv, t0, t0 + nsteps - 1);
  return FREHD_OK;
}

extern "C" int frehd_domain_set_wait_test(frehd_domain *d, long long wait_limit_ns,
                                          int skip_barrier_rank) {
  if (d && d->in_batch) return fail(FREHD_ERR_STATE, "the domain is stepped by a batch (release it first)");
  if (!d || wait_limit_ns < 0 || skip_barrier_rank < -1)
    return fail(FREHD_ERR_INVALID, "bad argument");
  CUDA_TRY(cudaSetDevice(d->device));
  k_set_wait_test<<<1, 1, 0, d->stream>>>(d->sc, (unsigned long long)wait_limit_ns,
                                          skip_barrier_rank + 1);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(d->stream));
  return FREHD_OK;
}

extern "C" int frehd_domain_step(frehd_domain *d, int tt) {
  if (d && d->in_batch) return fail(FREHD_ERR_STATE, "the domain is stepped by a batch (release it first)"); return frehd_domain_run(d, tt, 1); }

extern "C" int frehd_domain_download_system(frehd_domain *d, double *GnCt, double *GnXP,
                                            double *GnXM, double *GnYP, double *GnYM, double *z) {
  if (!d) return fail(FREHD_ERR_INVALID, "null domain");
  CUDA_TRY(cudaSetDevice(d->device));
  const long N = d->N;
  double *h[6] = {GnCt, GnXP, GnXM, GnYP, GnYM, z};
  View w = make_view(d);
  for (int a = 0; a < 6; ++a) {
    if (!h[a]) continue;
    double *o[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    o[a] = d->stage;
    k_system_to_ref<<<(unsigned)((N + 255) / 256), 256, 0, d->stream>>>(w, o[0], o[1], o[2], o[3],
                                                                          o[4], o[5], o[6]);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(h[a], d->stage, sizeof(double) * N, cudaMemcpyDeviceToHost, d->stream));
    CUDA_TRY(cudaStreamSynchronize(d->stream));
  }
  return FREHD_OK;
}

extern "C" int frehd_domain_download_solution(frehd_domain *d, double *xs) {
  if (!d || !xs) return fail(FREHD_ERR_INVALID, "null argument");
  CUDA_TRY(cudaSetDevice(d->device));
  View w = make_view(d);
  k_system_to_ref<<<(unsigned)((d->N + 255) / 256), 256, 0, d->stream>>>(
      w, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, d->stage);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemcpyAsync(xs, d->stage, sizeof(double) * d->N, cudaMemcpyDeviceToHost, d->stream));
  CUDA_TRY(cudaStreamSynchronize(d->stream));
  return FREHD_OK;
}

extern "C" int frehd_domain_stats(frehd_domain *d, frehd_step_stats *out) {
  if (!d || !out) return fail(FREHD_ERR_INVALID, "null argument");
  int rc = read_stats(d);
  if (rc) return rc;
  *out = d->last;
  return FREHD_OK;
}

extern "C" int frehd_domain_set_profiling(frehd_domain *d, int on) {
  if (!d) return fail(FREHD_ERR_INVALID, "null domain");
  d->profiling = on ? 1 : 0;
  d->times = frehd_kernel_times{};
  int rc = read_stats(d);
  if (rc) return rc;
  d->iters_at_prof_start = d->out_host->cg_iters_total;
  return FREHD_OK;
}

extern "C" int frehd_domain_kernel_times(frehd_domain *d, frehd_kernel_times *out) {
  if (!d || !out) return fail(FREHD_ERR_INVALID, "null argument");
  *out = d->times;
  return FREHD_OK;
}

extern "C" int frehd_domain_stream(frehd_domain *d, void **stream) {
  if (!d || !stream) return fail(FREHD_ERR_INVALID, "null argument");
  *stream = (void *)d->stream;
  return FREHD_OK;
}

extern "C" int frehd_domain_sync(frehd_domain *d) {
  if (!d) return fail(FREHD_ERR_INVALID, "null domain");
  CUDA_TRY(cudaSetDevice(d->device));
  CUDA_TRY(cudaStreamSynchronize(d->stream));
  return FREHD_OK;
}

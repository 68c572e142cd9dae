// Batched stepping of many resident domains (include/frehd_b200.h, frehd_batch_*).
//
// Domains are set up one by one with the single-domain calls (create, geometry,
// tide, init), then admitted into a batch, which owns their stepping until they
// are released.  One batch step advances every admitted domain by one time step
// with five launches in total, whatever the number of domains:
//   k_explicit_batch, k_update_geo_batch, k_update_vel_batch   one block per
//       (domain, 32 x 8 tile) entry of a tile table over all domains
//   the solve, one cooperative launch over all co-resident CTAs, in one of two
//       packings (frehd_batch_set_cg_packing):
//     k_cg1_batch (FREHD_BATCH_CTA_GROUPS, the default): each domain solved by a group of
//       CTAs whose size depends on the domain's own cell count only (multi-CTA
//       groups on CTAs of their own; single-CTA domains, longest first, taken
//       one after another by whichever CTA is free)
//     k_cg1_tiles (FREHD_BATCH_TILE_LIST): the CG tiles of every domain form one
//       list spread over all CTAs; each domain's sums are added in its own tile
//       order, so its result depends neither on the mix nor on cells_per_cta
//   k_finish_batch   one block per domain; flips the domain's ping-pong half
// The five launches are captured once per batch composition into a CUDA graph
// and replayed every step.
//
// Admission is by device-memory footprint (a budget given at creation) and, in
// the CTA-group packing, by the CTA capacity of the cooperative solve.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "cg1.h"
#include "cg_common.cuh"
#include "domain_host.h"
#include "frehd_internal.h"
#include "kernels.cuh"

using namespace frehd;

#define BATCH_TRY(expr)                                                               \
  do {                                                                                \
    cudaError_t e_ = (expr);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return fail(FREHD_ERR_CUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_),     \
                  __FILE__, __LINE__);                                                \
  } while (0)

namespace {

// Stencil tiles (32 x 8) one block of the batched stencil kernels runs at most,
// one after another along a tile row: the domain's view is staged once for
// them (frehd_batch_set_stencil_tiles; the default, and the largest allowed).
constexpr int kTilesPerBlock = 4, kMaxTilesPerBlock = 8;

struct Slot {
  frehd_domain *d = nullptr;
  long long steps = 0;  // batch steps taken since admission
};

template <class T>
struct DevArray {
  T *p = nullptr;
  size_t cap = 0;
  // grows by half at least, so that a stream of admissions reallocates (and
  // cudaFree synchronises the device) only a logarithmic number of times
  int reserve(size_t n) {
    if (n <= cap) return FREHD_OK;
    const size_t want = std::max<size_t>(std::max<size_t>(n, cap + cap / 2), 16);
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    if (cudaMalloc(&p, sizeof(T) * want) != cudaSuccess) {
      cudaGetLastError();
      return fail(FREHD_ERR_NOMEM, "batch tables: %zu bytes", sizeof(T) * want);
    }
    cap = want;
    return FREHD_OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

}  // namespace

struct frehd_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  long long budget = 0, used = 0;
  double cells_per_cta = 0;
  int capacity = 0;        // co-resident CTAs of k_cg1_batch
  int capacity_tiles = 0;  // co-resident CTAs of k_cg1_tiles
  std::vector<Slot> slots;
  bool dirty = true;
  // tables of the current composition
  DevArray<View> views2;
  DevArray<const Cg1Maps *> maps;
  DevArray<BatchTile> tiles;
  DevArray<FinishJob> fins;
  DevArray<int> job_start;
  DevArray<CgJob> jobs;
  DevArray<CgJob> singles;  // single-CTA solves, longest first
  int nsingles = 0;
  int any_mixed = 0;        // an admitted domain solves in mixed precision
  // tile-list packing
  int packing = FREHD_BATCH_CTA_GROUPS;
  int tiles_per_block = kTilesPerBlock;
  DevArray<BDom> bdoms;
  DevArray<BTile> btiles;
  DevArray<BState> bstates;
  DevArray<double> bpartials, bpart;
  DevArray<Scratch> bsync;
  int nbdoms = 0, nbtiles = 0;
  long ntiles = 0, ntiles_upwind = 0;  // stencil tiles; those of upwind domains come first
  int nfin = 0, nctas = 0;
  // per-slot device status after each step, written by k_finish_batch into
  // host-mapped pinned memory (read by the server between steps)
  int *status_host = nullptr, *status_dev = nullptr;
  int status_cap = 0;
  // captured launches
  int use_graph = 1;
  cudaGraphExec_t graph = nullptr;
  int graph_live = 0;
  long long steps = 0;
};

namespace {

// CTAs that solve a domain of `cells` cells (by its size alone).
int group_size(const frehd_batch *b, const frehd_domain *d) {
  const long ntiles = (long)((d->gr.nx + CTX - 1) / CTX) * ((d->gr.ny + CTY - 1) / CTY);
  const double cells = (double)d->gr.nx * d->gr.ny;
  // ceil: no CTA of a group carries more than cells_per_cta cells
  long g = (long)std::ceil(cells / b->cells_per_cta);
  g = std::max(1L, std::min(g, std::min(ntiles, (long)b->capacity)));
  return (int)g;
}

// CTAs the batch needs with the given domains: the multi-CTA groups plus one
// CTA for the single-CTA domains (if any); the tile-list packing takes any mix.
int ctas_needed(const frehd_batch *b, const frehd_domain *extra) {
  if (b->packing == FREHD_BATCH_TILE_LIST) return 1;
  int dedicated = 0, singles = 0;
  auto add = [&](const frehd_domain *d) {
    const int g = group_size(b, d);
    if (g > 1) dedicated += g; else ++singles;
  };
  for (const Slot &s : b->slots)
    if (s.d) add(s.d);
  if (extra) add(extra);
  return dedicated + (singles ? 1 : 0);
}

// Room for `n` slot statuses; growing waits for the queued steps, which may
// still write the old array.
int reserve_status(frehd_batch *b, int n) {
  if (n <= b->status_cap) return FREHD_OK;
  const int cap = std::max(n, std::max(64, 2 * b->status_cap));
  BATCH_TRY(cudaStreamSynchronize(b->stream));
  int *h = nullptr, *dv = nullptr;
  if (cudaHostAlloc(&h, sizeof(int) * cap, cudaHostAllocMapped) != cudaSuccess ||
      cudaHostGetDevicePointer(&dv, h, 0) != cudaSuccess) {
    cudaGetLastError();
    if (h) cudaFreeHost(h);
    return fail(FREHD_ERR_NOMEM, "batch status array: %d slots", cap);
  }
  for (int k = 0; k < cap; ++k) h[k] = k < b->status_cap ? b->status_host[k] : FREHD_OK;
  if (b->status_host) cudaFreeHost(b->status_host);
  b->status_host = h;
  b->status_dev = dv;
  b->status_cap = cap;
  return FREHD_OK;
}

void drop_graph(frehd_batch *b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
  b->graph_live = 0;
}

int launch_step(frehd_batch *b) {
  const dim3 bb(32, 8);
  k_explicit_batch<<<(unsigned)b->ntiles, bb, 0, b->stream>>>(b->views2.p, b->tiles.p);
  const bool tl = b->packing == FREHD_BATCH_TILE_LIST;
  int rc = tl ? cg1_launch_tiles(b->views2.p, b->maps.p, b->bdoms.p, b->bstates.p, b->btiles.p,
                                 b->nbdoms, b->nbtiles, b->bpartials.p, b->bsync.p, b->bpart.p,
                                 b->nctas, b->stream)
              : cg1_launch_batch(b->views2.p, b->maps.p, b->job_start.p, b->jobs.p, b->singles.p,
                                 b->nsingles, &b->bsync.p->n_done, b->nctas, b->any_mixed,
                                 b->stream);
  if (rc) return rc;
  k_update_geo_batch<<<(unsigned)b->ntiles, bb, 0, b->stream>>>(b->views2.p, b->tiles.p);
  if (b->ntiles_upwind > 0)
    k_update_vel_batch<<<(unsigned)b->ntiles_upwind, bb, 0, b->stream>>>(b->views2.p, b->tiles.p);
  if (b->ntiles > b->ntiles_upwind)
    k_update_vel_tvd_batch<<<(unsigned)(b->ntiles - b->ntiles_upwind), bb, 0, b->stream>>>(
        b->views2.p, b->tiles.p + b->ntiles_upwind);
  k_finish_batch<<<(unsigned)b->nfin, 256, 0, b->stream>>>(b->views2.p, b->fins.p, b->bsync.p);
  BATCH_TRY(cudaGetLastError());
  return FREHD_OK;
}

// Rebuild the tables for the current composition (and the graph, lazily).
int rebuild(frehd_batch *b) {
  drop_graph(b);
  const int nslot = (int)b->slots.size();
  {
    const int rc = reserve_status(b, nslot);
    if (rc) return rc;
  }
  std::vector<View> views(2 * (size_t)std::max(nslot, 1));
  std::vector<const Cg1Maps *> maps(std::max(nslot, 1), nullptr);
  std::vector<BatchTile> tiles;
  std::vector<FinishJob> fins;
  struct Dom {
    int slot, g;
    double cells;
  };
  std::vector<Dom> doms;
  // stencil tiles of the upwind domains first, then the TVD ones (two kernels)
  for (int pass = 0; pass < 2; ++pass)
    for (int s = 0; s < nslot; ++s) {
      frehd_domain *d = b->slots[s].d;
      if (!d || (d->p.scalarAdv == 2) != (pass == 1)) continue;
      const int gx = (d->gr.nx + 31) / 32, gy = (d->gr.ny + 7) / 8;
      for (int by = 0; by < gy; ++by)
        for (int bx = 0; bx < gx; bx += b->tiles_per_block)
          tiles.push_back(BatchTile{s, bx, by, gx, std::min(b->tiles_per_block, gx - bx), 0});
    }
  long nup = 0;
  for (const BatchTile &t : tiles)
    if (b->slots[t.d].d->p.scalarAdv != 2) ++nup;
  for (int s = 0; s < nslot; ++s) {
    frehd_domain *d = b->slots[s].d;
    if (!d) continue;
    views[2 * s] = domain_view(d, 0);
    views[2 * s + 1] = domain_view(d, 1);
    maps[s] = d->cg1_maps_dev;
    const int gx = (d->gr.nx + 31) / 32, gy = (d->gr.ny + 7) / 8;
    fins.push_back(FinishJob{s, gx * gy, d->out, b->status_dev + s});
    doms.push_back(Dom{s, group_size(b, d), (double)d->gr.nx * d->gr.ny});
  }
  // the launch sizes describe the device tables: they stay zero (no launch) and
  // the batch stays dirty until every table of this composition is uploaded
  b->ntiles = 0;
  b->ntiles_upwind = 0;
  b->nfin = 0;
  b->nctas = 0;
  if (doms.empty()) {
    b->dirty = false;
    return FREHD_OK;
  }

  auto flags_of = [&](int s) {
    const frehd_domain *d = b->slots[s].d;
    return (d->x0_mode == FREHD_X0_SURFACE ? 1 : 0) | (d->eliminate ? 2 : 0);
  };
  // tile-list packing: every domain's CG tiles, domain after domain
  std::vector<BDom> bd;
  std::vector<BTile> bt;
  if (b->packing == FREHD_BATCH_TILE_LIST) {
    for (const Dom &m : doms) {
      const frehd_domain *d = b->slots[m.slot].d;
      const int ntx = (d->gr.nx + CTX - 1) / CTX, nty = (d->gr.ny + CTY - 1) / CTY;
      bd.push_back(BDom{m.slot, (int)bt.size(), ntx * nty, ntx, flags_of(m.slot), 0});
      for (int t = 0; t < ntx * nty; ++t) bt.push_back(BTile{(int)bd.size() - 1, t});
    }
  }
  // CTA-group packing: multi-CTA groups on CTAs of their own; single-CTA
  // domains in one list that every CTA takes from once its own jobs are done.
  std::vector<std::vector<CgJob>> per_cta;
  std::vector<Dom> singles;
  for (const Dom &m : doms) {
    if (b->packing == FREHD_BATCH_TILE_LIST) break;
    if (m.g > 1) {
      for (int r = 0; r < m.g; ++r) per_cta.push_back({CgJob{m.slot, r, m.g, flags_of(m.slot)}});
    } else {
      singles.push_back(m);
    }
  }
  const int free_ctas = b->capacity - (int)per_cta.size();
  if (b->packing != FREHD_BATCH_TILE_LIST && free_ctas < (singles.empty() ? 0 : 1))
    return fail(FREHD_ERR_STATE, "batch CTA capacity exceeded (%d CTAs for multi-CTA domains of %d)",
                (int)per_cta.size(), b->capacity);
  // single-CTA domains, longest first, taken by whichever CTA is free (k_cg1_batch)
  std::stable_sort(singles.begin(), singles.end(),
                   [](const Dom &a, const Dom &c) { return a.cells > c.cells; });
  std::vector<CgJob> single_jobs;
  for (const Dom &m : singles) single_jobs.push_back(CgJob{m.slot, 0, 1, flags_of(m.slot)});
  const int ngroups = (int)per_cta.size();
  const int nctas_groups = single_jobs.empty() ? ngroups : b->capacity;
  per_cta.resize(std::max(ngroups, nctas_groups));
  std::vector<int> start(per_cta.size() + 1, 0);
  std::vector<CgJob> jobs;
  for (size_t c = 0; c < per_cta.size(); ++c) {
    start[c] = (int)jobs.size();
    jobs.insert(jobs.end(), per_cta[c].begin(), per_cta[c].end());
  }
  start[per_cta.size()] = (int)jobs.size();

  int rc = 0;
  rc = rc ? rc : b->views2.reserve(views.size());
  rc = rc ? rc : b->maps.reserve(maps.size());
  rc = rc ? rc : b->tiles.reserve(tiles.size());
  rc = rc ? rc : b->fins.reserve(fins.size());
  rc = rc ? rc : b->job_start.reserve(start.size());
  rc = rc ? rc : b->jobs.reserve(jobs.size());
  rc = rc ? rc : b->singles.reserve(single_jobs.size());
  {  // the launch counter (both packings), zeroed once and reset by k_finish_batch
    const bool fresh_sync = b->bsync.cap == 0;
    rc = rc ? rc : b->bsync.reserve(1);
    if (!rc && fresh_sync)
      BATCH_TRY(cudaMemsetAsync(b->bsync.p, 0, sizeof(Scratch) * b->bsync.cap, b->stream));
  }
  const bool tl = b->packing == FREHD_BATCH_TILE_LIST;
  if (tl) {
    rc = rc ? rc : b->bdoms.reserve(bd.size());
    rc = rc ? rc : b->btiles.reserve(bt.size());
    rc = rc ? rc : b->bstates.reserve(bd.size());
    rc = rc ? rc : b->bpartials.reserve(bt.size() * (size_t)kTilePartStride);
    rc = rc ? rc : b->bpart.reserve(((size_t)b->capacity_tiles + 1) * kCg1PartialStride);
  }
  if (rc) return rc;
  BATCH_TRY(cudaMemcpyAsync(b->views2.p, views.data(), sizeof(View) * views.size(), cudaMemcpyHostToDevice, b->stream));
  BATCH_TRY(cudaMemcpyAsync(b->maps.p, maps.data(), sizeof(const Cg1Maps *) * maps.size(), cudaMemcpyHostToDevice, b->stream));
  BATCH_TRY(cudaMemcpyAsync(b->tiles.p, tiles.data(), sizeof(BatchTile) * tiles.size(), cudaMemcpyHostToDevice, b->stream));
  BATCH_TRY(cudaMemcpyAsync(b->fins.p, fins.data(), sizeof(FinishJob) * fins.size(), cudaMemcpyHostToDevice, b->stream));
  BATCH_TRY(cudaMemcpyAsync(b->job_start.p, start.data(), sizeof(int) * start.size(), cudaMemcpyHostToDevice, b->stream));
  BATCH_TRY(cudaMemcpyAsync(b->jobs.p, jobs.data(), sizeof(CgJob) * jobs.size(), cudaMemcpyHostToDevice, b->stream));
  if (!single_jobs.empty())
    BATCH_TRY(cudaMemcpyAsync(b->singles.p, single_jobs.data(), sizeof(CgJob) * single_jobs.size(),
                              cudaMemcpyHostToDevice, b->stream));
  if (tl) {
    BATCH_TRY(cudaMemcpyAsync(b->bdoms.p, bd.data(), sizeof(BDom) * bd.size(), cudaMemcpyHostToDevice, b->stream));
    BATCH_TRY(cudaMemcpyAsync(b->btiles.p, bt.data(), sizeof(BTile) * bt.size(), cudaMemcpyHostToDevice, b->stream));
  }
  // the host vectors go out of scope: the copies must have left them
  BATCH_TRY(cudaStreamSynchronize(b->stream));
  b->ntiles = (long)tiles.size();
  b->ntiles_upwind = nup;
  b->nfin = (int)fins.size();
  b->nctas = tl ? b->capacity_tiles : (int)per_cta.size();
  b->nsingles = (int)single_jobs.size();
  b->any_mixed = 0;
  for (const Dom &m : doms) b->any_mixed |= b->slots[m.slot].d->p.mixed ? 1 : 0;
  b->nbdoms = (int)bd.size();
  b->nbtiles = (int)bt.size();
  b->dirty = false;
  return FREHD_OK;
}

// Capture the five launches of one step into a graph; on any failure the batch
// keeps launching them directly.
void capture(frehd_batch *b) {
  if (!b->use_graph || b->graph_live || b->nfin == 0) return;
  cudaGraph_t g = nullptr;
  if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    b->use_graph = 0;
    return;
  }
  const int rc = launch_step(b);
  const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
  if (rc || e != cudaSuccess || !g) {
    cudaGetLastError();
    clear_error();
    if (g) cudaGraphDestroy(g);
    b->use_graph = 0;
    return;
  }
  if (cudaGraphInstantiate(&b->graph, g, 0) != cudaSuccess) {
    cudaGetLastError();
    b->graph = nullptr;
    b->use_graph = 0;
  } else {
    b->graph_live = 1;
  }
  cudaGraphDestroy(g);
}

}  // namespace

int frehd::batch_slot_status(const frehd_batch *b, int slot) {
  if (!b || slot < 0 || slot >= b->status_cap) return FREHD_OK;
  return *(volatile int *)&b->status_host[slot];
}

extern "C" int frehd_domain_footprint(const frehd_config *cfg, int r, long long *bytes) {
  if (!cfg || !bytes || r < 1 || cfg->nx < 2 || cfg->ny < 2) return fail(FREHD_ERR_INVALID, "bad argument");
  const Grid g = Grid::make(cfg->nx, cfg->ny);
  const long long tot = g.total, N = (long long)cfg->nx * cfg->ny;
  const long long T = (long long)(cfg->nx + 2) * (cfg->ny + 2);
  const long long nvel = (long long)((cfg->nx + 31) / 32) * ((cfg->ny + 7) / 8);
  long long b = 0;
  b += 2 * (3 * 8 + 4) * tot;       // surf, depth, S (double) and ind (int), both halves
  if (cfg->useScalar && cfg->nscalar > 1) b += 2 * 8 * tot * (long long)(cfg->nscalar - 1);  // tracers
  b += 36 * 8 * tot;                // persistent, per-step and CG arrays
  b += tot;                         // rmv flags
  b += 4 * N + 2 * 8 * T;           // fix list, staging
  b += 8 * std::max(nvel, 8LL * 148 + 8) + 4096;  // partials, scratch, maps
  b += 8 * N * (long long)r * r;    // fine bottoms
  b += (20 * 8 + 2 * 4) * tot;      // level-value cache of the fine geometry
  *bytes = b;
  return FREHD_OK;
}

extern "C" int frehd_batch_create(int device, long long hbm_budget_bytes, double cells_per_cta,
                                  frehd_batch **out) {
  clear_error();
  if (!out || hbm_budget_bytes <= 0 || !(cells_per_cta > 0)) return fail(FREHD_ERR_INVALID, "bad argument");
  *out = nullptr;
  BATCH_TRY(cudaSetDevice(device));
  frehd_batch *b = new frehd_batch();
  b->device = device;
  b->budget = hbm_budget_bytes;
  b->cells_per_cta = cells_per_cta;
  int rc = cg1_batch_capacity(device, &b->capacity);
  if (!rc) rc = cg1_tiles_capacity(device, &b->capacity_tiles);
  if (!rc && cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
    rc = fail(FREHD_ERR_CUDA, "stream creation failed");
  if (rc) {
    delete b;
    return rc;
  }
  *out = b;
  return FREHD_OK;
}

extern "C" int frehd_batch_destroy(frehd_batch *b) {
  if (!b) return FREHD_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (Slot &s : b->slots)
    if (s.d) {  // hand back in a consistent state before the caller destroys it
      int cur = 0;
      cudaMemcpy(&cur, &s.d->sc->cur, sizeof(int), cudaMemcpyDeviceToHost);
      s.d->cur = cur & 1;
      s.d->in_batch = 0;
    }
  drop_graph(b);
  if (b->status_host) cudaFreeHost(b->status_host);
  b->views2.release();
  b->maps.release();
  b->tiles.release();
  b->fins.release();
  b->job_start.release();
  b->jobs.release();
  b->singles.release();
  b->bdoms.release();
  b->btiles.release();
  b->bstates.release();
  b->bpartials.release();
  b->bpart.release();
  b->bsync.release();
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return FREHD_OK;
}

extern "C" int frehd_batch_admit(frehd_batch *b, frehd_domain *d, int t0, int *slot) {
  clear_error();
  if (!b || !d || !slot) return fail(FREHD_ERR_INVALID, "null argument");
  if (!d->ready) return fail(FREHD_ERR_STATE, "domain has no state (init or upload first)");
  if (d->in_batch) return fail(FREHD_ERR_STATE, "domain is already in a batch");
  if (d->device != b->device) return fail(FREHD_ERR_INVALID, "domain and batch are on different devices");
  if (b->used + d->bytes > b->budget)
    return fail(FREHD_ERR_NOMEM, "batch memory budget: %lld + %lld bytes > %lld", b->used, d->bytes, b->budget);
  if (ctas_needed(b, d) > b->capacity)
    return fail(FREHD_ERR_NOMEM, "batch CTA capacity: %d CTAs needed, %d available", ctas_needed(b, d),
                b->capacity);
  BATCH_TRY(cudaSetDevice(b->device));
  // the domain's own queued work (init, uploads) ends before the batch uses it
  BATCH_TRY(cudaStreamSynchronize(d->stream));
  const int cur = d->cur;
  BATCH_TRY(cudaMemcpy(&d->sc->cur, &cur, sizeof(int), cudaMemcpyHostToDevice));
  BATCH_TRY(cudaMemcpy(&d->sc->tt, &t0, sizeof(int), cudaMemcpyHostToDevice));
  int s = -1;
  for (size_t k = 0; k < b->slots.size(); ++k)
    if (!b->slots[k].d) {
      s = (int)k;
      break;
    }
  if (s < 0) {
    s = (int)b->slots.size();
    b->slots.push_back(Slot{});
  }
  b->slots[s].d = d;
  b->slots[s].steps = 0;
  // the slot's previous occupant was released after its steps ended
  if (s < b->status_cap) b->status_host[s] = FREHD_OK;
  b->used += d->bytes;
  d->in_batch = 1;
  b->dirty = true;
  *slot = s;
  return FREHD_OK;
}

extern "C" int frehd_batch_release(frehd_batch *b, int slot, frehd_domain **out) {
  clear_error();
  if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].d)
    return fail(FREHD_ERR_INVALID, "no domain in slot %d", slot);
  BATCH_TRY(cudaSetDevice(b->device));
  BATCH_TRY(cudaStreamSynchronize(b->stream));
  frehd_domain *d = b->slots[slot].d;
  int cur = 0;
  BATCH_TRY(cudaMemcpy(&cur, &d->sc->cur, sizeof(int), cudaMemcpyDeviceToHost));
  d->cur = cur & 1;
  d->in_batch = 0;
  b->used -= d->bytes;
  b->slots[slot].d = nullptr;
  b->dirty = true;
  if (out) *out = d;
  // the last step's statistics (written by k_finish_batch) into d->last
  return domain_read_stats(d);
}

extern "C" int frehd_batch_step(frehd_batch *b) {
  if (!b) return fail(FREHD_ERR_INVALID, "null batch");
  BATCH_TRY(cudaSetDevice(b->device));
  if (b->dirty) {
    const int rc = rebuild(b);
    if (rc) return rc;
  }
  if (b->nfin == 0) return FREHD_OK;
  capture(b);
  if (b->graph_live) {
    BATCH_TRY(cudaGraphLaunch(b->graph, b->stream));
  } else {
    const int rc = launch_step(b);
    if (rc) return rc;
  }
  for (Slot &s : b->slots)
    if (s.d) ++s.steps;
  ++b->steps;
  return FREHD_OK;
}

extern "C" int frehd_batch_sync(frehd_batch *b) {
  if (!b) return fail(FREHD_ERR_INVALID, "null batch");
  BATCH_TRY(cudaSetDevice(b->device));
  BATCH_TRY(cudaStreamSynchronize(b->stream));
  return FREHD_OK;
}

extern "C" int frehd_batch_info(frehd_batch *b, frehd_batch_info_t *out) {
  if (!b || !out) return fail(FREHD_ERR_INVALID, "null argument");
  if (b->dirty) {
    BATCH_TRY(cudaSetDevice(b->device));
    const int rc = rebuild(b);
    if (rc) return rc;
  }
  int n = 0;
  for (const Slot &s : b->slots) n += s.d != nullptr;
  out->domains = n;
  out->cg_ctas = b->nctas;
  out->cg_capacity = b->packing == FREHD_BATCH_TILE_LIST ? b->capacity_tiles : b->capacity;
  out->tiles = b->ntiles;
  out->graph = b->graph_live;
  out->bytes_used = b->used;
  out->bytes_budget = b->budget;
  out->steps = b->steps;
  return FREHD_OK;
}

extern "C" int frehd_batch_stream(frehd_batch *b, void **stream) {
  if (!b || !stream) return fail(FREHD_ERR_INVALID, "null argument");
  *stream = b->stream;
  return FREHD_OK;
}

extern "C" int frehd_batch_set_cg_packing(frehd_batch *b, int packing) {
  if (!b || (packing != FREHD_BATCH_TILE_LIST && packing != FREHD_BATCH_CTA_GROUPS))
    return fail(FREHD_ERR_INVALID, "bad argument");
  BATCH_TRY(cudaSetDevice(b->device));
  BATCH_TRY(cudaStreamSynchronize(b->stream));  // queued steps use the current tables
  if (packing == FREHD_BATCH_CTA_GROUPS && b->packing != packing) {
    b->packing = packing;
    if (ctas_needed(b, nullptr) > b->capacity) {
      b->packing = FREHD_BATCH_TILE_LIST;
      return fail(FREHD_ERR_NOMEM, "batch CTA capacity: the admitted domains need %d CTAs in groups",
                  ctas_needed(b, nullptr));
    }
  }
  b->packing = packing;
  b->dirty = true;
  return FREHD_OK;
}

extern "C" int frehd_batch_set_stencil_tiles(frehd_batch *b, int tiles_per_block) {
  if (!b || tiles_per_block < 1 || tiles_per_block > kMaxTilesPerBlock)
    return fail(FREHD_ERR_INVALID, "bad argument");
  BATCH_TRY(cudaSetDevice(b->device));
  BATCH_TRY(cudaStreamSynchronize(b->stream));  // queued steps use the current tables
  b->tiles_per_block = tiles_per_block;
  b->dirty = true;
  return FREHD_OK;
}

extern "C" int frehd_batch_set_graph(frehd_batch *b, int on) {
  if (!b) return fail(FREHD_ERR_INVALID, "null batch");
  drop_graph(b);
  b->use_graph = on ? 1 : 0;
  return FREHD_OK;
}

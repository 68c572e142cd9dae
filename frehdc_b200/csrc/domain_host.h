// Host-side state of one domain, shared by the single-domain C ABI (capi.cu)
// and the batch engine (batch.cu).
#ifndef FREHD_DOMAIN_HOST_H
#define FREHD_DOMAIN_HOST_H

#include <cuda_runtime.h>

#include <vector>

#include "cg1.h"
#include "domain.cuh"
#include "frehd_b200.h"
#include "kernels.cuh"

struct frehd_domain {
  frehd_config cfg;
  int device = 0;
  cudaStream_t stream = nullptr;
  frehd::Grid gr;
  frehd::Params p;
  long N = 0, T = 0;
  double *surf[2] = {}, *depth[2] = {}, *S[2] = {};
  double *Tr[FREHD_MAX_SCALARS - 1][2] = {};  // tracers 1 .. nscalar-1 (both halves)
  int *ind[2] = {};
  double *u = nullptr, *v = nullptr, *CDXP = nullptr, *CDYP = nullptr, *CFLx = nullptr,
         *CFLy = nullptr;
  double *V = nullptr, *Z = nullptr, *Nx = nullptr, *Oy = nullptr, *Vx = nullptr, *Vy = nullptr,
         *Zx = nullptr, *Zy = nullptr;
  double *bottomZ = nullptr, *bottomXP = nullptr, *bottomYP = nullptr;
  double *EnXP = nullptr, *EnYP = nullptr, *Gx = nullptr, *Gy = nullptr, *Ct = nullptr,
         *b = nullptr;
  double *Hx = nullptr, *Hy = nullptr;
  float *fr0 = nullptr, *fr1 = nullptr, *fp0 = nullptr, *fp1 = nullptr, *fd = nullptr,
        *fhx = nullptr, *fhy = nullptr, *fs = nullptr;  // mixed-precision CG (allocated when enabled)
  double *x = nullptr, *r = nullptr, *p0 = nullptr, *p1 = nullptr, *q = nullptr;
  double *cellV = nullptr, *Sm = nullptr, *Fuu = nullptr, *Fvv = nullptr;
  unsigned char *rmv = nullptr;
  int *fix_list = nullptr;
  double *partials = nullptr;
  long npartials = 0;
  double *tide = nullptr;
  int ntide = 0;
  double *inflow = nullptr, *wspd = nullptr, *wcos = nullptr, *wsin = nullptr;
  int ninflow = 0, nwspd = 0, nwdir = 0;
  double *dXP = nullptr, *dYP = nullptr;  // face depths read by the wind term
  double *tables = nullptr, *zf = nullptr;
  double *lvc = nullptr;  // level-value cache (fine geometry), 20 planes
  int *lvi = nullptr;     // its level indices, 2 planes
  long long zf_bytes = 0, lvc_bytes = 0, tables_bytes = 0;
  frehd::Scratch *sc = nullptr;
  frehd::StepOut *out = nullptr;
  frehd::StepOut *out_host = nullptr;  // pinned
  double *stage = nullptr;      // device staging, T doubles
  double *stage2 = nullptr;
  int cur = 0;
  int x0_mode = FREHD_X0_ZERO;
  int cg_blocks = 1;
  int cg_schedule = FREHD_CG_SINGLE_SWEEP;
  int eliminate = 0;  // FREHD_DECOUPLED_ELIMINATED selected
  frehd::Cg1Maps cg1_maps{};
  frehd::Cg1Maps *cg1_maps_dev = nullptr;  // device copy read by the kernel
  int cg1_blocks_n = 1;
  int geom_set = 0, ready = 0;
  frehd_step_stats last{};
  std::vector<void *> allocs;
  long long bytes = 0;    // device memory held (footprint)
  int in_batch = 0;       // stepped by a frehd_batch: its parity lives in sc->cur
  // profiling: one event before each kernel of a step plus one after
  int profiling = 0;
  std::vector<cudaEvent_t> ev;
  frehd_kernel_times times{};
  long long iters_at_prof_start = 0;
  long long noconv_seen = 0;  // steps stopped at maxIter already reported to the caller
};

namespace frehd {
// The kernels' view of domain d with the ping-pong half `cur` as current.
View domain_view(const frehd_domain *d, int cur);
// Read the last step's statistics (StepOut) into d->last; synchronises d->stream.
int domain_read_stats(frehd_domain *d);
// Steps whose solve stopped at maxIter since the last call (from the statistics
// last read); the count is then marked as reported.
long long domain_take_noconv(frehd_domain *d);
}  // namespace frehd

struct frehd_batch;
namespace frehd {
// Device status of the domain in `slot` after the latest completed batch step
// (FREHD_OK while it steps normally); valid once the caller has waited for
// that step.
int batch_slot_status(const frehd_batch *b, int slot);
}  // namespace frehd

#endif

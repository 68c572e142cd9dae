// Status strings, per-thread last-error text and the Config defaults.
#include <cstring>

#include "frehd_internal.h"

namespace {
thread_local char g_last_error[512] = {0};
}

namespace frehd {

int fail(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return code;
}

void clear_error() { g_last_error[0] = 0; }

}  // namespace frehd

extern "C" const char *frehd_last_error(void) { return g_last_error; }

extern "C" const char *frehd_version(void) { return "frehd_b200 0.1 (sm_100a)"; }

extern "C" const char *frehd_status_string(int status) {
  switch (status) {
    case FREHD_OK: return "ok";
    case FREHD_ERR_INVALID: return "invalid argument";
    case FREHD_ERR_UNSUPPORTED: return "unsupported configuration option";
    case FREHD_ERR_CUDA: return "CUDA runtime error";
    case FREHD_ERR_NOMEM: return "device out of memory";
    case FREHD_ERR_CG_NOCONVERGE: return "CG did not converge within maxIter";
    case FREHD_ERR_CFL: return "max CFL exceeds 20";
    case FREHD_ERR_TIMEOUT: return "bounded device wait timed out";
    case FREHD_ERR_STATE: return "call out of order";
    default: return "unknown status";
  }
}

// Values of the shipped data.dat (frehdc5+/data.dat:8-102) for the fields the
// step reads; grid size, geometry and tide placement are the caller's to set.
extern "C" void frehd_config_defaults(frehd_config *c) {
  std::memset(c, 0, sizeof(*c));
  c->nx = c->ny = 0;
  c->dx = c->dy = 16.0;
  c->dt = 2.0;
  c->g = 9.8066;
  c->NUx = c->NUy = 1e-4;
  c->Kx = c->Ky = 1e-4;
  c->CDx = c->CDy = 0.01;
  c->manningN = 0.03;
  c->CDmax = 1.0;
  c->hD = 0.1;
  c->CwT = 10.0;
  c->CDnotN = 0;
  c->useThinLayer = 1;
  c->useSubgrid = 1;
  c->useSubDrag = 0;
  c->staggeredV = 1;
  c->useminA = 0;
  c->useminV = 3;
  c->dxf = c->dyf = 1.0;
  c->subR = 16.0;
  c->surfmin = 0.25;
  c->surfmax = 0.75;
  c->dsurf = 0.01;
  c->bcType = 1;
  c->tideLocFirstP = 0;
  c->tideLocLengthP = 0;
  c->useScalar = 1;
  c->scalarAdv = 1;
  c->useConstTidePS = 1;
  c->tidePS = 20.0;
  c->minDepth = 1e-5;
  c->wtfh = 1e-5;
  c->CFLl = 0.5;
  c->CFLh = 0.7;
  c->eps = 1e-8;
  c->maxIter = 10000000;
  c->offset = 0.0;
  c->inflowI0 = c->inflowI1 = c->inflowJ0 = c->inflowJ1 = 0;
  c->inflowS = 0.0;
  c->northAngle = 0.0;
  c->rhoa = 1.25;
  c->Cw = 0.0013;
  c->nscalar = 1;
}

/*
 * nssolve_b200.c -- replacement of the reference's nssolve.c
 * (frehdc5+/nssolve.c) that runs the time steps on a B200 through the
 * frehd_b200 C ABI.  Linked with the reference's own FREHD.c main and every
 * other reference translation unit unchanged, it turns the reference program
 * into the device-stepped program: same input deck, same output files.
 *
 * What stays on the host, in the reference's code: reading the deck, Init,
 * DataOutput/SubOutput, and monitorCFL's reporting and exit.  What moves to the
 * device: oneCompleteStep and the CFL maxima of monitorCFL
 * (frehd_domain_run).  The host arrays are refreshed from the device only
 * where the host reads them: before each DataOutput (tt % OutItvl == 0,
 * nssolve.c:91), before a CFL exit, and once after the last step.
 *
 * DataOutput subtracts and re-adds the bathymetry offset to the interior
 * surface in place (fileio.c:65-66,120-121), which can move the last bit; the
 * reference's next step starts from those doubles, so after each output the
 * surface is copied back to the device.
 *
 * Environment (all optional):
 *   FREHD_DEVICE        CUDA device ordinal (default 0)
 *   FREHD_PRECISION     "fp64" (default) or "mixed" (FP32 inner CG iterations
 *                       inside FP64 refinement, frehd_domain_set_precision)
 *   FREHD_EPS_INNER     inner tolerance of the mixed form (default 1e-5)
 *   FREHD_HOST_MONITOR  1: run monitorCFL on the host after every step, which
 *                       prints the reference's per-cell warnings (copies the
 *                       velocities back every step); otherwise one summary line
 *                       per device run when a cell exceeded CFL 2
 *   FREHD_CHUNK         most steps per device run between host checks (1000)
 *   FREHD_DEVICE_OUTPUT 1: write the output files from the device
 *                       (frehd_domain_write_output: the same bytes, formatted on
 *                       the GPU) instead of copying the state back for the
 *                       reference's DataOutput/SubOutput
 *   FREHD_DUMP          path: after the last step, write the final state in
 *                       full precision (FRHDDUMP: "FRHDDUMP", int32 version 1,
 *                       int32 count, then per array char name[24], int64 n,
 *                       int32 type 0 double / 1 int32, int32 pad, data); a
 *                       path holding one "%d" is a pattern, written after every
 *                       output step's DataOutput and after the last step with
 *                       the step number substituted
 */
#define _GNU_SOURCE
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "bathymetry.h"
#include "configuration.h"
#include "fileio.h"
#include "initialize.h"
#include "map.h"
#include "nsfunctions.h"
#include "nssolve.h"
#include "subgrid.h"

#include "frehd_b200.h"
#include "frehd_dropin.h"

static frehd_domain *g_dom = NULL;
static int g_status = FREHD_OK;
static int g_nx, g_ny;
static long g_N, g_T;

static int note(int rc) {
  g_status = rc;
  return rc;
}

static void die(const char *what, int rc) {
  fprintf(stderr, "frehd_b200: %s failed: %s (%s)\n", what, frehd_status_string(rc),
          frehd_last_error());
  exit(EXIT_FAILURE);
}

static double wall(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static int env_int(const char *name, int dflt) {
  const char *s = getenv(name);
  return (s && *s) ? atoi(s) : dflt;
}

/* Config (configuration.h:4-111) -> frehd_config.  The tidal cells are the
 * contiguous run tideLocP[k] = first + k + nx*(ny-1) (configuration.c:147-148). */
static int make_config(const Config *s, const Bath *bath, frehd_config *c) {
  frehd_config_defaults(c);
  c->nx = s->nx;
  c->ny = s->ny;
  c->dx = s->dx;
  c->dy = s->dy;
  c->dt = s->dt;
  c->g = s->g;
  c->NUx = s->NUx;
  c->NUy = s->NUy;
  c->Kx = s->Kx;
  c->Ky = s->Ky;
  c->CDx = s->CDx;
  c->CDy = s->CDy;
  c->manningN = s->manningN;
  c->CDmax = s->CDmax;
  c->hD = s->hD;
  c->CwT = s->CwT;
  c->CDnotN = s->CDnotN;
  c->useThinLayer = s->useThinLayer;
  c->useSubgrid = s->useSubgrid;
  c->useSubDrag = s->useSubDrag;
  c->staggeredV = s->staggeredV;
  c->useminA = s->useminA;
  c->useminV = s->useminV;
  c->dxf = s->dxf;
  c->dyf = s->dyf;
  c->subR = s->subR;
  c->surfmin = s->surfmin;
  c->surfmax = s->surfmax;
  c->dsurf = s->dsurf;
  c->bcType = s->bcType;
  c->tideLocLengthP = s->tideLocLengthP;
  c->tideLocFirstP = 0;
  if (s->tideLocLengthP > 0) {
    const int row = s->nx * (s->ny - 1);
    c->tideLocFirstP = s->tideLocP[0] - row;
    for (int k = 1; k < s->tideLocLengthP; ++k)
      if (s->tideLocP[k] != s->tideLocP[0] + k) {
        fprintf(stderr, "frehd_b200: tidal cells must be one contiguous run of the north row\n");
        return FREHD_ERR_UNSUPPORTED;
      }
  }
  c->useScalar = s->useScalar;
  c->scalarAdv = s->scalarAdv;
  c->useConstTidePS = s->useConstTidePS;
  c->tidePS = s->tidePS;
  c->useWind = s->useWind;
  c->useEvap = s->useEvap;
  c->useRain = s->useRain;
  c->inflowLocLength = s->inflowLocLength;
  /* inflow cells: the rectangle configuration.c:53-60 lists (i-index minus one
   * in its loop) */
  if (s->inflowLocLength > 0) {
    int i0 = s->nx, i1 = -1, j0 = s->ny, j1 = -1;
    for (int k = 0; k < s->inflowLocLength; ++k) {
      const int i = s->inflowLoc[k] % s->nx, j = s->inflowLoc[k] / s->nx;
      if (s->inflowLoc[k] < 0 || j >= s->ny) {
        fprintf(stderr, "frehd_b200: inflow cell %d outside the domain\n", s->inflowLoc[k]);
        return FREHD_ERR_UNSUPPORTED;
      }
      if (i < i0) i0 = i;
      if (i > i1) i1 = i;
      if (j < j0) j0 = j;
      if (j > j1) j1 = j;
    }
    c->inflowI0 = i0;
    c->inflowI1 = i1 + 1;
    c->inflowJ0 = j0;
    c->inflowJ1 = j1 + 1;
    if ((long)(i1 + 1 - i0) * (j1 + 1 - j0) != s->inflowLocLength) {
      fprintf(stderr, "frehd_b200: inflow cells must form a rectangle\n");
      return FREHD_ERR_UNSUPPORTED;
    }
  }
  c->inflowS = s->inflowS;
  c->northAngle = s->northAngle;
  c->rhoa = s->rhoa;
  c->Cw = s->Cw;
  c->useSubStep = s->useSubStep;
  c->checkConservation = s->checkConservation;
  c->minDepth = s->minDepth;
  c->wtfh = s->wtfh;
  c->CFLl = s->CFLl;
  c->CFLh = s->CFLh;
  c->eps = s->eps;
  c->maxIter = s->maxIter;
  c->offset = bath->offset[0];
  return FREHD_OK;
}

/* The persistent state the step reads (the arrays the reference's step carries
 * from one step to the next). */
static void persistent_fields(frehd_state *st, Data *data, Sub *sub) {
  memset(st, 0, sizeof(*st));
  st->surf = data->surf;
  st->uuXP = data->uuXP;
  st->vvYP = data->vvYP;
  st->S = data->S;
  st->depth = data->depth;
  st->CDXP = data->CDXP;
  st->CDYP = data->CDYP;
  st->CFLx = data->CFLx;
  st->CFLy = data->CFLy;
  st->V = sub->V;
  st->Z = sub->Z;
  st->Nx = sub->Nx;
  st->Oy = sub->Oy;
  st->Vx = sub->Vx;
  st->Vy = sub->Vy;
  st->Zx = sub->Zx;
  st->Zy = sub->Zy;
  st->ind = sub->ind;
  st->depthXP = data->depthXP;  /* read by the wind term; held only with useWind */
  st->depthYP = data->depthYP;
}

int frehd_gpu_init(Data *data, Sub *sub, Bath *bath, BC *bc, Config *setting, int device) {
  if (!data || !sub || !bath || !bc || !setting) return note(FREHD_ERR_INVALID);
  if (g_dom) frehd_gpu_finalize();
  frehd_config c;
  int rc = make_config(setting, bath, &c);
  if (rc) return note(rc);
  rc = frehd_domain_create(&c, device, &g_dom);
  if (rc) return note(rc);
  g_nx = setting->nx;
  g_ny = setting->ny;
  g_N = (long)setting->N2ci;
  g_T = (long)setting->N2ct;
  /* the reference's level tables, packed in frehd_build_tables' order */
  const int Ne = sub->Ne;
  const size_t per = (size_t)Ne * (size_t)g_N;
  const double *src[10] = {sub->allV,  sub->allZ,  sub->allVxp, sub->allVxm, sub->allVyp,
                           sub->allVym, sub->allNp, sub->allNm,  sub->allOp,  sub->allOm};
  double *tables = (double *)malloc(10 * per * sizeof(double));
  if (!tables) return note(FREHD_ERR_NOMEM);
  for (int t = 0; t < 10; ++t) memcpy(tables + t * per, src[t], per * sizeof(double));
  rc = frehd_domain_set_tables(g_dom, Ne, tables);
  free(tables);
  if (rc) return note(rc);
  rc = frehd_domain_set_tide(g_dom, setting->Nt, bc->tideP);
  if (rc) return note(rc);
  /* readBC (initialize.c:345-378) loads inflow always, the wind only with useWind */
  rc = frehd_domain_set_series(g_dom, FREHD_SERIES_INFLOW, setting->Nt, bc->inflow);
  if (!rc && setting->useWind == 1)
    rc = frehd_domain_set_series(g_dom, FREHD_SERIES_WIND_SPEED, setting->Nt, bc->windspd);
  if (!rc && setting->useWind == 1)
    rc = frehd_domain_set_series(g_dom, FREHD_SERIES_WIND_DIR, setting->Nt, bc->winddir);
  if (rc) return note(rc);
  const char *prec = getenv("FREHD_PRECISION");
  if (prec && !strcmp(prec, "mixed")) {
    const char *e = getenv("FREHD_EPS_INNER");
    rc = frehd_domain_set_precision(g_dom, FREHD_PRECISION_MIXED, (e && *e) ? atof(e) : 1e-5);
    if (rc) return note(rc);
  } else if (prec && *prec && strcmp(prec, "fp64")) {
    fprintf(stderr, "frehd_b200: FREHD_PRECISION must be fp64 or mixed\n");
    return note(FREHD_ERR_INVALID);
  }
  frehd_state st;
  persistent_fields(&st, data, sub);
  st.bottomZ = bath->bottomZ;
  st.bottomXP = bath->bottomXP;
  st.bottomYP = bath->bottomYP;
  return note(frehd_domain_upload_state(g_dom, &st));
}

int frehd_gpu_run(int t0, int nsteps) {
  if (!g_dom) return note(FREHD_ERR_STATE);
  return note(frehd_domain_run(g_dom, t0, nsteps));
}

int frehd_gpu_step(int tt) { return frehd_gpu_run(tt, 1); }

int frehd_gpu_sync_to_host(Data *data, Sub *sub) {
  if (!g_dom) return note(FREHD_ERR_STATE);
  if (!data || !sub) return note(FREHD_ERR_INVALID);
  frehd_state st;
  persistent_fields(&st, data, sub);
  st.surfOld = data->surfOld;
  st.uuYP = data->uuYP;
  st.vvXP = data->vvXP;
  st.EnXP = data->EnXP;
  st.EnYP = data->EnYP;
  st.cellV = data->cellV;
  st.Sm = data->Sm;
  st.Fuu = data->Fuu;
  st.Fvv = data->Fvv;
  return note(frehd_domain_download_state(g_dom, &st));
}

int frehd_gpu_sync_from_host(Data *data, Sub *sub) {
  if (!g_dom) return note(FREHD_ERR_STATE);
  if (!data || !sub) return note(FREHD_ERR_INVALID);
  frehd_state st;
  persistent_fields(&st, data, sub);
  return note(frehd_domain_upload_state(g_dom, &st));
}

int frehd_gpu_last_step(void) {
  frehd_step_stats s;
  if (!g_dom || frehd_domain_stats(g_dom, &s)) return 0;
  return s.step;
}

int frehd_gpu_status(void) { return g_status; }

frehd_domain *frehd_gpu_domain(void) { return g_dom; }

int frehd_gpu_finalize(void) {
  int rc = FREHD_OK;
  if (g_dom) rc = frehd_domain_destroy(g_dom);
  g_dom = NULL;
  return note(rc);
}

/* ------------------------------------------------------------ final-state dump */
static void dump_arr(FILE *f, int *count, const char *name, const void *p, long n, int type) {
  if (!p) return;
  char nm[24];
  memset(nm, 0, sizeof(nm));
  strncpy(nm, name, sizeof(nm) - 1);
  int64_t nn = n;
  int32_t ty = type, pad = 0;
  fwrite(nm, 1, 24, f);
  fwrite(&nn, 8, 1, f);
  fwrite(&ty, 4, 1, f);
  fwrite(&pad, 4, 1, f);
  fwrite(p, type == 0 ? 8 : 4, (size_t)n, f);
  ++*count;
}

static void dump_step(const char *pattern, Data *data, Sub *sub, Config *setting, int tt) {
  char path[4096];
  const char *pc = strstr(pattern, "%d");
  if (pc && strlen(pattern) < sizeof(path) - 16)
    snprintf(path, sizeof(path), "%.*s%d%s", (int)(pc - pattern), pattern, tt, pc + 2);
  else
    snprintf(path, sizeof(path), "%s", pattern);
  FILE *f = fopen(path, "wb");
  if (!f) {
    fprintf(stderr, "frehd_b200: cannot write %s\n", path);
    exit(EXIT_FAILURE);
  }
  fwrite("FRHDDUMP", 1, 8, f);
  int32_t ver = 1, count = 0;
  fwrite(&ver, 4, 1, f);
  long count_pos = ftell(f);
  fwrite(&count, 4, 1, f);
  const long N = g_N, T = g_T;
  int32_t meta[8] = {setting->nx, setting->ny, sub->Ne, setting->Nt, tt, 0, 0, 0};
  frehd_step_stats s;
  if (!frehd_domain_stats(g_dom, &s)) meta[5] = s.cg_iters;
  int c = 0;
  dump_arr(f, &c, "meta", meta, 8, 1);
  dump_arr(f, &c, "surf", data->surf, T, 0);
  dump_arr(f, &c, "surfOld", data->surfOld, T, 0);
  dump_arr(f, &c, "uuXP", data->uuXP, T, 0);
  dump_arr(f, &c, "vvYP", data->vvYP, T, 0);
  dump_arr(f, &c, "uuYP", data->uuYP, N, 0);
  dump_arr(f, &c, "vvXP", data->vvXP, N, 0);
  dump_arr(f, &c, "depth", data->depth, N, 0);
  dump_arr(f, &c, "EnXP", data->EnXP, T, 0);
  dump_arr(f, &c, "EnYP", data->EnYP, T, 0);
  dump_arr(f, &c, "CDXP", data->CDXP, T, 0);
  dump_arr(f, &c, "CDYP", data->CDYP, T, 0);
  dump_arr(f, &c, "S", data->S, T, 0);
  dump_arr(f, &c, "Sm", data->Sm, N, 0);
  dump_arr(f, &c, "cellV", data->cellV, N, 0);
  dump_arr(f, &c, "Fuu", data->Fuu, T, 0);
  dump_arr(f, &c, "Fvv", data->Fvv, T, 0);
  dump_arr(f, &c, "CFLx", data->CFLx, T, 0);
  dump_arr(f, &c, "CFLy", data->CFLy, T, 0);
  dump_arr(f, &c, "V", sub->V, T, 0);
  dump_arr(f, &c, "Z", sub->Z, T, 0);
  dump_arr(f, &c, "Nx", sub->Nx, T, 0);
  dump_arr(f, &c, "Oy", sub->Oy, T, 0);
  dump_arr(f, &c, "Vx", sub->Vx, T, 0);
  dump_arr(f, &c, "Vy", sub->Vy, T, 0);
  dump_arr(f, &c, "Zx", sub->Zx, T, 0);
  dump_arr(f, &c, "Zy", sub->Zy, T, 0);
  dump_arr(f, &c, "ind", sub->ind, T, 1);
  count = c;
  fseek(f, count_pos, SEEK_SET);
  fwrite(&count, 4, 1, f);
  fclose(f);
}

/* The files DataOutput and SubOutput write for these settings (fileio.c:100-121,
 * 145-153; SubOutput is called only in subgrid mode, nssolve.c:92). */
static int output_fields(const Config *s) {
  int f = 0;
  if (s->saveuu == 1) f |= FREHD_OUT_U;
  if (s->savevv == 1) f |= FREHD_OUT_V;
  if (s->savesurface == 1) f |= FREHD_OUT_SURFACE;
  if (s->savedepth == 1) f |= FREHD_OUT_DEPTH;
  if (s->saveCD == 1) f |= FREHD_OUT_CD;
  if (s->useScalar == 1 && s->savescalar == 1) f |= FREHD_OUT_SCALAR;
  if (s->useSubgrid != 0 && s->savesub == 1) f |= FREHD_OUT_SUB;
  return f;
}

/* ------------------------------------------------------------ nssolve.h entry points */

/* The time loop (nssolve.c:48-107).  Steps run on the device in runs that end
 * at each output step; the host's Data/Sub arrays are refreshed before every
 * DataOutput and after the last step. */
void SolveAll(Data **data, Sub **sub, Maps *map, BC *bc, Bath *bath, Config *setting, int irank,
              int nrank) {
  (void)map;
  const int root = 0;
  DataOutput(data, bath, setting, 0, root, irank);
  if (setting->useSubgrid != 0) SubOutput(sub, setting, 0, root, irank);
  if (setting->useMPI == 1 || nrank != 1) {
    fprintf(stderr, "frehd_b200: useMPI = 1 is not supported (one domain per process and GPU)\n");
    exit(EXIT_FAILURE);
  }
  int rc = frehd_gpu_init(*data, *sub, bath, bc, setting, env_int("FREHD_DEVICE", 0));
  if (rc) die("frehd_gpu_init", rc);
  const int host_monitor = env_int("FREHD_HOST_MONITOR", 0);
  int chunk = env_int("FREHD_CHUNK", 1000);
  if (chunk < 1) chunk = 1;
  const int itvl = setting->OutItvl;
  const char *dump = getenv("FREHD_DUMP");
  if (dump && !*dump) dump = NULL;
  const int dump_every = dump && strstr(dump, "%d") != NULL;
  /* vloss (checkConservation) has no device counterpart: the host writes then */
  const int device_output = env_int("FREHD_DEVICE_OUTPUT", 0) && setting->checkConservation != 1;
  if (irank == 0) printf("Ready for time stepping ...\n");
  int tt = 1;
  while (tt <= setting->Nt) {
    int last = setting->Nt;
    if (itvl > 0) {
      const int next_out = ((tt + itvl - 1) / itvl) * itvl;
      if (next_out < last) last = next_out;
    }
    if (last - tt + 1 > chunk) last = tt + chunk - 1;
    if (host_monitor) last = tt;
    const double t0 = wall();
    rc = frehd_gpu_run(tt, last - tt + 1);
    const double el = wall() - t0;
    frehd_step_stats s;
    if (rc == FREHD_ERR_CFL) {
      /* the device stopped after step s.step, where the reference's monitorCFL
       * writes the state and exits (nsfunctions.c:1225-1231): run it on the
       * host copy of that state */
      frehd_domain_stats(g_dom, &s);
      rc = frehd_gpu_sync_to_host(*data, *sub);
      if (rc) die("frehd_gpu_sync_to_host", rc);
      monitorCFL(data, bath, irank, setting, s.step, root);
      exit(EXIT_FAILURE);
    }
    if (rc == FREHD_ERR_CG_NOCONVERGE) {
      /* laspack stops at maxIter without an error either (itersolv.c:355-456) */
      fprintf(stderr, "frehd_b200: WARNING: CG reached maxIter at a step of %d..%d\n", tt, last);
    } else if (rc) {
      die("frehd_gpu_run", rc);
    }
    rc = frehd_domain_stats(g_dom, &s);
    if (rc) die("frehd_domain_stats", rc);
    if (host_monitor) {
      frehd_state st;
      memset(&st, 0, sizeof(st));
      st.uuXP = (*data)->uuXP;
      st.vvYP = (*data)->vvYP;
      rc = frehd_domain_download_state(g_dom, &st);
      if (rc) die("frehd_domain_download_state", rc);
      monitorCFL(data, bath, irank, setting, tt, root);
    } else if (s.n_cfl_warn > 0 && irank == 0) {
      printf("WARNING: %d cells with CFL > 2 at step %d (max CFL x %lf, y %lf)\n", s.n_cfl_warn,
             s.step, s.max_cflx, s.max_cfly);
    }
    if (itvl > 0 && last % itvl == 0 && device_output) {
      rc = frehd_domain_write_output(g_dom, setting->saveFolder, last, output_fields(setting));
      if (rc) die("frehd_domain_write_output", rc);
      if (dump_every) {
        rc = frehd_gpu_sync_to_host(*data, *sub);
        if (rc) die("frehd_gpu_sync_to_host", rc);
        dump_step(dump, *data, *sub, setting, last);
      }
    } else if (itvl > 0 && last % itvl == 0) {
      rc = frehd_gpu_sync_to_host(*data, *sub);
      if (rc) die("frehd_gpu_sync_to_host", rc);
      DataOutput(data, bath, setting, last, root, irank);
      if (setting->useSubgrid != 0) SubOutput(sub, setting, last, root, irank);
      if (dump_every) dump_step(dump, *data, *sub, setting, last);
      frehd_state st;
      memset(&st, 0, sizeof(st));
      st.surf = (*data)->surf;
      rc = frehd_domain_upload_state(g_dom, &st);
      if (rc) die("frehd_domain_upload_state", rc);
    }
    if (irank == 0) {
      if (last == tt)
        printf("---------- Step %d executed with time %.4f sec... ----------\n", tt, el);
      else
        printf("---------- Steps %d-%d executed with time %.4f sec (%.6f per step)... ----------\n",
               tt, last, el, el / (last - tt + 1));
    }
    tt = last + 1;
  }
  rc = frehd_gpu_sync_to_host(*data, *sub);
  if (rc) die("frehd_gpu_sync_to_host", rc);
  if (dump) dump_step(dump, *data, *sub, setting, setting->Nt);
  if (irank == 0) printf("Time stepping completed...\n");
  frehd_gpu_finalize();
}

/* A caller-driven step uploads the host's persistent state, so the host arrays
 * stay the source of truth between calls (a caller may edit them, and
 * DataOutput does), and the first call creates the domain. */
static void ensure_domain_with_host_state(Data **data, Sub **sub, BC *bc, Bath *bath,
                                          Config *setting) {
  int rc;
  if (!g_dom) {
    rc = frehd_gpu_init(*data, *sub, bath, bc, setting, env_int("FREHD_DEVICE", 0));
    if (rc) die("frehd_gpu_init", rc);
  } else {
    rc = frehd_gpu_sync_from_host(*data, *sub);
    if (rc) die("frehd_gpu_sync_from_host", rc);
  }
}

/* One complete step (nssolve.c:110-118): host state in, host state out.  The
 * caller's monitorCFL then reads the stepped velocities as in the reference.
 * A, x and z (the caller's laspack objects) are not used: the system is
 * assembled and solved on the device. */
void oneCompleteStep(Data **data, Sub **sub, Maps *map, BC *bc, Bath *bath, Config *setting, int tt,
                     QMatrix A, Vector x, Vector z, int irank, int nrank) {
  (void)map; (void)A; (void)x; (void)z; (void)irank; (void)nrank;
  ensure_domain_with_host_state(data, sub, bc, bath, setting);
  int rc = frehd_gpu_run(tt, 1);
  /* CFL > 20 is reported by the caller's own monitorCFL; CG at maxIter goes on
   * as in laspack */
  if (rc && rc != FREHD_ERR_CFL && rc != FREHD_ERR_CG_NOCONVERGE) die("frehd_gpu_run", rc);
  rc = frehd_gpu_sync_to_host(*data, *sub);
  if (rc) die("frehd_gpu_sync_to_host", rc);
}

/* The three parts of a step map onto the device phases of frehd_domain_phase:
 * the explicit terms with the matrix assembly, the solve, and everything from
 * getFreeSurface on (including scalarTransport).  Only the last one copies the
 * state back to the host. */
void solveSourceTerm(Data **data, Sub *sub, Maps *map, BC *bc, Bath *bath, Config *setting, int tt,
                     int irank, int nrank) {
  (void)map; (void)irank; (void)nrank;
  Sub *s = sub;
  ensure_domain_with_host_state(data, &s, bc, bath, setting);
  int rc = frehd_domain_phase(g_dom, FREHD_PHASE_EXPLICIT, tt, NULL);
  if (rc) die("frehd_domain_phase(explicit)", rc);
}

void solveFreeSurface(Data **data, Sub *sub, Maps *map, BC *bc, Bath *bath, Config *setting, int tt,
                      QMatrix A, Vector x, Vector z, int irank, int nrank) {
  (void)data; (void)sub; (void)map; (void)bc; (void)bath; (void)setting;
  (void)A; (void)x; (void)z; (void)irank; (void)nrank;
  if (!g_dom) die("solveFreeSurface before solveSourceTerm", FREHD_ERR_STATE);
  int rc = frehd_domain_phase(g_dom, FREHD_PHASE_SOLVE, tt, NULL);
  if (rc && rc != FREHD_ERR_CG_NOCONVERGE) die("frehd_domain_phase(solve)", rc);
}

void updateData(Data **data, Sub **sub, Maps *map, BC *bc, Bath *bath, Config *setting, int tt,
                int irank, int nrank) {
  (void)map; (void)bc; (void)bath; (void)setting; (void)irank; (void)nrank;
  if (!g_dom) die("updateData before solveSourceTerm", FREHD_ERR_STATE);
  int rc = frehd_domain_phase(g_dom, FREHD_PHASE_UPDATE, tt, NULL);
  if (rc && rc != FREHD_ERR_CFL) die("frehd_domain_phase(update)", rc);
  rc = frehd_gpu_sync_to_host(*data, *sub);
  if (rc) die("frehd_gpu_sync_to_host", rc);
}

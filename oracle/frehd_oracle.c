/*
 * frehd_oracle.c -- CPU restatement of one FrehdC time step (subgrid path),
 * written from the reference's algorithm, for use as a test oracle only.
 *
 * TEST INFRASTRUCTURE: only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg may load this library.  The product path (the CUDA library)
 * never calls it.
 *
 * Parity: pinned against the reference itself.  oracle/ref builds the unchanged
 * reference sources into oracle/_ref/frehd_ref, whose phase dumps the tests
 * compare with this restatement array by array (bit for bit outside the linear
 * solve; the solve to the CG tolerance).
 *
 * Layout is the reference's own (map.c:45-127): interior ii = j*nx + i, the
 * ghost ring appended after N = nx*ny.  Reads the reference makes outside an
 * array (depth and edgeX/edgeY at ghost indices, velocityInterp's index - 1 and
 * index - nx at the domain start) are defined here as 0.0, which is what the
 * reference reads when run under the oracle's zero-guarded allocator.
 *
 * Supported Config subset (others are rejected at creation): useSubgrid = 1,
 * staggeredV = 1, useSubDrag = 0, CDnotN = 0, useminA = 0, useminV not in {1,2},
 * bcType = 1, no evaporation/rain/sub-stepping, scalarAdv = 1 or 2,
 * useConstTidePS = 1, checkConservation = 0.  Inflow cells and wind are
 * supported (their series set with oracle_set_series).
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "frehd_oracle.h"

#define NTAB 10
enum { T_V, T_Z, T_VXP, T_VXM, T_VYP, T_VYM, T_NP, T_NM, T_OP, T_OM };

struct oracle_domain {
  oracle_cfg c;
  int nx, ny;
  long N, T;
  /* maps (map.c:31-143) */
  int *iPjc, *iMjc, *icjP, *icjM, *trps, *sprt;
  int *iPPjc, *iMMjc, *icjPP, *icjMM;
  int *iPbd, *iPgt, *iMbd, *iMgt, *jPbd, *jPgt, *jMbd, *jMgt;
  int iMjP, iPjP, iPjM, iMjM;
  /* Data (initialize.h:10-21) */
  double *uuXP, *uuYP, *vvXP, *vvYP, *surf, *surfOld, *Fuu, *Fvv, *cellV;
  double *depth, *depthXP, *depthYP, *EnXP, *EnYP, *DragXP, *DragYP, *CDXP, *CDYP;
  double *GnCt, *GnXP, *GnYP, *GnXM, *GnYM, *z, *wtfXP, *wtfYP, *S, *Sm, *rmvCFL;
  double *advX, *advY, *CFLx, *CFLy;
  double Vloss[4];
  /* Sub (subgrid.h:8-29) */
  int Ne;
  double *allSurf, *tab[NTAB];
  double *V, *Z, *Vxp, *Vyp, *Vxm, *Vym, *Np, *Nm, *Op, *Om, *Nx, *Oy, *Vx, *Vy, *Zx, *Zy;
  int *ind;
  /* Bath (bathymetry.h:7-14) */
  double *bottomZ, *bottomXP, *bottomYP, *edgeX, *edgeY;
  /* BC */
  int nt;
  double *tideP;
  int ninflow, nwind, nwdir;
  double *inflow, *windspd, *winddir;  /* bc->inflow, windspd, winddir, indexed by tt */
  int tt;                              /* step of the phase being run */
  /* solver */
  int precond, x0mode, last_iters;
  double last_acc;
  double *x, *wr, *wp, *wq, *wz; /* transposed order */
  char err[256];
};

static double *dz(long n) { return (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double)); }
static int *iz(long n) { return (int *)calloc((size_t)(n > 0 ? n : 1), sizeof(int)); }

/* ------------------------------------------------------------------ maps */
/* createMaps (map.c:31-143): transposed/neighbour/ghost index maps. */
static void make_maps(oracle_domain *d) {
  const int nx = d->nx, ny = d->ny;
  const long N = d->N;
  d->iPjc = iz(N); d->iMjc = iz(N); d->icjP = iz(N); d->icjM = iz(N);
  d->trps = iz(N); d->sprt = iz(N);
  d->iPbd = iz(ny); d->iPgt = iz(ny); d->iMbd = iz(ny); d->iMgt = iz(ny);
  d->jPbd = iz(nx); d->jPgt = iz(nx); d->jMbd = iz(nx); d->jMgt = iz(nx);
  for (long k = 0; k < N; ++k) {
    d->trps[k] = (int)((k % ny) * nx + k / ny);  /* transposed k -> row-major */
    d->sprt[k] = (int)((k % nx) * ny + k / nx);  /* row-major -> transposed */
  }
  for (long ii = 0; ii < N; ++ii) {
    int i = (int)(ii % nx), j = (int)(ii / nx);
    d->icjP[ii] = j == ny - 1 ? (int)(N + i) : (int)(ii + nx);
    d->icjM[ii] = j == 0 ? (int)(N + nx + i) : (int)(ii - nx);
    d->iPjc[ii] = i == nx - 1 ? (int)(N + 2 * nx + j) : (int)(ii + 1);
    d->iMjc[ii] = i == 0 ? (int)(N + 2 * nx + ny + j) : (int)(ii - 1);
  }
  /* two-cell maps of the TVD scheme (map.c:66-77,89-97).  icjMM of the second
   * row (j = 1) is never assigned there: the first loop writes from index 2nx
   * on (and past the array's end), the second the first row.  Under the
   * zero-filled allocator of the parity build it holds 0, i.e. cell (0, 0). */
  d->iPPjc = iz(N); d->iMMjc = iz(N); d->icjPP = iz(N); d->icjMM = iz(N);
  for (long ii = 0; ii < N; ++ii) {
    int i = (int)(ii % nx), j = (int)(ii / nx);
    d->icjPP[ii] = j < ny - 1 ? d->icjP[d->icjP[ii]] : d->icjP[ii];
    d->icjMM[ii] = j >= 2 ? (int)(ii - 2 * nx) : (j == 0 ? d->icjM[ii] : 0);
    d->iPPjc[ii] = i == nx - 1 ? d->iPjc[ii] : d->iPjc[d->iPjc[ii]];
    d->iMMjc[ii] = i == 0 ? d->iMjc[ii] : d->iMjc[d->iMjc[ii]];
  }
  d->iMjP = (int)d->T - 4;
  d->iPjP = (int)d->T - 3;
  d->iPjM = (int)d->T - 2;
  d->iMjM = (int)d->T - 1;
  for (int i = 0; i < nx; ++i) {
    d->jPbd[i] = (int)(N - nx + i); d->jMbd[i] = i;
    d->jPgt[i] = (int)(N + i);      d->jMgt[i] = (int)(N + nx + i);
  }
  for (int j = 0; j < ny; ++j) {
    d->iPbd[j] = (j + 1) * nx - 1;        d->iMbd[j] = j * nx;
    d->iPgt[j] = (int)(N + 2 * nx + j);   d->iMgt[j] = (int)(N + 2 * nx + ny + j);
  }
}

/* read of an array the reference allocates with N entries, at any index */
static inline double rdN(const oracle_domain *d, const double *a, long k) {
  return (k >= 0 && k < d->N) ? a[k] : 0.0;
}
/* read of an array with N2ct entries at a raw (possibly negative) index */
static inline double rdT(const oracle_domain *d, const double *a, long k) {
  return (k >= 0 && k < d->T) ? a[k] : 0.0;
}

/* ------------------------------------------------------------------ create */
#define FAIL(...) do { snprintf(d->err, sizeof(d->err), __VA_ARGS__); return -1; } while (0)

static int check_cfg(oracle_domain *d) {
  const oracle_cfg *c = &d->c;
  if (c->nx <= 0 || c->ny <= 0) FAIL("bad grid %d x %d", c->nx, c->ny);
  if (c->useSubgrid != 1) FAIL("useSubgrid=%d unsupported", c->useSubgrid);
  if (c->staggeredV != 1) FAIL("staggeredV=%d unsupported", c->staggeredV);
  if (c->useSubDrag != 0) FAIL("useSubDrag=%d unsupported", c->useSubDrag);
  if (c->CDnotN != 0) FAIL("CDnotN=%d unsupported", c->CDnotN);
  if (c->useminA != 0) FAIL("useminA=%d unsupported", c->useminA);
  if (c->useminV == 1 || c->useminV == 2) FAIL("useminV=%d unsupported", c->useminV);
  if (c->bcType != 1) FAIL("bcType=%d unsupported", c->bcType);
  if (c->useEvap || c->useRain || c->useSubStep) FAIL("evap/rain/substep unsupported");
  if (c->inflowLocLength &&
      (c->inflowI0 < 0 || c->inflowJ0 < 0 || c->inflowI1 > c->nx || c->inflowJ1 > c->ny ||
       (long)(c->inflowI1 - c->inflowI0) * (c->inflowJ1 - c->inflowJ0) != c->inflowLocLength))
    FAIL("inflow cells must be the rectangle of inflowLocLength interior cells");
  if (c->useScalar && ((c->scalarAdv != 1 && c->scalarAdv != 2) || c->useConstTidePS != 1))
    FAIL("scalar options unsupported");
  if (c->tideLocFirstP < 0 || c->tideLocFirstP + c->tideLocLengthP > c->nx)
    FAIL("tidal cells outside the YP row");
  return 0;
}

oracle_domain *oracle_create(const oracle_cfg *cfg, char *errbuf, int errlen) {
  oracle_domain *d = (oracle_domain *)calloc(1, sizeof(oracle_domain));
  d->c = *cfg;
  if (check_cfg(d) != 0) {
    if (errbuf) snprintf(errbuf, (size_t)errlen, "%s", d->err);
    free(d);
    return NULL;
  }
  d->nx = cfg->nx;
  d->ny = cfg->ny;
  d->N = (long)d->nx * d->ny;
  d->T = (long)(d->nx + 2) * (d->ny + 2);
  make_maps(d);
  const long N = d->N, T = d->T;
  d->uuXP = dz(T); d->uuYP = dz(N); d->vvXP = dz(N); d->vvYP = dz(T);
  d->surf = dz(T); d->surfOld = dz(T); d->Fuu = dz(T); d->Fvv = dz(T); d->cellV = dz(N);
  d->depth = dz(N); d->depthXP = dz(T); d->depthYP = dz(T); d->EnXP = dz(T); d->EnYP = dz(T);
  d->DragXP = dz(T); d->DragYP = dz(T); d->CDXP = dz(T); d->CDYP = dz(T);
  d->GnCt = dz(N); d->GnXP = dz(N); d->GnYP = dz(N); d->GnXM = dz(N); d->GnYM = dz(N);
  d->z = dz(N); d->wtfXP = dz(T); d->wtfYP = dz(T); d->S = dz(T); d->Sm = dz(N);
  d->rmvCFL = dz(N); d->advX = dz(T); d->advY = dz(T); d->CFLx = dz(T); d->CFLy = dz(T);
  d->V = dz(T); d->Z = dz(T); d->Vxp = dz(T); d->Vyp = dz(T); d->Vxm = dz(T); d->Vym = dz(T);
  d->Np = dz(T); d->Nm = dz(T); d->Op = dz(T); d->Om = dz(T); d->Nx = dz(T); d->Oy = dz(T);
  d->Vx = dz(T); d->Vy = dz(T); d->Zx = dz(T); d->Zy = dz(T); d->ind = iz(T);
  d->bottomZ = dz(T); d->bottomXP = dz(T); d->bottomYP = dz(T); d->edgeX = dz(N);
  d->edgeY = dz(N);
  d->x = dz(N); d->wr = dz(N); d->wp = dz(N); d->wq = dz(N); d->wz = dz(N);
  d->precond = ORACLE_PRECOND_SSOR;
  d->x0mode = ORACLE_X0_ZERO;
  return d;
}

void oracle_destroy(oracle_domain *d) {
  if (!d) return;
  void *ptrs[] = {d->iPjc, d->iMjc, d->icjP, d->icjM, d->iPPjc, d->iMMjc, d->icjPP, d->icjMM,
                  d->trps, d->sprt, d->iPbd, d->iPgt,
                  d->iMbd, d->iMgt, d->jPbd, d->jPgt, d->jMbd, d->jMgt, d->uuXP, d->uuYP,
                  d->vvXP, d->vvYP, d->surf, d->surfOld, d->Fuu, d->Fvv, d->cellV, d->depth,
                  d->depthXP, d->depthYP, d->EnXP, d->EnYP, d->DragXP, d->DragYP, d->CDXP,
                  d->CDYP, d->GnCt, d->GnXP, d->GnYP, d->GnXM, d->GnYM, d->z, d->wtfXP,
                  d->wtfYP, d->S, d->Sm, d->rmvCFL, d->advX, d->advY, d->CFLx, d->CFLy,
                  d->allSurf, d->V, d->Z, d->Vxp, d->Vyp, d->Vxm, d->Vym, d->Np, d->Nm, d->Op,
                  d->Om, d->Nx, d->Oy, d->Vx, d->Vy, d->Zx, d->Zy, d->ind, d->bottomZ,
                  d->bottomXP, d->bottomYP, d->edgeX, d->edgeY, d->tideP, d->x, d->wr, d->wp,
                  d->wq, d->wz, d->inflow, d->windspd, d->winddir};
  for (size_t k = 0; k < sizeof(ptrs) / sizeof(ptrs[0]); ++k) free(ptrs[k]);
  for (int t = 0; t < NTAB; ++t) free(d->tab[t]);
  free(d);
}

const char *oracle_error(const oracle_domain *d) { return d ? d->err : "null domain"; }

int oracle_set_tables(oracle_domain *d, int Ne, const double *tables) {
  if (Ne <= 0) FAIL("Ne must be positive");
  d->Ne = Ne;
  const long n = d->N * (long)Ne;
  for (int t = 0; t < NTAB; ++t) {
    free(d->tab[t]);
    d->tab[t] = dz(n);
    memcpy(d->tab[t], tables + (long)t * n, (size_t)n * sizeof(double));
  }
  free(d->allSurf);
  d->allSurf = dz(Ne);
  /* initAllSubVar (subgrid.c:2116-2119) */
  for (int k = 0; k < Ne; ++k) d->allSurf[k] = d->c.surfmin + k * d->c.dsurf + d->c.offset;
  return 0;
}

/* bc->inflow (kind 1), bc->windspd (2), bc->winddir (3), indexed by tt. */
int oracle_set_series(oracle_domain *d, int kind, int n, const double *v) {
  double **dst = kind == 1 ? &d->inflow : kind == 2 ? &d->windspd : kind == 3 ? &d->winddir : NULL;
  if (!dst || n < 0) return 1;
  free(*dst);
  *dst = dz(n);
  if (n) memcpy(*dst, v, (size_t)n * sizeof(double));
  if (kind == 1) d->ninflow = n; else if (kind == 2) d->nwind = n; else d->nwdir = n;
  return 0;
}

/* A series value at step tt; past its end the reference reads the zeroed guard. */
static double series_at(const double *a, int n, int tt) {
  return (a && tt >= 0 && tt < n) ? a[tt] : 0.0;
}

/* Inflow cell test: inflowLoc[k] = jj*NX + ii - 1 (configuration.c:53-60). */
static int is_inflow(const oracle_domain *d, long ii) {
  if (!d->c.inflowLocLength) return 0;
  const int i = (int)(ii % d->nx), j = (int)(ii / d->nx);
  return i >= d->c.inflowI0 && i < d->c.inflowI1 && j >= d->c.inflowJ0 && j < d->c.inflowJ1;
}

int oracle_set_tide(oracle_domain *d, int n, const double *tideP) {
  free(d->tideP);
  d->tideP = dz(n);
  memcpy(d->tideP, tideP, (size_t)n * sizeof(double));
  d->nt = n;
  return 0;
}

void oracle_set_solver(oracle_domain *d, int precond, int x0mode) {
  d->precond = precond;
  d->x0mode = x0mode;
}

/* ------------------------------------------------------------- boundaries */
/* enforceFreeSurfaceBC (nsfunctions.c:317-334) */
static void enforce_surf_bc(oracle_domain *d) {
  double *s = d->surf;
  for (int i = 0; i < d->nx; ++i) { s[d->jPgt[i]] = s[d->jPbd[i]]; s[d->jMgt[i]] = s[d->jMbd[i]]; }
  for (int j = 0; j < d->ny; ++j) { s[d->iPgt[j]] = s[d->iPbd[j]]; s[d->iMgt[j]] = s[d->iMbd[j]]; }
  s[d->iPjP] = s[d->iPgt[d->ny - 1]];
  s[d->iPjM] = s[d->iMgt[d->ny - 1]];
  s[d->iMjP] = s[d->iPgt[0]];
  s[d->iMjM] = s[d->iMgt[0]];
}

/* enforceVelocityBC (nsfunctions.c:289-314) */
static void enforce_vel_bc(oracle_domain *d) {
  double *u = d->uuXP, *v = d->vvYP;
  for (int i = 0; i < d->nx; ++i) {
    u[d->jPgt[i]] = u[d->jPbd[i]]; u[d->jMgt[i]] = u[d->jMbd[i]];
    v[d->jPgt[i]] = v[d->jPbd[i]]; v[d->jMgt[i]] = v[d->jMbd[i]];
  }
  for (int j = 0; j < d->ny; ++j) {
    u[d->iPgt[j]] = u[d->iPbd[j]]; u[d->iMgt[j]] = u[d->iMbd[j]];
    v[d->iPgt[j]] = v[d->iPbd[j]]; v[d->iMgt[j]] = v[d->iMbd[j]];
  }
  u[d->iPjP] = u[d->jPgt[d->nx - 1]];
  u[d->iPjM] = u[d->jMgt[d->nx - 1]];
  u[d->iMjP] = u[d->jPgt[0]];
  u[d->iMjM] = u[d->jMgt[0]];
  v[d->iPjP] = v[d->iPgt[d->ny - 1]];
  v[d->iPjM] = v[d->iMgt[d->ny - 1]];
  v[d->iMjP] = v[d->iPgt[0]];
  v[d->iMjM] = v[d->iMgt[0]];
}

static int tide_cell(const oracle_domain *d, int k) { return d->c.tideLocFirstP + k + d->nx * (d->ny - 1); }

static double tide_at(const oracle_domain *d, int tt) {
  return (tt >= 0 && tt < d->nt) ? d->tideP[tt] : 0.0;
}

/* enforceTidalBC (nsfunctions.c:412-433), YP row only (bcType = 1) */
static void enforce_tidal_bc(oracle_domain *d, int tt) {
  const double h = tide_at(d, tt) + d->c.offset;
  for (int k = 0; k < d->c.tideLocLengthP; ++k) {
    int c = tide_cell(d, k);
    if (h > d->bottomZ[c]) d->surf[c] = h;
  }
}

/* zeroNegSurf (nsfunctions.c:436-449) */
static void zero_neg_surf(oracle_domain *d, int tt) {
  for (long ii = 0; ii < d->N; ++ii)
    if (d->surf[ii] < d->bottomZ[ii]) {
      double diff = d->bottomZ[ii] - d->surf[ii];
      d->surf[ii] = d->bottomZ[ii];
      if (tt > 1) d->Vloss[2] -= diff * d->c.dx * d->c.dy;
    }
}

/* updateDepth (nsfunctions.c:239-247) */
static void update_depth(oracle_domain *d) {
  for (long ii = 0; ii < d->N; ++ii) {
    d->depth[ii] = d->surf[ii] - d->bottomZ[ii];
    if (d->depth[ii] < 0) d->depth[ii] = 0;
  }
}

/* updateAllFaceDepth (nsfunctions.c:143-236), one rank */
static void update_face_depth(oracle_domain *d) {
  const int nx = d->nx, ny = d->ny;
  double *s = d->surf, *hx = d->depthXP, *hy = d->depthYP, *bx = d->bottomXP, *by = d->bottomYP;
  for (long k = 0; k < d->T; ++k) { hx[k] = 0; hy[k] = 0; }
  for (long ii = 0; ii < d->N; ++ii) {
    double a = s[ii], b = s[d->iPjc[ii]];
    hx[ii] = (a > b ? a : b) - bx[ii];
  }
  for (int j = 0; j < ny; ++j) {
    hx[d->iMgt[j]] = s[d->iMbd[j]] - bx[d->iMgt[j]];
    hx[d->iPgt[j]] = s[d->iPgt[j]] - bx[d->iPgt[j]];
    hx[d->iPbd[j]] = 0;
    hx[d->iPgt[j]] = 0;
    hx[d->iMgt[j]] = 0;
  }
  for (int i = 0; i < nx; ++i) {
    int g = d->jMgt[i];
    hx[g] = (s[g] > s[g + 1] ? s[g] : s[g + 1]) - bx[g];
    g = d->jPgt[i];
    hx[g] = (s[g] > s[g + 1] ? s[g] : s[g + 1]) - bx[g];
  }
  for (long ii = 0; ii < d->N; ++ii) {
    double a = s[ii], b = s[d->icjP[ii]];
    hy[ii] = (a > b ? a : b) - by[ii];
  }
  for (int i = 0; i < nx; ++i) {
    int g = d->jMgt[i];
    double a = s[g], b = s[d->jMbd[i]];
    hy[g] = (a > b ? a : b) - by[g];
    hy[d->jPgt[i]] = s[d->jPgt[i]] - by[d->jPgt[i]];
    hy[g] = 0;
  }
  for (int j = 0; j < ny; ++j) {
    hy[d->iMgt[j]] = hy[d->iMbd[j]];
    hy[d->iPgt[j]] = hy[d->iPbd[j]];
  }
  for (int i = 0; i < nx; ++i) { hy[d->jPbd[i]] = 0; hy[d->jPgt[i]] = 0; }
  for (int i = 0; i < nx; ++i) hy[d->jMgt[i]] = 0;
  for (long k = 0; k < d->T; ++k) {
    if (hx[k] < 0) hx[k] = 0;
    if (hy[k] < 0) hy[k] = 0;
  }
}

/* velocityInterp (nsfunctions.c:337-347): raw index arithmetic, wraps across rows */
static void velocity_interp(oracle_domain *d) {
  const long nx = d->nx;
  for (long ii = 0; ii < d->N; ++ii) {
    d->uuYP[ii] = 0.25 * (rdT(d, d->uuXP, ii) + rdT(d, d->uuXP, ii - 1) +
                          rdT(d, d->uuXP, ii + nx) + rdT(d, d->uuXP, ii - 1 + nx));
    d->vvXP[ii] = 0.25 * (rdT(d, d->vvYP, ii) + rdT(d, d->vvYP, ii + 1) +
                          rdT(d, d->vvYP, ii - nx) + rdT(d, d->vvYP, ii + 1 - nx));
  }
}

/* ------------------------------------------------------------- subgrid */
/* interpSurf (utilities.c:155-162) */
static inline double interp_surf(double x, double x1, double y1, double x2, double y2) {
  if (x2 == x1) return y1;
  return (y2 - y1) * (x - x2) / (x2 - x1) + y2;
}

/* computeSubArea (subgrid.c:55-251), useSubDrag = 0, useminA = 0.  The minV*
 * interpolations (subgrid.c:149-156) feed only useminV = 1/2 and are skipped. */
static void compute_sub_area(oracle_domain *d) {
  const long N = d->N;
  const double ds = d->c.dsurf;
  for (long ii = 0; ii < N; ++ii) {
    const double s = d->surf[ii];
    int *ind = &d->ind[ii];
    while (fabs(d->allSurf[*ind] - s) > 0.5 * ds + ds / 100) {
      if (s > d->allSurf[*ind]) *ind += 1; else *ind -= 1;
      if (*ind < 0) { *ind = 0; break; }
      if (*ind > d->Ne - 1) { *ind = d->Ne - 1; break; }
    }
    int j1 = *ind, j2;
    if (j1 == 0) j2 = 0;
    else if (j1 == d->Ne - 1) j2 = d->Ne - 1;
    else j2 = s > d->allSurf[j1] ? j1 + 1 : j1 - 1;
    const long k1 = N * j1 + ii, k2 = N * j2 + ii;
    const double a1 = d->allSurf[j1], a2 = d->allSurf[j2];
#define IP(t) interp_surf(s, a1, d->tab[t][k1], a2, d->tab[t][k2])
    d->V[ii] = IP(T_V);
    d->Z[ii] = IP(T_Z);
    d->Vxp[ii] = IP(T_VXP);
    d->Vyp[ii] = IP(T_VYP);
    d->Vxm[ii] = IP(T_VXM);
    d->Vym[ii] = IP(T_VYM);
    /* face areas with the wet/dry edge special case (subgrid.c:159-218) */
    const double wd[4] = {rdN(d, d->edgeX, ii), rdN(d, d->edgeX, d->iMjc[ii]),
                          rdN(d, d->edgeY, ii), rdN(d, d->edgeY, d->icjM[ii])};
    const int tb[4] = {T_NP, T_NM, T_OP, T_OM};
    double *outp[4] = {d->Np, d->Nm, d->Op, d->Om};
    for (int f = 0; f < 4; ++f) {
      double w = wd[f];
      if (w > a1 && w < a2) {
        outp[f][ii] = w > s ? 0.0 : interp_surf(s, w, 0.0, a2, d->tab[tb[f]][k2]);
      } else {
        outp[f][ii] = IP(tb[f]);
      }
    }
#undef IP
    if (d->depth[ii] == 0) { d->Vxp[ii] = 0; d->Vyp[ii] = 0; d->Vxm[ii] = 0; d->Vym[ii] = 0; }
    if (s - d->bottomXP[ii] <= 0) d->Np[ii] = 0;
    if (s - d->bottomYP[ii] <= 0) d->Op[ii] = 0;
    if (d->iMjc[ii] < N && s - d->bottomXP[d->iMjc[ii]] <= 0) d->Nm[ii] = 0;
    if (d->icjM[ii] < N && s - d->bottomYP[d->icjM[ii]] <= 0) d->Om[ii] = 0;
  }
}

/* combineSubArea (subgrid.c:254-526), useminA = 0, useminV not 1/2, one rank. */
static void combine_sub_area(oracle_domain *d) {
  const long N = d->N;
  const double dxdy = d->c.dx * d->c.dy;
  const double Vmin = 0.002, Amin = 0.002, Azmin = 0.002;
  for (long ii = 0; ii < N; ++ii) {
    const int e = d->iPjc[ii], n = d->icjP[ii];
    if (e < N) d->Nx[ii] = d->Np[ii] >= d->Nm[e] ? d->Np[ii] : d->Nm[e];
    else d->Nx[ii] = d->Np[ii];
    if (n < N) d->Oy[ii] = d->Op[ii] >= d->Om[n] ? d->Op[ii] : d->Om[n];
    else d->Oy[ii] = d->Op[ii];
    if (e < N) {
      if (d->Vxp[ii] > 0 && d->Vxm[e] > 0) d->Vx[ii] = d->Vxp[ii] + d->Vxm[e];
      else d->Vx[ii] = 2.0 * (d->Vxp[ii] + d->Vxm[e]);
      d->Zx[ii] = d->Z[ii];
      if (d->Vx[ii] > 0 && d->Zx[ii] <= 0) d->Zx[ii] = dxdy;
      if (d->surf[ii] < d->bottomXP[ii]) { d->Vx[ii] = d->Vxm[e]; d->Zx[ii] = 0.5 * d->Z[ii]; }
      if (d->surf[e] < d->bottomXP[ii]) { d->Vx[ii] = d->Vxp[ii]; d->Zx[ii] = 0.5 * d->Z[ii]; }
    } else {
      d->Vx[ii] = 2 * d->Vxp[ii];
      d->Zx[ii] = 2 * d->Z[ii];
    }
    if (n < N) {
      if (d->Vyp[ii] > 0 && d->Vym[n] > 0) d->Vy[ii] = d->Vyp[ii] + d->Vym[n];
      else d->Vy[ii] = 2.0 * (d->Vyp[ii] + d->Vym[n]);
      d->Zy[ii] = d->Z[ii];
      if (d->Vy[ii] > 0 && d->Zy[ii] <= 0) d->Zy[ii] = dxdy;
      if (d->surf[ii] < d->bottomYP[ii]) { d->Vy[ii] = d->Vym[n]; d->Zy[ii] = 0.5 * d->Z[ii]; }
      if (d->surf[n] < d->bottomYP[ii]) { d->Vy[ii] = d->Vyp[ii]; d->Zy[ii] = 0.5 * d->Z[ii]; }
    } else {
      d->Vy[ii] = 2 * d->Vyp[ii];
      d->Zy[ii] = 2 * d->Z[ii];
    }
  }
  for (long ii = 0; ii < N; ++ii) {
    if (d->Vx[ii] < Vmin) d->Vx[ii] = 0.0;
    if (d->Vy[ii] < Vmin) d->Vy[ii] = 0.0;
    if (d->V[ii] < Vmin) d->V[ii] = 0.0;
    if (d->Z[ii] < Azmin) d->Z[ii] = 1.0;
    if (d->Zx[ii] < Amin) d->Zx[ii] = 0.0;
    if (d->Zy[ii] < Amin) d->Zy[ii] = 0.0;
    if (d->Nx[ii] < Amin) d->Nx[ii] = 0.0;
    if (d->Oy[ii] < Amin) d->Oy[ii] = 0.0;
  }
  double *g8[8] = {d->Vx, d->Vy, d->Zx, d->Zy, d->Nx, d->Oy, d->V, d->Z};
  for (int j = 0; j < d->ny; ++j) {
    for (int a = 0; a < 8; ++a) {
      g8[a][d->iMgt[j]] = g8[a][d->iMbd[j]];
      g8[a][d->iPgt[j]] = g8[a][d->iPbd[j]];
    }
    d->Nx[d->iMgt[j]] = 0;
    d->Nx[d->iPgt[j]] = 0;
    d->Nx[d->iPbd[j]] = 0;
  }
  for (int i = 0; i < d->nx; ++i) {
    for (int a = 0; a < 8; ++a) {
      g8[a][d->jMgt[i]] = g8[a][d->jMbd[i]];
      g8[a][d->jPgt[i]] = g8[a][d->jPbd[i]];
    }
    d->Oy[d->jMgt[i]] = 0;
  }
  /* faces of the YP row closed except at tidal cells (subgrid.c:511-525) */
  for (int i = 0; i < d->nx; ++i) {
    int tidal = i >= d->c.tideLocFirstP && i < d->c.tideLocFirstP + d->c.tideLocLengthP;
    if (!tidal) { d->Oy[d->jPbd[i]] = 0; d->Oy[d->jPgt[i]] = 0; }
  }
}

/* ------------------------------------------------------------- drag */
/* updateCDSub (subgrid.c:1447-1538), useSubDrag = 0 branch */
static void update_cd(oracle_domain *d) {
  const double coeff = d->c.g * d->c.manningN * d->c.manningN;
  for (long ii = 0; ii < d->N; ++ii)
    if (d->V[ii] > 0) {
      double h = d->V[ii] / d->Z[ii];
      d->CDXP[ii] = coeff / pow(h, 1.0 / 3.0);
      d->CDYP[ii] = coeff / pow(h, 1.0 / 3.0);
    }
}

/* thinLayerDrag (nsfunctions.c:691-727), CDnotN = 0 branch */
static void thin_layer_drag(oracle_domain *d) {
  const double coeff = d->c.g * d->c.manningN * d->c.manningN;
  for (long ii = 0; ii < d->N; ++ii)
    if (d->depth[ii] > 0) {
      if (d->depthXP[ii] <= d->c.hD) d->CDXP[ii] = coeff / pow(d->depth[ii], 2.0 / 3.0);
      if (d->depthYP[ii] <= d->c.hD) d->CDYP[ii] = coeff / pow(d->depth[ii], 2.0 / 3.0);
    }
}

/* ------------------------------------------------------------- init */
/* updateAllFaceElev (nsfunctions.c:76-140), subgrid branch (edge files) */
static void update_face_elev(oracle_domain *d) {
  double *z = d->bottomZ, *bx = d->bottomXP, *by = d->bottomYP;
  for (long k = 0; k < d->T; ++k) { bx[k] = 0; by[k] = 0; }
  for (long ii = 0; ii < d->N; ++ii) bx[ii] = d->edgeX[ii];
  for (int j = 0; j < d->ny; ++j) { bx[d->iMgt[j]] = z[d->iMbd[j]]; bx[d->iPgt[j]] = bx[d->iPbd[j]]; }
  for (int i = 0; i < d->nx; ++i) { bx[d->jMgt[i]] = bx[d->jMbd[i]]; bx[d->jPgt[i]] = bx[d->jPbd[i]]; }
  for (long ii = 0; ii < d->N; ++ii) by[ii] = d->edgeY[ii];
  for (int i = 0; i < d->nx; ++i) {
    int g = d->jMgt[i];
    by[g] = z[g] > z[i] ? z[g] : z[i];
    by[d->jPgt[i]] = by[d->jPbd[i]];
  }
  for (int j = 0; j < d->ny; ++j) { by[d->iMgt[j]] = by[d->iMbd[j]]; by[d->iPgt[j]] = by[d->iPbd[j]]; }
}

/* Init (initialize.c:40-155) for the subgrid path, plus SolveAll's tt = 0
 * output round trip of surf (nssolve.c:54, fileio.c:65-66,120-121). */
int oracle_init(oracle_domain *d, const double *bottom, const double *bottomXP,
                const double *bottomYP, const double *surf0, const double *u0,
                const double *v0, const double *S0, int round_trip_output) {
  if (!d->tab[0]) FAIL("tables not set");
  const long N = d->N;
  const double off = d->c.offset;
  /* InitBathymetry (bathymetry.c:104-121) */
  for (long k = 0; k < d->T; ++k) d->bottomZ[k] = 0;
  for (long ii = 0; ii < N; ++ii) {
    d->bottomZ[ii] = bottom[ii] + off;
    d->edgeX[ii] = bottomXP[ii] + off;
    d->edgeY[ii] = bottomYP[ii] + off;
  }
  /* enforceBathBC (initialize.c:158-175) */
  for (int i = 0; i < d->nx; ++i) {
    d->bottomZ[d->jMgt[i]] = d->bottomZ[d->jMbd[i]];
    d->bottomZ[d->jPgt[i]] = d->bottomZ[d->jPbd[i]];
  }
  for (int j = 0; j < d->ny; ++j) {
    d->bottomZ[d->iMgt[j]] = d->bottomZ[d->iMbd[j]];
    d->bottomZ[d->iPgt[j]] = d->bottomZ[d->iPbd[j]];
  }
  update_face_elev(d);
  /* initFieldValues (initialize.c:393-443) */
  for (long ii = 0; ii < N; ++ii) {
    d->surf[ii] = surf0[ii] + off;
    d->uuXP[ii] = u0 ? u0[ii] : 0.0;
    d->vvYP[ii] = v0 ? v0[ii] : 0.0;
    if (d->c.useScalar) d->S[ii] = S0 ? S0[ii] : 0.0;
  }
  /* initCD (initialize.c:382-390) */
  for (long k = 0; k < d->T; ++k) { d->CDXP[k] = d->c.CDx; d->CDYP[k] = d->c.CDy; }
  zero_neg_surf(d, 0);
  enforce_surf_bc(d);
  enforce_vel_bc(d);
  enforce_tidal_bc(d, 0);
  update_depth(d);
  update_face_depth(d);
  for (long k = 0; k < d->T; ++k) d->ind[k] = d->Ne / 2;  /* subgrid.c:2268-2270 */
  compute_sub_area(d);
  combine_sub_area(d);
  /* computeVolume (nsfunctions.c:361-370), plain form at init */
  for (long ii = 0; ii < N; ++ii) {
    d->cellV[ii] = d->c.dx * d->c.dy * d->depth[ii];
    if (d->c.useScalar) d->Sm[ii] = d->S[ii] * d->cellV[ii];
  }
  velocity_interp(d);
  thin_layer_drag(d); /* unconditional at init (initialize.c:140) */
  if (d->c.useScalar) {
    for (long ii = 0; ii < N; ++ii)
      if (d->depth[ii] <= 0) d->S[ii] = 0;
    for (long ii = 0; ii < N; ++ii) d->Sm[ii] = d->S[ii] * d->cellV[ii];
  }
  if (round_trip_output) {
    for (long ii = 0; ii < N; ++ii) d->surf[ii] = d->surf[ii] - off;
    for (long ii = 0; ii < N; ++ii) d->surf[ii] = d->surf[ii] + off;
  }
  return 0;
}

/* ------------------------------------------------------------- explicit */
/* explicitVelocity + advectionTerm (nsfunctions.c:498-586) */
static void advection(oracle_domain *d) {
  const double dx = d->c.dx, dy = d->c.dy, dt = d->c.dt;
  const double CFLh = d->c.CFLh, CFLl = d->c.CFLl;
  double *u = d->uuXP, *v = d->vvYP, *ax = d->advX, *ay = d->advY;
  for (long ii = 0; ii < d->N; ++ii) { d->EnXP[ii] = u[ii]; d->EnYP[ii] = v[ii]; }
  for (long ii = 0; ii < d->N; ++ii) {
    const int e = d->iPjc[ii], w = d->iMjc[ii], n = d->icjP[ii], s = d->icjM[ii];
    ax[ii] = (0.5 / dx) * (u[ii] + fabs(u[ii])) * (u[ii] - u[w]) +
             (0.5 / dx) * (u[ii] - fabs(u[ii])) * (u[e] - u[ii]) +
             (0.5 / dy) * (d->vvXP[ii] + fabs(d->vvXP[ii])) * (u[ii] - u[s]) +
             (0.5 / dy) * (d->vvXP[ii] - fabs(d->vvXP[ii])) * (u[n] - u[ii]);
    ay[ii] = (0.5 / dx) * (d->uuYP[ii] + fabs(d->uuYP[ii])) * (v[ii] - v[w]) +
             (0.5 / dx) * (d->uuYP[ii] - fabs(d->uuYP[ii])) * (v[e] - v[ii]) +
             (0.5 / dy) * (v[ii] + fabs(v[ii])) * (v[ii] - v[s]) +
             (0.5 / dy) * (v[ii] - fabs(v[ii])) * (v[n] - v[ii]);
    if (u[ii] == 0) ax[ii] = 0;
    if (v[ii] == 0) ay[ii] = 0;
  }
  /* order-dependent CFL limiter, restated as the same sequential sweep */
  for (long ii = 0; ii < d->N; ++ii) {
    const int nb[5] = {(int)ii, d->iPjc[ii], d->iMjc[ii], d->icjP[ii], d->icjM[ii]};
    const double cx = d->CFLx[ii], cy = d->CFLy[ii];
    if (cx > CFLl && cx <= CFLh) {
      for (int q = 0; q < 5; ++q) ax[nb[q]] = ax[nb[q]] * (CFLh - d->CFLx[nb[q]]) / (CFLh - CFLl);
    } else if (cx > CFLh) {
      for (int q = 0; q < 5; ++q) ax[nb[q]] = 0;
    }
    if (cy > CFLl && cy < CFLh) {
      for (int q = 0; q < 5; ++q) ay[nb[q]] = ay[nb[q]] * (CFLh - d->CFLy[nb[q]]) / (CFLh - CFLl);
    } else if (cx > CFLh) { /* the reference tests CFLx here (nsfunctions.c:574) */
      for (int q = 0; q < 5; ++q) ay[nb[q]] = 0;
    }
    d->EnXP[ii] = d->EnXP[ii] - dt * ax[ii];
    d->EnYP[ii] = d->EnYP[ii] - dt * ay[ii];
  }
}

/* diffusionTermSub (subgrid.c:781-812) */
static void diffusion(oracle_domain *d) {
  const double dx = d->c.dx, dy = d->c.dy, dt = d->c.dt, NUx = d->c.NUx, NUy = d->c.NUy;
  double *u = d->uuXP, *v = d->vvYP, *Nx = d->Nx, *Oy = d->Oy;
  for (long ii = 0; ii < d->N; ++ii) {
    const int e = d->iPjc[ii], w = d->iMjc[ii], n = d->icjP[ii], s = d->icjM[ii];
    double fx = 0, fy = 0;
    if (d->Vx[ii] > 0)
      fx = (NUx / d->Vx[ii]) * (Nx[e] * (u[e] - u[ii]) / dx - Nx[ii] * (-u[w] + u[ii]) / dx) +
           (NUy / d->Vx[ii]) * (Oy[ii] * (u[n] - u[ii]) / dy - Oy[s] * (-u[s] + u[ii]) / dy);
    if (d->Vy[ii] > 0)
      fy = (NUx / d->Vy[ii]) * (Nx[ii] * (v[e] - v[ii]) / dx - Nx[w] * (-v[w] + v[ii]) / dx) +
           (NUy / d->Vy[ii]) * (Oy[n] * (v[n] - v[ii]) / dy - Oy[ii] * (-v[s] + v[ii]) / dy);
    d->EnXP[ii] = d->EnXP[ii] + dt * fx;
    d->EnYP[ii] = d->EnYP[ii] + dt * fy;
  }
}

/* windTerm (nsfunctions.c:609-648): uniform wind stress with the thin-layer
 * decay, pi and the water density as the reference writes them, on the face
 * depths of the last updateAllFaceDepth.  Note the sign of the y term. */
static void wind(oracle_domain *d) {
  const double pi = 3.1415926, rho = 1000;
  const double W = series_at(d->windspd, d->nwind, d->tt);
  const double phi = series_at(d->winddir, d->nwdir, d->tt) + d->c.northAngle;
  const double omega = phi * pi / 180.0;
  const double dt = d->c.dt, hD = d->c.hD, CwT = d->c.CwT;
  for (long ii = 0; ii < d->N; ++ii) {
    const double tau = d->c.rhoa * d->c.Cw *
                       (W - d->uuXP[ii] * cos(omega) - d->vvYP[ii] * sin(omega)) *
                       (W - d->uuXP[ii] * cos(omega) - d->vvYP[ii] * sin(omega));
    double tauXP, tauYP;
    if (d->depthXP[ii] < hD && d->c.useThinLayer == 1)
      tauXP = tau * exp(CwT * (d->depthXP[ii] - hD) / hD);
    else
      tauXP = tau;
    if (d->depthYP[ii] < hD && d->c.useThinLayer == 1)
      tauYP = tau * exp(CwT * (d->depthYP[ii] - hD) / hD);
    else
      tauYP = tau;
    if (d->depthXP[ii] > 0)
      d->EnXP[ii] = d->EnXP[ii] + dt * tauXP * cos(omega) / (d->depthXP[ii] * rho);
    if (d->depthYP[ii] > 0)
      d->EnYP[ii] = d->EnYP[ii] - dt * tauYP * sin(omega) / (d->depthYP[ii] * rho);
  }
}

/* dragTermSub (subgrid.c:857-927, staggeredV = 1) and dragInversion
 * (nsfunctions.c:730-746) */
static void drag(oracle_domain *d) {
  const double dt = d->c.dt;
  for (long ii = 0; ii < d->N; ++ii) {
    double velx = sqrt(d->uuXP[ii] * d->uuXP[ii] + d->vvXP[ii] * d->vvXP[ii]);
    double vely = sqrt(d->uuYP[ii] * d->uuYP[ii] + d->vvYP[ii] * d->vvYP[ii]);
    double hx = d->Vx[ii] > 0 ? d->Zx[ii] / d->Vx[ii] : 0;
    double hy = d->Vy[ii] > 0 ? d->Zy[ii] / d->Vy[ii] : 0;
    d->DragXP[ii] = 0.5 * dt * d->CDXP[ii] * velx * hx;
    d->DragYP[ii] = 0.5 * dt * d->CDYP[ii] * vely * hy;
  }
  for (int i = 0; i < d->nx; ++i) d->DragXP[d->jMgt[i]] = d->DragXP[d->jMbd[i]];
  for (int j = 0; j < d->ny; ++j) d->DragYP[d->iMgt[j]] = d->DragYP[d->iMbd[j]];
  for (long ii = 0; ii < d->N; ++ii) {
    d->EnXP[ii] = d->EnXP[ii] / (1 + d->DragXP[ii]);
    d->EnYP[ii] = d->EnYP[ii] / (1 + d->DragYP[ii]);
  }
  for (int i = 0; i < d->nx; ++i) d->EnXP[d->jMgt[i]] = d->EnXP[d->jMbd[i]];
  for (int j = 0; j < d->ny; ++j) d->EnYP[d->iMgt[j]] = d->EnYP[d->iMbd[j]];
}

/* matrixSourceTermSub (subgrid.c:930-975) */
static void rhs(oracle_domain *d) {
  const double dt = d->c.dt;
  for (long k = 0; k < d->N; ++k) {
    const int c = d->trps[k], w = d->iMjc[c], s = d->icjM[c];
    d->z[k] = d->surf[c] * d->Z[c] - dt * (d->EnXP[c] * d->Nx[c] - d->EnXP[w] * d->Nx[w]) -
              dt * (d->EnYP[c] * d->Oy[c] - d->EnYP[s] * d->Oy[s]);
  }
  /* inflow cells (subgrid.c:959-968; bcType != 3) */
  if (d->c.inflowLocLength) {
    const double q = series_at(d->inflow, d->ninflow, d->tt);
    for (long ii = 0; ii < d->N; ++ii)
      if (is_inflow(d, ii)) {
        const long k = d->sprt[ii];
        d->z[k] = d->z[k] + dt * (q / d->c.inflowLocLength);
      }
  }
  for (long k = 0; k < d->N; ++k) {
    const int c = d->trps[k];
    if (d->z[k] == 0 || d->z[k] == d->surf[c] * d->c.dx * d->c.dy)
      d->z[k] = d->surf[c] * d->c.dx * d->c.dy;
  }
}

/* matrixCoeffSub (subgrid.c:978-1081, useSubgrid = 1, staggeredV = 1),
 * adjustMatrixBoundary (nsfunctions.c:846-884) and adjustTidalBoundary
 * (nsfunctions.c:887-924), one rank. */
static void assemble(oracle_domain *d, int tt) {
  const double coef = d->c.g * (d->c.dt * d->c.dt), divider = 1.0, dxdy = d->c.dx * d->c.dy;
  const long N = d->N;
  for (long ii = 0; ii < N; ++ii) {
    const int w = d->iMjc[ii], s = d->icjM[ii];
    d->GnXP[ii] = 0; d->GnXM[ii] = 0; d->GnYP[ii] = 0; d->GnYM[ii] = 0;
    if (d->Vx[ii] > 0)
      d->GnXP[ii] = coef * d->Nx[ii] * d->Nx[ii] / d->Vx[ii] / divider / (1 + d->DragXP[ii]);
    if (d->Vx[w] > 0)
      d->GnXM[ii] = coef * d->Nx[w] * d->Nx[w] / d->Vx[w] / divider / (1 + d->DragXP[w]);
    if (d->Vy[ii] > 0)
      d->GnYP[ii] = coef * d->Oy[ii] * d->Oy[ii] / d->Vy[ii] / divider / (1 + d->DragYP[ii]);
    if (d->Vy[s] > 0)
      d->GnYM[ii] = coef * d->Oy[s] * d->Oy[s] / d->Vy[s] / divider / (1 + d->DragYP[s]);
    d->GnCt[ii] = d->Z[ii] + d->GnXP[ii] + d->GnYP[ii] + d->GnXM[ii] + d->GnYM[ii];
  }
  for (long ii = 0; ii < N; ++ii) {
    if (d->GnCt[ii] == 0.0 || d->GnCt[ii] == dxdy) d->GnCt[ii] = dxdy;
    if (d->depth[ii] == 0 && d->uuXP[ii] == 0 && d->uuXP[d->iMjc[ii]] == 0 &&
        d->vvYP[ii] == 0 && d->vvYP[d->icjM[ii]] == 0) {
      d->GnCt[ii] = dxdy;
      d->GnXM[ii] = 0.0; d->GnXP[ii] = 0.0; d->GnYM[ii] = 0.0; d->GnYP[ii] = 0.0;
      d->z[d->sprt[ii]] = d->surf[ii] * d->c.dx * d->c.dy;
    }
  }
  for (int j = 0; j < d->ny; ++j) {
    long a = (long)j * d->nx, b = (long)j * d->nx + d->nx - 1;
    d->GnCt[a] = d->GnCt[a] - d->GnXM[a]; d->GnXM[a] = 0;
    d->GnCt[b] = d->GnCt[b] - d->GnXP[b]; d->GnXP[b] = 0;
  }
  for (int i = 0; i < d->nx; ++i) {
    long a = i, b = N - d->nx + i;
    d->GnCt[a] = d->GnCt[a] - d->GnYM[a]; d->GnYM[a] = 0;
    d->GnCt[b] = d->GnCt[b] - d->GnYP[b]; d->GnYP[b] = 0;
  }
  const double h = tide_at(d, tt) + d->c.offset;
  for (int k = 0; k < d->c.tideLocLengthP; ++k) {
    int c = tide_cell(d, k);
    d->GnCt[c] = 1; d->GnXM[c] = 0; d->GnXP[c] = 0; d->GnYM[c] = 0; d->GnYP[c] = 0;
    d->z[d->sprt[c]] = h;
  }
}

void oracle_explicit(oracle_domain *d, int tt) {
  d->tt = tt;
  advection(d);
  diffusion(d);
  if (d->c.useWind) wind(d);
  drag(d);
  rhs(d);
  assemble(d, tt);
}

/* ------------------------------------------------------------- solve */
/* The assembled 5-point matrix in laspack's transposed order (setupMatrix,
 * nsfunctions.c:927-1001): row k <-> cell trps[k]; couplings across the domain
 * boundary are not stored. */
static void matvec(const oracle_domain *d, const double *p, double *q) {
  const int nx = d->nx, ny = d->ny;
  for (long k = 0; k < d->N; ++k) {
    const int c = d->trps[k], i = c % nx, j = c / nx;
    double s = d->GnCt[c] * p[k];
    if (j > 0) s -= d->GnYM[c] * p[k - 1];
    if (j < ny - 1) s -= d->GnYP[c] * p[k + 1];
    if (i > 0) s -= d->GnXM[c] * p[k - ny];
    if (i < nx - 1) s -= d->GnXP[c] * p[k + ny];
    q[k] = s;
  }
}

static double dot(const double *a, const double *b, long n) {
  double s = 0.0;
  for (long k = 0; k < n; ++k) s += a[k] * b[k];
  return s;
}

/* y = M^-1 r: Jacobi (precond.c:26-46) or SSOR with omega = 1 (precond.c:48-73):
 * forward Gauss-Seidel sweep over the lower part, scaling by the diagonal,
 * backward sweep over the upper part, in the transposed row order. */
static void precondition(const oracle_domain *d, const double *r, double *y) {
  const int nx = d->nx, ny = d->ny;
  const long N = d->N;
  if (d->precond == ORACLE_PRECOND_JACOBI) {
    for (long k = 0; k < N; ++k) y[k] = r[k] / d->GnCt[d->trps[k]];
    return;
  }
  for (long k = 0; k < N; ++k) {
    const int c = d->trps[k], i = c % nx, j = c / nx;
    double s = r[k];
    if (i > 0) s += d->GnXM[c] * y[k - ny];
    if (j > 0) s += d->GnYM[c] * y[k - 1];
    y[k] = s / d->GnCt[c];
  }
  for (long k = 0; k < N; ++k) y[k] = d->GnCt[d->trps[k]] * y[k];
  for (long k = N - 1; k >= 0; --k) {
    const int c = d->trps[k], i = c % nx, j = c / nx;
    double s = y[k];
    if (j < ny - 1) s += d->GnYP[c] * y[k + 1];
    if (i < nx - 1) s += d->GnXP[c] * y[k + ny];
    y[k] = s / d->GnCt[c];
  }
}

/* CGIter (itersolv.c:355-456) with the residual test of RTCResult (rtc.c:48-78):
 * stop when ||r||_2 < eps*||b||_2, checked before each iteration. */
void oracle_solve(oracle_domain *d) {
  const long N = d->N;
  double *x = d->x, *r = d->wr, *p = d->wp, *q = d->wq, *zz = d->wz;
  const double *b = d->z;
  if (d->x0mode == ORACLE_X0_SURFACE) {
    for (long k = 0; k < N; ++k) x[k] = d->surf[d->trps[k]];
  } else {
    for (long k = 0; k < N; ++k) x[k] = 0.0;
  }
  const double bnorm = sqrt(dot(b, b, N));
  matvec(d, x, q);
  for (long k = 0; k < N; ++k) r[k] = b[k] - q[k];
  double rho_old = 0.0;
  int it = 0;
  double rnorm = sqrt(dot(r, r, N));
  while (!(rnorm < d->c.eps * bnorm) && it < d->c.maxIter) {
    ++it;
    precondition(d, r, zz);
    double rho = dot(r, zz, N);
    if (it == 1) {
      for (long k = 0; k < N; ++k) p[k] = zz[k];
    } else {
      double beta = rho / rho_old;
      for (long k = 0; k < N; ++k) p[k] = zz[k] + beta * p[k];
    }
    matvec(d, p, q);
    double alpha = rho / dot(p, q, N);
    for (long k = 0; k < N; ++k) x[k] += alpha * p[k];
    for (long k = 0; k < N; ++k) r[k] -= alpha * q[k];
    rho_old = rho;
    rnorm = sqrt(dot(r, r, N));
  }
  d->last_iters = it;
  d->last_acc = bnorm != 0 ? rnorm / bnorm : 1.0;
}

int oracle_last_iters(const oracle_domain *d) { return d->last_iters; }
double oracle_last_accuracy(const oracle_domain *d) { return d->last_acc; }

/* ------------------------------------------------------------- update */
/* limiterCFL (nsfunctions.c:452-495): depth is read at ghost indices (0.0). */
static void limiter_cfl(oracle_domain *d) {
  const double md = d->c.minDepth;
  for (long ii = 0; ii < d->N; ++ii) {
    double diff = d->surf[ii] - d->bottomZ[ii];
    if (d->depth[ii] <= 0 && diff > 0) {
      const double so = d->surfOld[ii];
      const int nb[4] = {d->iPjc[ii], d->iMjc[ii], d->icjP[ii], d->icjM[ii]};
      int all = 1;
      for (int q = 0; q < 4; ++q) {
        int ok = (d->surfOld[nb[q]] <= so + md) | (rdN(d, d->depth, nb[q]) <= 0);
        all &= ok;
      }
      if (all) {
        if (ii < d->N - d->c.dx) d->Vloss[0] += diff * d->c.dx * d->c.dy;
        d->surf[ii] = d->bottomZ[ii];
        d->rmvCFL[ii] = 1;
      }
    }
  }
  for (long ii = 0; ii < d->N; ++ii) {
    double diff = d->surf[ii] - d->bottomZ[ii];
    if (diff <= md && diff > 0) {
      d->Vloss[1] += diff * d->c.dx * d->c.dy;
      d->surf[ii] = d->bottomZ[ii];
      d->cellV[ii] = 0;
      d->rmvCFL[ii] = 0;
    }
  }
}

/* detectWaterfallLocationSub (subgrid.c:1335-1396) */
static void detect_waterfall(oracle_domain *d) {
  const double wtfh = d->c.wtfh;
  double *s = d->surf;
  for (long ii = 0; ii < d->N; ++ii) { d->wtfXP[ii] = 0; d->wtfYP[ii] = 0; }
  for (long ii = 0; ii < d->N; ++ii) {
    double b = d->bottomXP[ii];
    if (s[ii] < b && s[d->iPjc[ii]] - b >= wtfh) d->wtfXP[ii] = -1;
  }
  for (long ii = 0; ii < d->N; ++ii) {
    int w = d->iMjc[ii];
    double b = d->bottomXP[w];
    if (s[ii] < b && s[w] - b >= wtfh) d->wtfXP[w] = 1;
  }
  for (long ii = 0; ii < d->N; ++ii) {
    double b = d->bottomYP[ii];
    if (s[ii] < b && s[d->icjP[ii]] - b >= wtfh) d->wtfYP[ii] = -1;
  }
  for (long ii = 0; ii < d->N; ++ii) {
    int sm = d->icjM[ii];
    double b = d->bottomYP[sm];
    if (s[ii] < b && s[sm] - b >= wtfh) d->wtfYP[sm] = 1;
  }
}

/* updateVelocitySub (subgrid.c:1084-1187), useSubgrid = 1, staggeredV = 1 */
static void update_velocity(oracle_domain *d) {
  const double g = d->c.g, dt = d->c.dt, divider = 1.0;
  double *u = d->uuXP, *v = d->vvYP;
  for (long ii = 0; ii < d->N; ++ii) {
    u[ii] = 0;
    v[ii] = 0;
    double hx = d->Vx[ii] > 0 ? d->Nx[ii] / d->Vx[ii] : 0;
    double hy = d->Vy[ii] > 0 ? d->Oy[ii] / d->Vy[ii] : 0;
    u[ii] = d->EnXP[ii] - (g * dt * hx) * (d->surf[d->iPjc[ii]] - d->surf[ii]) / divider;
    v[ii] = d->EnYP[ii] - (g * dt * hy) * (d->surf[d->icjP[ii]] - d->surf[ii]) / divider;
  }
  for (long ii = 0; ii < d->N; ++ii) {
    if (d->Nx[ii] == 0) u[ii] = 0;
    if (d->Oy[ii] == 0) v[ii] = 0;
  }
  for (long ii = 0; ii < d->N; ++ii)
    if (d->depth[ii] == 0) {
      if (u[ii] > 0) u[ii] = 0;
      if (u[d->iMjc[ii]] < 0) u[d->iMjc[ii]] = 0;
      if (v[ii] > 0) v[ii] = 0;
      if (v[d->icjM[ii]] < 0) v[d->icjM[ii]] = 0;
    }
  for (long ii = 0; ii < d->N; ++ii)
    if (d->rmvCFL[ii] == 1) {
      u[ii] = 0; v[ii] = 0; u[d->iMjc[ii]] = 0; v[d->icjM[ii]] = 0;
      d->rmvCFL[ii] = 0;
    }
}

/* waterfallCorrectionSub (subgrid.c:1400-1444) */
static void waterfall_correction(oracle_domain *d) {
  const double Cw = 0.7, CFLmax = 0.24 / d->c.subR, g = d->c.g, dt = d->c.dt;
  for (long ii = 0; ii < d->N; ++ii) {
    if (d->wtfXP[ii] != 0) {
      double v0 = d->uuXP[ii];
      d->uuXP[ii] = d->wtfXP[ii] * Cw * sqrt(2 * g * d->Nx[ii] / d->c.dy);
      if (fabs(d->uuXP[ii]) > CFLmax * d->c.dx / dt) d->uuXP[ii] = d->wtfXP[ii] * CFLmax * d->c.dx / dt;
      d->Vloss[3] -= (v0 - d->uuXP[ii]) * dt * d->Nx[ii];
    }
    if (d->wtfYP[ii] != 0) {
      double v0 = d->vvYP[ii];
      d->vvYP[ii] = d->wtfYP[ii] * Cw * sqrt(2 * g * d->Oy[ii] / d->c.dx);
      if (fabs(d->vvYP[ii]) > CFLmax * d->c.dy / dt) d->vvYP[ii] = d->wtfYP[ii] * CFLmax * d->c.dy / dt;
      d->Vloss[3] -= (v0 - d->vvYP[ii]) * dt * d->Oy[ii];
    }
  }
}

/* adjustTidalVelocitySub (subgrid.c:1291-1333), YP row */
static void tidal_velocity(oracle_domain *d) {
  for (int k = 0; k < d->c.tideLocLengthP; ++k) {
    int c = tide_cell(d, k);
    double Fww = (d->surf[c] - d->surfOld[c]) * d->Z[c] / d->c.dt;
    double all = d->Fvv[d->icjM[c]] + d->Fuu[d->iMjc[c]] - d->Fuu[c] - Fww;
    if (all != 0 && d->Oy[c] > 0) d->vvYP[c] = all / d->Oy[c];
    else d->vvYP[c] = 0;
  }
}

/* volumeByFluxSub (subgrid.c:1227-1263), inflow cells, no evaporation/rain */
static void volume_by_flux(oracle_domain *d) {
  const double q = series_at(d->inflow, d->ninflow, d->tt);
  for (long ii = 0; ii < d->N; ++ii) {
    d->cellV[ii] = d->cellV[ii] + d->c.dt * (d->Fuu[d->iMjc[ii]] - d->Fuu[ii] +
                                             d->Fvv[d->icjM[ii]] - d->Fvv[ii]);
    if (is_inflow(d, ii)) d->cellV[ii] = d->cellV[ii] + q * d->c.dt;
    if (d->cellV[ii] < 0) d->cellV[ii] = 0;
  }
}

/* updateData (nssolve.c:181-290), subgrid path */
static void update_data(oracle_domain *d) {
  limiter_cfl(d);
  /* computeVolumeSub (subgrid.c:1215-1224) */
  for (long ii = 0; ii < d->N; ++ii) {
    d->cellV[ii] = d->V[ii];
    if (d->c.useScalar) d->Sm[ii] = d->S[ii] * d->cellV[ii];
  }
  compute_sub_area(d);
  combine_sub_area(d);
  update_depth(d);
  update_face_depth(d);
  detect_waterfall(d);
  update_velocity(d);
  waterfall_correction(d);
  enforce_vel_bc(d);
  /* computeFaceFlowRateSub (subgrid.c:1190-1212) */
  for (long k = 0; k < d->T; ++k) {
    d->Fuu[k] = d->uuXP[k] * d->Nx[k];
    d->Fvv[k] = d->vvYP[k] * d->Oy[k];
  }
  tidal_velocity(d);
  velocity_interp(d);
  volume_by_flux(d);
  update_cd(d);
  if (d->c.useThinLayer) thin_layer_drag(d);
}

/* ------------------------------------------------------------- scalar */
/* The superbee limiter of scalar.c:115-119 (and its three repetitions). */
static double superbee(double r) {
  double p1, p2, phi;
  if (2 * r > 1) p1 = 1; else p1 = 2 * r;
  if (r > 2) p2 = 2; else p2 = r;
  if (p1 > 0) phi = p1; else phi = 0;
  if (p2 > phi) phi = p2;
  return phi;
}

static void scalar_transport(oracle_domain *d) {
  const long N = d->N;
  const double dt = d->c.dt, dx = d->c.dx, dy = d->c.dy, Kx = d->c.Kx, Ky = d->c.Ky;
  double *S = d->S, *Sm = d->Sm, *F = d->Fuu, *G = d->Fvv;
  if (d->c.scalarAdv == 2) {
    /* scalarAdvection, TVD with the superbee limiter (scalar.c:99-249), term by
     * term: first-order upwind where the stencil reaches a face without flow
     * toward the cell, r = 0 below dSmin; the YM Courant number uses dx
     * (scalar.c:214). */
    const double dSmin = 0.00001;
    for (long ii = 0; ii < N; ++ii) {
      const int e = d->iPjc[ii], w = d->iMjc[ii], n = d->icjP[ii], s = d->icjM[ii];
      const int ee = d->iPPjc[ii], ww = d->iMMjc[ii], nn = d->icjPP[ii], ss = d->icjMM[ii];
      double Sd, Su, Sr, Sl, Cu, r;
      /* XP face */
      Cu = d->uuXP[ii] * dt / dx;
      if (F[ii] > 0) {
        if (F[w] <= 0) Sd = S[ii];
        else {
          if (fabs(S[e] - S[ii]) < dSmin) r = 0;
          else r = (S[ii] - S[w]) / (S[e] - S[ii]);
          Sd = S[ii] + 0.5 * superbee(r) * (S[e] - S[ii]) * Cu * (1 - Cu);
        }
      } else {
        if (F[e] >= 0) Sd = S[e];
        else {
          if (fabs(S[e] - S[ii]) < dSmin) r = 0;
          else r = (S[e] - S[ee]) / (S[ii] - S[e]);
          Sd = S[e] + 0.5 * superbee(r) * (S[ii] - S[e]) * Cu * (1 - Cu);
        }
      }
      /* XM face */
      Cu = d->uuXP[w] * dt / dx;
      if (F[w] > 0) {
        if (F[ww] <= 0) Su = S[w];
        else {
          if (fabs(S[ii] - S[w]) < dSmin) r = 0;
          else r = (S[w] - S[ww]) / (S[ii] - S[w]);
          Su = S[w] + 0.5 * superbee(r) * (S[ii] - S[w]) * Cu * (1 - Cu);
        }
      } else {
        if (F[ii] >= 0) Su = S[ii];
        else {
          if (fabs(S[ii] - S[w]) < dSmin) r = 0;
          else r = (S[ii] - S[e]) / (S[w] - S[ii]);
          Su = S[ii] + 0.5 * superbee(r) * (S[w] - S[ii]) * Cu * (1 - Cu);
        }
      }
      /* YP face */
      Cu = d->vvYP[ii] * dt / dy;
      if (G[ii] > 0) {
        if (G[s] <= 0) Sr = S[ii];
        else {
          if (fabs(S[n] - S[ii]) < dSmin) r = 0;
          else r = (S[ii] - S[s]) / (S[n] - S[ii]);
          Sr = S[ii] + 0.5 * superbee(r) * (S[n] - S[ii]) * Cu * (1 - Cu);
        }
      } else {
        if (G[n] >= 0) Sr = S[n];
        else {
          if (fabs(S[n] - S[ii]) < dSmin) r = 0;
          else r = (S[n] - S[nn]) / (S[ii] - S[n]);
          Sr = S[n] + 0.5 * superbee(r) * (S[ii] - S[n]) * Cu * (1 - Cu);
        }
      }
      /* YM face */
      Cu = d->vvYP[s] * dt / dx;
      if (G[s] > 0) {
        if (G[ss] <= 0) Sl = S[s];
        else {
          if (fabs(S[ii] - S[s]) < dSmin) r = 0;
          else r = (S[s] - S[ss]) / (S[ii] - S[s]);
          Sl = S[s] + 0.5 * superbee(r) * (S[ii] - S[s]) * Cu * (1 - Cu);
        }
      } else {
        if (G[ii] >= 0) Sl = S[ii];
        else {
          if (fabs(S[ii] - S[s]) < dSmin) r = 0;
          else r = (S[ii] - S[n]) / (S[s] - S[ii]);
          Sl = S[ii] + 0.5 * superbee(r) * (S[s] - S[ii]) * Cu * (1 - Cu);
        }
      }
      Sm[ii] = Sm[ii] + dt * (-F[ii] * Sd + F[w] * Su - G[ii] * Sr + G[s] * Sl);
    }
  } else {
    /* scalarAdvection, first-order upwind (scalar.c:72-97) */
    for (long ii = 0; ii < N; ++ii) {
      const int e = d->iPjc[ii], w = d->iMjc[ii], n = d->icjP[ii], s = d->icjM[ii];
      double Sd = F[ii] > 0 ? S[ii] : S[e];
      double Su = F[w] > 0 ? S[w] : S[ii];
      double Sr = G[ii] > 0 ? S[ii] : S[n];
      double Sl = G[s] > 0 ? S[s] : S[ii];
      Sm[ii] = Sm[ii] + dt * (-F[ii] * Sd + F[w] * Su - G[ii] * Sr + G[s] * Sl);
    }
  }
  /* scalarDiffusionSub (subgrid.c:1552-1567) */
  for (long ii = 0; ii < N; ++ii) {
    const int e = d->iPjc[ii], w = d->iMjc[ii], n = d->icjP[ii], s = d->icjM[ii];
    Sm[ii] = Sm[ii] + dt * ((Kx * d->Nx[ii] / dx) * (S[e] - S[ii]) -
                            (Kx * d->Nx[w] / dx) * (S[ii] - S[w]) +
                            (Ky * d->Oy[ii] / dy) * (S[n] - S[ii]) -
                            (Ky * d->Oy[s] / dy) * (S[ii] - S[s]));
  }
  /* updateScalarSub (subgrid.c:1570-1713), one rank */
  int *cnt = iz(N);
  double *smax = dz(N), *smin = dz(N);
  for (long ii = 0; ii < N; ++ii) {
    const int e = d->iPjc[ii], w = d->iMjc[ii], n = d->icjP[ii], s = d->icjM[ii];
    double vals[4];
    int c = 0;
    if (d->Nx[ii] > 0 && d->surfOld[e] - d->bottomZ[e] > 0) vals[c++] = S[e];
    if (d->Nx[w] > 0 && d->surfOld[w] - d->bottomZ[w] > 0) vals[c++] = S[w];
    if (n <= N && d->Oy[ii] > 0 && d->surfOld[n] - d->bottomZ[n] > 0) vals[c++] = S[n];
    if (s <= N && d->Oy[s] > 0 && d->surfOld[s] - d->bottomZ[s] > 0) vals[c++] = S[s];
    cnt[ii] = c;
    if (c) {
      double mx = vals[0], mn = vals[0];
      for (int q = 1; q < c; ++q) {
        if (vals[q] > mx) mx = vals[q];
        if (vals[q] < mn) mn = vals[q];
      }
      smax[ii] = mx;
      smin[ii] = mn;
    }
  }
  /* scalar from inflow (subgrid.c:1648-1654); inflow cells skip the limiter */
  if (d->c.inflowLocLength) {
    const double q = series_at(d->inflow, d->ninflow, d->tt);
    for (long ii = 0; ii < N; ++ii)
      if (is_inflow(d, ii))
        Sm[ii] = Sm[ii] + d->c.inflowS * q * dt / d->c.inflowLocLength;
  }
  for (long ii = 0; ii < N; ++ii) {
    S[ii] = d->cellV[ii] > 0 ? Sm[ii] / d->cellV[ii] : 0;
    const int flag = is_inflow(d, ii);
    if (cnt[ii] != 0 && S[ii] > smax[ii] && !flag) S[ii] = smax[ii];
    else if (cnt[ii] != 0 && S[ii] < smin[ii] && !flag) S[ii] = smin[ii];
  }
  free(cnt); free(smax); free(smin);
  for (long ii = 0; ii < N; ++ii)
    if (S[ii] > 100 || S[ii] < 0) {
      if (!(d->icjM[ii] > N) && !(d->icjP[ii] > N)) {
        S[ii] = 0;
        d->surf[ii] = d->surf[ii] - d->depth[ii];
        d->depth[ii] = 0;
      }
    }
  /* enforceScalarBC (scalar.c:419-471) */
  for (int i = 0; i < d->nx; ++i) { S[d->jPgt[i]] = S[d->jPbd[i]]; S[d->jMgt[i]] = S[d->jMbd[i]]; }
  for (int j = 0; j < d->ny; ++j) { S[d->iPgt[j]] = S[d->iPbd[j]]; S[d->iMgt[j]] = S[d->iMbd[j]]; }
  for (int k = 0; k < d->c.tideLocLengthP; ++k) S[tide_cell(d, k)] = d->c.tidePS;
  for (long ii = 0; ii < N; ++ii)
    if (d->depth[ii] <= 0) S[ii] = 0;
}

/* monitorCFL (nsfunctions.c:1192-1232) without printing; returns max CFL */
static double monitor_cfl(oracle_domain *d) {
  double mx = 0, my = 0;
  for (long ii = 0; ii < d->N; ++ii) {
    d->CFLx[ii] = fabs(d->uuXP[ii]) * d->c.dt / d->c.dx;
    d->CFLy[ii] = fabs(d->vvYP[ii]) * d->c.dt / d->c.dy;
    if (d->CFLx[ii] > mx) mx = d->CFLx[ii];
    if (d->CFLy[ii] > my) my = d->CFLy[ii];
  }
  return mx > my ? mx : my;
}

/* getFreeSurface .. enforceTidalBC (nsfunctions.c:1020-1031; nssolve.c:169-177),
 * updateData, scalarTransport and monitorCFL.  x: transposed order. */
double oracle_update(oracle_domain *d, int tt, const double *x) {
  d->tt = tt;
  for (long k = 0; k < d->T; ++k) d->surfOld[k] = d->surf[k];
  for (long k = 0; k < d->N; ++k) d->surf[d->trps[k]] = x[k];
  zero_neg_surf(d, tt);
  enforce_surf_bc(d);
  enforce_tidal_bc(d, tt);
  update_data(d);
  if (d->c.useScalar) scalar_transport(d);
  return monitor_cfl(d);
}

double oracle_step(oracle_domain *d, int tt) {
  oracle_explicit(d, tt);
  oracle_solve(d);
  return oracle_update(d, tt, d->x);
}

const double *oracle_solution(const oracle_domain *d) { return d->x; }

/* ------------------------------------------------------------- access */
typedef struct { const char *name; int kind; } field_desc; /* kind: 0 N, 1 T */

static void *field_ptr(oracle_domain *d, const char *name, long *n, int *is_int) {
  *is_int = 0;
#define F(nm, len) if (!strcmp(name, #nm)) { *n = len; return d->nm; }
  F(uuXP, d->T) F(uuYP, d->N) F(vvXP, d->N) F(vvYP, d->T) F(surf, d->T) F(surfOld, d->T)
  F(Fuu, d->T) F(Fvv, d->T) F(cellV, d->N) F(depth, d->N) F(depthXP, d->T) F(depthYP, d->T)
  F(EnXP, d->T) F(EnYP, d->T) F(DragXP, d->T) F(DragYP, d->T) F(CDXP, d->T) F(CDYP, d->T)
  F(GnCt, d->N) F(GnXP, d->N) F(GnYP, d->N) F(GnXM, d->N) F(GnYM, d->N) F(z, d->N)
  F(wtfXP, d->T) F(wtfYP, d->T) F(S, d->T) F(Sm, d->N) F(rmvCFL, d->N) F(advX, d->T)
  F(advY, d->T) F(CFLx, d->T) F(CFLy, d->T) F(V, d->T) F(Z, d->T) F(Vxp, d->T) F(Vyp, d->T)
  F(Vxm, d->T) F(Vym, d->T) F(Np, d->T) F(Nm, d->T) F(Op, d->T) F(Om, d->T) F(Nx, d->T)
  F(Oy, d->T) F(Vx, d->T) F(Vy, d->T) F(Zx, d->T) F(Zy, d->T) F(bottomZ, d->T)
  F(bottomXP, d->T) F(bottomYP, d->T) F(edgeX, d->N) F(edgeY, d->N) F(x, d->N)
#undef F
  if (!strcmp(name, "ind")) { *n = d->T; *is_int = 1; return d->ind; }
  if (!strcmp(name, "Vloss")) { *n = 4; return d->Vloss; }
  return NULL;
}

long oracle_field_len(oracle_domain *d, const char *name) {
  long n = -1;
  int is_int;
  if (!field_ptr(d, name, &n, &is_int)) return -1;
  return n;
}

int oracle_get(oracle_domain *d, const char *name, double *out, long n) {
  long len;
  int is_int;
  void *p = field_ptr(d, name, &len, &is_int);
  if (!p || n != len) FAIL("get %s: unknown field or length %ld != %ld", name, n, len);
  if (is_int) for (long k = 0; k < n; ++k) out[k] = ((int *)p)[k];
  else memcpy(out, p, (size_t)n * sizeof(double));
  return 0;
}

int oracle_set(oracle_domain *d, const char *name, const double *in, long n) {
  long len;
  int is_int;
  void *p = field_ptr(d, name, &len, &is_int);
  if (!p || n != len) FAIL("set %s: unknown field or length %ld != %ld", name, n, len);
  if (is_int) for (long k = 0; k < n; ++k) ((int *)p)[k] = (int)in[k];
  else memcpy(p, in, (size_t)n * sizeof(double));
  return 0;
}

// Stencil kernels of one FrehdC step (plain FP64 form).
//
// Every expression keeps the reference's evaluation order and this file is
// built with --fmad=false, so the doubles produced here equal those of the
// reference's sequential loops (reference functions cited per block).  The
// reference's order-dependent loops are restated in closed form where they are
// order dependent only through a fixed neighbour set (the advection CFL limiter,
// the dry-cell outflow rule, the waterfall flag precedence).
//
// Kernels per step (after the persistent CG in cg.cu):
//   k_explicit   solveSourceTerm + matrixCoeffSub + adjustMatrixBoundary +
//                adjustTidalBoundary (nssolve.c:121-166)
//   k_update_geo getFreeSurface .. enforceTidalBC, limiterCFL, computeSubArea,
//                combineSubArea, updateDepth (nssolve.c:169-225)
//   k_update_vel detectWaterfall .. thinLayerDrag, scalarTransport, monitorCFL
//                (nssolve.c:237-290, scalar.c:30-57, nsfunctions.c:1192-1232)
//   k_finish     scalar-singularity surface fix-up, step statistics
#include <cmath>

#include "domain.cuh"
#include "kernels.cuh"
#include "subgrid_levels.h"

namespace frehd {

// ---------------------------------------------------------------- helpers
// Thread-block tile of the stencil kernels: 32 cells along x (one warp) by 8 rows.
constexpr int TBX = 32, TBY = 8, EX = TBX + 1, EY = TBY + 1;

__device__ __forceinline__ double rd(const double *a, const Grid &g, int i, int j) {
  return a[g.at(i, j)];
}

// velocityInterp (nsfunctions.c:337-347): the reference indexes the linear
// array directly, so "ii - 1" of the first column is the last cell of the
// previous row, "ii + nx" of the last row is the north ghost row, and indices
// before the array start read 0.
__device__ __forceinline__ double uuYP_at(const View &w, int i, int j) {
  const Grid &g = w.gr;
  const double a = rd(w.u, g, i, j);
  const double b = (i > 0) ? rd(w.u, g, i - 1, j) : (j > 0 ? rd(w.u, g, g.nx - 1, j - 1) : 0.0);
  const double c = rd(w.u, g, i, j + 1);
  const double d = (i > 0) ? rd(w.u, g, i - 1, j + 1) : rd(w.u, g, g.nx - 1, j);
  return 0.25 * (a + b + c + d);
}

__device__ __forceinline__ double vvXP_at(const View &w, int i, int j) {
  const Grid &g = w.gr;
  const double a = rd(w.v, g, i, j);
  const double b = (i < g.nx - 1) ? rd(w.v, g, i + 1, j) : rd(w.v, g, 0, j + 1);
  const double c = (j > 0) ? rd(w.v, g, i, j - 1) : 0.0;
  const double d = (i < g.nx - 1) ? (j > 0 ? rd(w.v, g, i + 1, j - 1) : 0.0) : rd(w.v, g, 0, j);
  return 0.25 * (a + b + c + d);
}

struct Ex {
  double En, Drag;
};

// windTerm (nsfunctions.c:609-648) of cell k: the stress (the same for both
// faces) and the cosine and sine of the step's wind direction, which the host
// takes with its libm as the reference does (frehd_domain_set_series).
struct Wind {
  double tau, c, s;
};

__device__ __forceinline__ Wind wind_at(const View &w, long k) {
  const Params &p = w.p;
  const int tt = w.sc->tt;
  const double W = (tt >= 0 && tt < w.nwspd) ? w.wspd[tt] : 0.0;
  const int q = (tt >= 0 && tt < w.nwdir) ? tt : w.nwdir;
  Wind r;
  r.c = w.wcos[q];
  r.s = w.wsin[q];
  const double a = W - w.u[k] * r.c - w.v[k] * r.s;
  r.tau = p.rhoa * p.Cw * a * a;
  return r;
}

// The face's share: the thin-layer decay below hD (the reference's depth test),
// no stress on a dry face.
__device__ __forceinline__ double wind_face(const Params &p, double tau, double h) {
  return (h < p.hD && p.useThinLayer == 1) ? tau * exp(p.CwT * (h - p.hD) / p.hD) : tau;
}

// One cell's x-momentum source: explicitVelocity, advectionTerm with the CFL
// limiter (nsfunctions.c:498-586), diffusionTermSub (subgrid.c:781-812),
// dragTermSub with staggeredV = 1 (subgrid.c:857-927) and dragInversion
// (nsfunctions.c:730-746).  The limiter scales advX[k] once for each cell of
// the sweep that reaches k before k's own update: k - nx, k - 1, then k.
__device__ Ex explicit_x(const View &w, int i, int j) {
  const Params &p = w.p;
  const Grid &g = w.gr;
  const long k = g.at(i, j);
  const double *u = w.u;
  const double u0 = u[k], uE = rd(u, g, i + 1, j), uW = rd(u, g, i - 1, j);
  const double uN = rd(u, g, i, j + 1), uS = rd(u, g, i, j - 1);
  const double vX = vvXP_at(w, i, j);
  double ax = (0.5 / p.dx) * (u0 + fabs(u0)) * (u0 - uW) + (0.5 / p.dx) * (u0 - fabs(u0)) * (uE - u0) +
              (0.5 / p.dy) * (vX + fabs(vX)) * (u0 - uS) + (0.5 / p.dy) * (vX - fabs(vX)) * (uN - u0);
  if (u0 == 0) ax = 0;
  const double ck = w.CFLx[k];
  const double den = p.CFLh - p.CFLl;
#define FREHD_LIMIT_X(cc)                                              \
  {                                                                    \
    const double c_ = (cc);                                            \
    if (c_ > p.CFLl && c_ <= p.CFLh) ax = ax * (p.CFLh - ck) / den;    \
    else if (c_ > p.CFLh) ax = 0;                                      \
  }
  if (j > 0) FREHD_LIMIT_X(rd(w.CFLx, g, i, j - 1));
  if (i > 0) FREHD_LIMIT_X(rd(w.CFLx, g, i - 1, j));
  FREHD_LIMIT_X(ck);
#undef FREHD_LIMIT_X
  double En = u0 - p.dt * ax;
  const double Vx = w.Vx[k];
  double fx = 0;
  if (Vx > 0) {
    fx = (p.NUx / Vx) * (rd(w.Nx, g, i + 1, j) * (uE - u0) / p.dx - w.Nx[k] * (-uW + u0) / p.dx) +
         (p.NUy / Vx) * (w.Oy[k] * (uN - u0) / p.dy - rd(w.Oy, g, i, j - 1) * (-uS + u0) / p.dy);
  }
  En = En + p.dt * fx;
  if (p.useWind) {
    const Wind wd = wind_at(w, k);
    const double h = w.dXP[k];
    if (h > 0) En = En + p.dt * wind_face(p, wd.tau, h) * wd.c / (h * 1000.0);
  }
  const double velx = sqrt(u0 * u0 + vX * vX);
  const double hx = Vx > 0 ? w.Zx[k] / Vx : 0;
  Ex r;
  r.Drag = 0.5 * p.dt * w.CDXP[k] * velx * hx;
  r.En = En / (1 + r.Drag);
  return r;
}

// y-momentum counterpart.  The y limiter uses a strict upper bound and its
// zeroing branch tests CFLx, not CFLy (nsfunctions.c:561,574).
__device__ Ex explicit_y(const View &w, int i, int j) {
  const Params &p = w.p;
  const Grid &g = w.gr;
  const long k = g.at(i, j);
  const double *v = w.v;
  const double v0 = v[k], vE = rd(v, g, i + 1, j), vW = rd(v, g, i - 1, j);
  const double vN = rd(v, g, i, j + 1), vS = rd(v, g, i, j - 1);
  const double uY = uuYP_at(w, i, j);
  double ay = (0.5 / p.dx) * (uY + fabs(uY)) * (v0 - vW) + (0.5 / p.dx) * (uY - fabs(uY)) * (vE - v0) +
              (0.5 / p.dy) * (v0 + fabs(v0)) * (v0 - vS) + (0.5 / p.dy) * (v0 - fabs(v0)) * (vN - v0);
  if (v0 == 0) ay = 0;
  const double ck = w.CFLy[k];
  const double den = p.CFLh - p.CFLl;
#define FREHD_LIMIT_Y(ii_, jj_)                                        \
  {                                                                    \
    const long c_ = g.at(ii_, jj_);                                    \
    const double cy_ = w.CFLy[c_];                                     \
    if (cy_ > p.CFLl && cy_ < p.CFLh) ay = ay * (p.CFLh - ck) / den;   \
    else if (w.CFLx[c_] > p.CFLh) ay = 0;                              \
  }
  if (j > 0) FREHD_LIMIT_Y(i, j - 1);
  if (i > 0) FREHD_LIMIT_Y(i - 1, j);
  FREHD_LIMIT_Y(i, j);
#undef FREHD_LIMIT_Y
  double En = v0 - p.dt * ay;
  const double Vy = w.Vy[k];
  double fy = 0;
  if (Vy > 0) {
    fy = (p.NUx / Vy) * (w.Nx[k] * (vE - v0) / p.dx - rd(w.Nx, g, i - 1, j) * (-vW + v0) / p.dx) +
         (p.NUy / Vy) * (rd(w.Oy, g, i, j + 1) * (vN - v0) / p.dy - w.Oy[k] * (-vS + v0) / p.dy);
  }
  En = En + p.dt * fy;
  if (p.useWind) {  // the y term is subtracted (nsfunctions.c:642-645)
    const Wind wd = wind_at(w, k);
    const double h = w.dYP[k];
    if (h > 0) En = En - p.dt * wind_face(p, wd.tau, h) * wd.s / (h * 1000.0);
  }
  const double vely = sqrt(uY * uY + v0 * v0);
  const double hy = Vy > 0 ? w.Zy[k] / Vy : 0;
  Ex r;
  r.Drag = 0.5 * p.dt * w.CDYP[k] * vely * hy;
  r.En = En / (1 + r.Drag);
  return r;
}

// Face coefficient of matrixCoeffSub (subgrid.c:1012-1019); the same double
// from either side of the face.
__device__ __forceinline__ double gface(double coef, double N, double Vf, double Drag) {
  return Vf > 0 ? coef * N * N / Vf / 1.0 / (1 + Drag) : 0.0;
}

// ---------------------------------------------------------------- k_explicit
// Writes EnXP/EnYP, the face coefficients Gx (east face) and Gy (north face),
// the row diagonal Ct (negated for rows the reference decouples: tidal rows and
// closed dry cells) and the right-hand side b, all in the padded layout.
// A 32 x 8 block evaluates the explicit term of every x face and y face it
// needs once: each thread its own east and north face, threads 0-31 the south
// halo row's north faces and threads 32-39 the west halo column's east faces.
static __device__ __forceinline__ void explicit_tile(const View &w, int bx, int by) {
  const Params &p = w.p;
  const Grid &g = w.gr;
  __shared__ double sEx[TBY][TBX + 1], sDx[TBY][TBX + 1];  // x faces, column 0 = west halo
  __shared__ double sEy[TBY + 1][TBX], sDy[TBY + 1][TBX];  // y faces, row 0 = south halo
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TBX + tx;
  const int i0 = bx * TBX, j0 = by * TBY;
  const int i = i0 + tx, j = j0 + ty;
  const bool in = i < g.nx && j < g.ny;
  Ex ex{0.0, 0.0}, ey{0.0, 0.0};
  if (in) {
    ex = explicit_x(w, i, j);
    ey = explicit_y(w, i, j);
  }
  sEx[ty][tx + 1] = ex.En;
  sDx[ty][tx + 1] = ex.Drag;
  sEy[ty + 1][tx] = ey.En;
  sDy[ty + 1][tx] = ey.Drag;
  if (tid < TBX) {  // north faces of the row below the block (ghosts never written: 0)
    Ex e{0.0, 0.0};
    if (i0 + tid < g.nx && j0 > 0 && j0 - 1 < g.ny) e = explicit_y(w, i0 + tid, j0 - 1);
    sEy[0][tid] = e.En;
    sDy[0][tid] = e.Drag;
  } else if (tid < TBX + TBY) {  // east faces of the column left of the block
    const int t = tid - TBX;
    Ex e{0.0, 0.0};
    if (i0 > 0 && j0 + t < g.ny) e = explicit_x(w, i0 - 1, j0 + t);
    sEx[t][0] = e.En;
    sDx[t][0] = e.Drag;
  }
  __syncthreads();
  if (!in) return;
  const long k = g.at(i, j);
  const double EnW = sEx[ty][tx], DrW = sDx[ty][tx];  // i = 0: the halo holds 0
  const double EnS = sEy[ty][tx], DrS = sDy[ty][tx];  // j = 0: the halo holds 0
  w.EnXP[k] = ex.En;
  w.EnYP[k] = ey.En;
  if (j == 0) w.EnXP[g.at(i, -1)] = ex.En;  // dragInversion ghost copies
  if (i == 0) w.EnYP[g.at(-1, j)] = ey.En;

  const double coef = p.g * (p.dt * p.dt);
  const double NxW = rd(w.Nx, g, i - 1, j), OyS = rd(w.Oy, g, i, j - 1);
  double GnXP = gface(coef, w.Nx[k], w.Vx[k], ex.Drag);
  double GnXM = gface(coef, NxW, rd(w.Vx, g, i - 1, j), DrW);
  double GnYP = gface(coef, w.Oy[k], w.Vy[k], ey.Drag);
  double GnYM = gface(coef, OyS, rd(w.Vy, g, i, j - 1), DrS);
  const double gxe = GnXP, gyn = GnYP;
  const double dxdy = p.dx * p.dy;
  double Ct = w.Z[k] + GnXP + GnYP + GnXM + GnYM;
  // matrixSourceTermSub (subgrid.c:934-974) with its inflow cells (:959-968)
  const double s = w.surf_cur[k];
  double b = s * w.Z[k] - p.dt * (ex.En * w.Nx[k] - EnW * NxW) - p.dt * (ey.En * w.Oy[k] - EnS * OyS);
  if (is_inflow(p, i, j)) b = b + p.dt * (inflow_value(w) / p.inflowLen);
  if (b == 0 || b == s * p.dx * p.dy) b = s * p.dx * p.dy;
  // matrixCoeffSub singular-row guards (subgrid.c:1061-1078)
  if (Ct == 0.0 || Ct == dxdy) Ct = dxdy;
  bool iso = false;
  if (w.depth_cur[k] == 0 && w.u[k] == 0 && rd(w.u, g, i - 1, j) == 0 && w.v[k] == 0 &&
      rd(w.v, g, i, j - 1) == 0) {
    Ct = dxdy;
    GnXM = 0.0; GnXP = 0.0; GnYM = 0.0; GnYP = 0.0;
    b = s * p.dx * p.dy;
    iso = true;
  }
  // adjustMatrixBoundary (nsfunctions.c:846-884), one rank
  if (i == 0) { Ct = Ct - GnXM; GnXM = 0; }
  if (i == g.nx - 1) { Ct = Ct - GnXP; GnXP = 0; }
  if (j == 0) { Ct = Ct - GnYM; GnYM = 0; }
  if (j == g.ny - 1) { Ct = Ct - GnYP; GnYP = 0; }
  // adjustTidalBoundary (nsfunctions.c:887-905)
  if (is_tidal(p, i, j)) {
    Ct = 1;
    b = tide_value(w) + p.offset;
    iso = true;
  }
  w.Gx[k] = (i == g.nx - 1) ? 0.0 : gxe;
  w.Gy[k] = (j == g.ny - 1) ? 0.0 : gyn;
  w.Ct[k] = iso ? -Ct : Ct;
  w.b[k] = b;
}

// Six blocks per SM (40 registers, a few spills): the explicit terms wait on
// their neighbour loads and IEEE divisions, and the extra warps hide them --
// 1.58 ms per 4096^2 step against 1.83 at four blocks and 1.68 at five.
constexpr int kExplicitMinBlocks = 6;

__global__ void __launch_bounds__(TBX *TBY, kExplicitMinBlocks) k_explicit(View w) {
  if (*(volatile int *)&w.sc->status != FREHD_OK) return;  // a fatal step stops the run
  explicit_tile(w, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------- subgrid
__device__ __forceinline__ double interp_surf(double x, double x1, double y1, double x2, double y2) {
  // interpSurf (utilities.c:155-162)
  if (x2 == x1) return y1;
  return (y2 - y1) * (x - x2) / (x2 - x1) + y2;
}

__device__ __forceinline__ double level_surf(const Params &p, int k) {
  return frehd_level(p.surfmin, p.dsurf, k) + p.offset;  // subgrid.c:2118
}

// Table values of cell (i, j) at level k: all ten, or (part) only the west- or
// south-face pair.  bz: the cell's bottom with the offset (the minimum of its
// fine bottoms): a level below it leaves every fine depth zero, and then every
// value is +0, exactly what the evaluation would add up (the margin covers the
// two roundings of the offset).
__device__ __forceinline__ bool level_dry(const Params &p, int k, double bz) {
  return frehd_level(p.surfmin, p.dsurf, k) + p.offset < bz - 1e-9;
}

__device__ __forceinline__ void level_values(const Params &p, int i, int j, int k, frehd_cell_levels *o,
                                             int part, double bz) {
  if (p.geom_fine) {
    if (level_dry(p, k, bz)) {
      o->V = o->Z = o->Vxp = o->Vxm = o->Vyp = o->Vym = 0.0;
      o->Np = o->Nm = o->Op = o->Om = 0.0;
    } else if (p.r == 4 && !p.check_block)
      frehd_cell_levels_r4(p.zf, p.fpitch, p.nx, p.ny, i, j, frehd_level(p.surfmin, p.dsurf, k),
                           p.dxf * p.dyf, p.dxf, part, o);
    else  // every value (a part's caller reads only its own)
      frehd_cell_levels_at(p.zf, p.fpitch, p.nx, p.ny, p.r, i, j, frehd_level(p.surfmin, p.dsurf, k),
                           p.dxf * p.dyf, p.dxf, p.check_block, o);
  } else {
    const long N = (long)p.nx * p.ny, T = N * p.Ne;
    const double *t = p.tab + (long)k * N + (long)j * p.nx + i;
    o->V = t[0]; o->Z = t[T]; o->Vxp = t[2 * T]; o->Vxm = t[3 * T]; o->Vyp = t[4 * T];
    o->Vym = t[5 * T]; o->Np = t[6 * T]; o->Nm = t[7 * T]; o->Op = t[8 * T]; o->Om = t[9 * T];
  }
}

__device__ __forceinline__ int ld_acquire(const int *a) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(a) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int *a, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(a), "r"(v) : "memory");
}

// level_values through the domain's level-value cache (fine geometry).  The
// values of a level depend on the fine bottoms alone, and the two levels a
// cell interpolates between are consecutive, so one even and one odd: each
// cell keeps the last level of each parity it evaluated (slot = level & 1).
// PART = FREHD_LV_ALL is the cell's own thread: on a miss it evaluates the
// level, stores the ten values and then publishes the index (release); no
// other thread writes the entry.  A halo evaluation (WEST / SOUTH) of another
// block's cell takes the entry only if the index it acquires is the level it
// needs -- then the values are the ones published with it -- and otherwise
// evaluates the level itself.  Either way the doubles are the same.
template <int PART>
__device__ __forceinline__ void cell_level(const View &w, int i, int j, long k, int lev,
                                           frehd_cell_levels *o, double bz) {
  const Params &p = w.p;
  if (!p.geom_fine || !w.lvc || level_dry(p, lev, bz)) {
    level_values(p, i, j, lev, o, PART, bz);
    return;
  }
  const long T = w.gr.total;
  const int slot = lev & 1;
  int *ip = w.lvi + slot * T + k;
  double *c = w.lvc + (long)slot * 10 * T + k;
  if (PART == FREHD_LV_ALL) {
    if (*ip == lev) {
      o->V = c[0]; o->Z = c[T]; o->Vxp = c[2 * T]; o->Vxm = c[3 * T]; o->Vyp = c[4 * T];
      o->Vym = c[5 * T]; o->Np = c[6 * T]; o->Nm = c[7 * T]; o->Op = c[8 * T]; o->Om = c[9 * T];
      return;
    }
    level_values(p, i, j, lev, o, FREHD_LV_ALL, bz);
    c[0] = o->V; c[T] = o->Z; c[2 * T] = o->Vxp; c[3 * T] = o->Vxm; c[4 * T] = o->Vyp;
    c[5 * T] = o->Vym; c[6 * T] = o->Np; c[7 * T] = o->Nm; c[8 * T] = o->Op; c[9 * T] = o->Om;
    st_release(ip, lev);
  } else {
    if (ld_acquire(ip) == lev) {
      if (PART == FREHD_LV_WEST) {
        o->Vxm = __ldcg(c + 3 * T);
        o->Nm = __ldcg(c + 7 * T);
      } else {
        o->Vym = __ldcg(c + 5 * T);
        o->Om = __ldcg(c + 9 * T);
      }
      return;
    }
    level_values(p, i, j, lev, o, PART, bz);
  }
}

struct SubCell {
  double V, Z, Vxp, Vxm, Vyp, Vym, Np, Nm, Op, Om;
};

// computeSubArea for one cell (subgrid.c:87-249) with useSubDrag = 0 and
// useminA = 0; the minV* interpolations feed only useminV = 1/2 and are skipped.
// PART = FREHD_LV_ALL computes every value; FREHD_LV_WEST only Nm and Vxm,
// FREHD_LV_SOUTH only Om and Vym (what the west/south neighbour's face needs).
template <int PART>
__device__ SubCell compute_sub_area(const View &w, int i, int j, double s, int *ind_io,
                                    double depth_old) {
  const Params &p = w.p;
  const Grid &g = w.gr;
  const double ds = p.dsurf;
  const double thr = 0.5 * ds + ds / 100;
  int ind = *ind_io;
  for (int guard = 0; guard <= p.Ne + 1 && fabs(level_surf(p, ind) - s) > thr; ++guard) {
    if (s > level_surf(p, ind)) ind += 1; else ind -= 1;
    if (ind < 0) { ind = 0; break; }
    if (ind > p.Ne - 1) { ind = p.Ne - 1; break; }
  }
  *ind_io = ind;
  const int j1 = ind;
  int j2;
  if (j1 == 0) j2 = 0;
  else if (j1 == p.Ne - 1) j2 = p.Ne - 1;
  else j2 = s > level_surf(p, j1) ? j1 + 1 : j1 - 1;
  const double a1 = level_surf(p, j1), a2 = level_surf(p, j2);
  frehd_cell_levels L1, L2;
  const long kc = g.at(i, j);
  const double bzc = w.bottomZ[kc];
  cell_level<PART>(w, i, j, kc, j1, &L1, bzc);
  if (j2 != j1) cell_level<PART>(w, i, j, kc, j2, &L2, bzc); else L2 = L1;
  SubCell c;
#define FREHD_FACE(out, wd, f)                                                         \
  {                                                                                    \
    const double wd_ = (wd);                                                           \
    if (wd_ > a1 && wd_ < a2) out = wd_ > s ? 0.0 : interp_surf(s, wd_, 0.0, a2, L2.f); \
    else out = interp_surf(s, a1, L1.f, a2, L2.f);                                     \
  }
  if (PART == FREHD_LV_ALL) {
    c.V = interp_surf(s, a1, L1.V, a2, L2.V);
    c.Z = interp_surf(s, a1, L1.Z, a2, L2.Z);
    c.Vxp = interp_surf(s, a1, L1.Vxp, a2, L2.Vxp);
    c.Vyp = interp_surf(s, a1, L1.Vyp, a2, L2.Vyp);
    const double bxp = rd(w.bottomXP, g, i, j), byp = rd(w.bottomYP, g, i, j);
    FREHD_FACE(c.Np, bxp, Np);
    FREHD_FACE(c.Op, byp, Op);
    if (depth_old == 0) { c.Vxp = 0; c.Vyp = 0; }
    if (s - bxp <= 0) c.Np = 0;
    if (s - byp <= 0) c.Op = 0;
  }
  if (PART != FREHD_LV_SOUTH) {
    c.Vxm = interp_surf(s, a1, L1.Vxm, a2, L2.Vxm);
    const double bxm = i > 0 ? rd(w.bottomXP, g, i - 1, j) : 0.0;  // edgeX is N-sized: ghost reads 0
    FREHD_FACE(c.Nm, bxm, Nm);
    if (depth_old == 0) c.Vxm = 0;
    if (i > 0 && s - bxm <= 0) c.Nm = 0;
  }
  if (PART != FREHD_LV_WEST) {
    c.Vym = interp_surf(s, a1, L1.Vym, a2, L2.Vym);
    const double bym = j > 0 ? rd(w.bottomYP, g, i, j - 1) : 0.0;
    FREHD_FACE(c.Om, bym, Om);
    if (depth_old == 0) c.Vym = 0;
    if (j > 0 && s - bym <= 0) c.Om = 0;
  }
#undef FREHD_FACE
  return c;
}

// New surface of one cell: getFreeSurface, zeroNegSurf, enforceTidalBC
// (nsfunctions.c:436-449,412-433,1020-1031) and limiterCFL (nsfunctions.c:452-495).
// pre = the value enforceFreeSurfaceBC copies into ghosts (before tide and limiter).
struct NewSurf {
  double s, pre;
  unsigned char rmv;
};

__device__ NewSurf new_surface(const View &w, int i, int j) {
  const Params &p = w.p;
  const Grid &g = w.gr;
  const long k = g.at(i, j);
  const double bz = w.bottomZ[k];
  NewSurf r;
  double s = w.x[k];
  if (s < bz) s = bz;
  r.pre = s;
  if (is_tidal(p, i, j)) {
    const double h = tide_value(w) + p.offset;
    if (h > bz) s = h;
  }
  r.rmv = 0;
  double diff = s - bz;
  if (w.depth_cur[k] <= 0 && diff > 0) {
    const double so = w.surf_cur[k] + p.minDepth;
    const bool iP = rd(w.surf_cur, g, i + 1, j) <= so | rd(w.depth_cur, g, i + 1, j) <= 0;
    const bool iM = rd(w.surf_cur, g, i - 1, j) <= so | rd(w.depth_cur, g, i - 1, j) <= 0;
    const bool jP = rd(w.surf_cur, g, i, j + 1) <= so | rd(w.depth_cur, g, i, j + 1) <= 0;
    const bool jM = rd(w.surf_cur, g, i, j - 1) <= so | rd(w.depth_cur, g, i, j - 1) <= 0;
    if (iP & iM & jP & jM) {
      s = bz;
      r.rmv = 1;
    }
  }
  diff = s - bz;
  if (diff <= p.minDepth && diff > 0) s = bz;
  r.s = s;
  return r;
}

// ---------------------------------------------------------------- k_update_geo
// Shared-memory tile: each 32x8 block evaluates the subgrid half-cell values of
// its cells plus one column east and one row north, then combines them.
// Blocks of k_update_geo per SM the register allocation aims for (2: 128
// registers without spills; 3: 80; 4: 64, with spill traffic to L1).  With the
// level-value cache the kernel waits on dependent loads, so the extra warps of
// four blocks pay for the spills: 1.85 ms per 4096^2 step against 2.01 at 3
// and 2.27 at 2.
#ifndef FREHD_GEO_MIN_BLOCKS
#define FREHD_GEO_MIN_BLOCKS 4
#endif

template <bool kInit>
static __device__ __forceinline__ void update_geo_tile(const View &w, int bx, int by) {
  const Params &p = w.p;
  const Grid &g = w.gr;
  __shared__ double sh_s[EY][EX], sh_Np[EY][EX], sh_Nm[EY][EX], sh_Op[EY][EX], sh_Om[EY][EX];
  __shared__ double sh_Vxp[EY][EX], sh_Vxm[EY][EX], sh_Vyp[EY][EX], sh_Vym[EY][EX];
  __shared__ double sh_V[EY][EX], sh_Z[EY][EX];
  const int i0 = bx * TBX, j0 = by * TBY;
  const int tid = threadIdx.y * TBX + threadIdx.x;
  // Each thread evaluates its own cell; threads 0..TBX-1 then evaluate the north
  // halo row (only Om, Vym, s are read from it) and threads TBX..TBX+TBY-1 the
  // east halo column (only Nm, Vxm, s).
  for (int pass = 0; pass < 2; ++pass) {
    int ex, ey;
    if (pass == 0) {
      ex = threadIdx.x;
      ey = threadIdx.y;
    } else {
      if (tid >= TBX + TBY) break;
      ex = tid < TBX ? tid : TBX;
      ey = tid < TBX ? TBY : tid - TBX;
    }
    const int i = i0 + ex, j = j0 + ey;
    if (i >= g.nx || j >= g.ny) continue;
    const long k = g.at(i, j);
    const bool own = pass == 0;
    double s;
    double depth_old = w.depth_cur[k];
    if (kInit) {
      s = w.surf_cur[k];
    } else {
      const NewSurf ns = new_surface(w, i, j);
      s = ns.s;
      if (own) {
        w.rmv[k] = ns.rmv;
        w.surf_nxt[k] = s;
        // enforceFreeSurfaceBC ghosts and corners (nsfunctions.c:317-334)
        if (i == 0) w.surf_nxt[g.at(-1, j)] = ns.pre;
        if (i == g.nx - 1) w.surf_nxt[g.at(g.nx, j)] = ns.pre;
        if (j == 0) w.surf_nxt[g.at(i, -1)] = ns.pre;
        if (j == g.ny - 1) w.surf_nxt[g.at(i, g.ny)] = ns.pre;
        if (i == g.nx - 1 && j == g.ny - 1) w.surf_nxt[g.at(g.nx, g.ny)] = ns.pre;
        if (i == 0 && j == g.ny - 1) w.surf_nxt[g.at(g.nx, -1)] = ns.pre;
        if (i == g.nx - 1 && j == 0) w.surf_nxt[g.at(-1, g.ny)] = ns.pre;
        if (i == 0 && j == 0) w.surf_nxt[g.at(-1, -1)] = ns.pre;
        // computeVolumeSub keeps the previous V as the volume to update
        w.cellV[k] = w.V[k];
        double dn = s - w.bottomZ[k];
        if (dn < 0) dn = 0;
        w.depth_nxt[k] = dn;  // updateDepth (nsfunctions.c:239-247)
      }
    }
    int ind = w.ind_cur[k];
    sh_s[ey][ex] = s;
    if (own) {
      const SubCell c = compute_sub_area<FREHD_LV_ALL>(w, i, j, s, &ind, depth_old);
      w.ind_nxt[k] = ind;
      sh_Np[ey][ex] = c.Np; sh_Nm[ey][ex] = c.Nm; sh_Op[ey][ex] = c.Op; sh_Om[ey][ex] = c.Om;
      sh_Vxp[ey][ex] = c.Vxp; sh_Vxm[ey][ex] = c.Vxm; sh_Vyp[ey][ex] = c.Vyp; sh_Vym[ey][ex] = c.Vym;
      sh_V[ey][ex] = c.V; sh_Z[ey][ex] = c.Z;
    } else if (ex == TBX) {
      const SubCell c = compute_sub_area<FREHD_LV_WEST>(w, i, j, s, &ind, depth_old);
      sh_Nm[ey][ex] = c.Nm; sh_Vxm[ey][ex] = c.Vxm;
    } else {
      const SubCell c = compute_sub_area<FREHD_LV_SOUTH>(w, i, j, s, &ind, depth_old);
      sh_Om[ey][ex] = c.Om; sh_Vym[ey][ex] = c.Vym;
    }
  }
  __syncthreads();
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = i0 + tx, j = j0 + ty;
  if (i >= g.nx || j >= g.ny) return;
  // combineSubArea (subgrid.c:264-525), useminA = 0, useminV not 1/2, one rank
  const double dxdy = p.dx * p.dy;
  const double s = sh_s[ty][tx], Z = sh_Z[ty][tx];
  const bool e = i + 1 < g.nx, n = j + 1 < g.ny;
  double Nx, Oy, Vx, Vy, Zx, Zy;
  if (e) Nx = sh_Np[ty][tx] >= sh_Nm[ty][tx + 1] ? sh_Np[ty][tx] : sh_Nm[ty][tx + 1];
  else Nx = sh_Np[ty][tx];
  if (n) Oy = sh_Op[ty][tx] >= sh_Om[ty + 1][tx] ? sh_Op[ty][tx] : sh_Om[ty + 1][tx];
  else Oy = sh_Op[ty][tx];
  const double bxp = rd(w.bottomXP, g, i, j), byp = rd(w.bottomYP, g, i, j);
  if (e) {
    const double a = sh_Vxp[ty][tx], bm = sh_Vxm[ty][tx + 1];
    if (a > 0 && bm > 0) Vx = a + bm; else Vx = 2.0 * (a + bm);
    Zx = Z;
    if (Vx > 0 && Zx <= 0) Zx = dxdy;
    if (s < bxp) { Vx = bm; Zx = 0.5 * Z; }
    if (sh_s[ty][tx + 1] < bxp) { Vx = a; Zx = 0.5 * Z; }
  } else {
    Vx = 2 * sh_Vxp[ty][tx];
    Zx = 2 * Z;
  }
  if (n) {
    const double a = sh_Vyp[ty][tx], bm = sh_Vym[ty + 1][tx];
    if (a > 0 && bm > 0) Vy = a + bm; else Vy = 2.0 * (a + bm);
    Zy = Z;
    if (Vy > 0 && Zy <= 0) Zy = dxdy;
    if (s < byp) { Vy = bm; Zy = 0.5 * Z; }
    if (sh_s[ty + 1][tx] < byp) { Vy = a; Zy = 0.5 * Z; }
  } else {
    Vy = 2 * sh_Vyp[ty][tx];
    Zy = 2 * Z;
  }
  const double Vmin = 0.002, Amin = 0.002, Azmin = 0.002;
  double V = sh_V[ty][tx], Zc = Z;
  if (Vx < Vmin) Vx = 0.0;
  if (Vy < Vmin) Vy = 0.0;
  if (V < Vmin) V = 0.0;
  if (Zc < Azmin) Zc = 1.0;
  if (Zx < Amin) Zx = 0.0;
  if (Zy < Amin) Zy = 0.0;
  if (Nx < Amin) Nx = 0.0;
  if (Oy < Amin) Oy = 0.0;
  // boundary copies (subgrid.c:438-525): x ghosts first, then Nx closed on
  // east/west faces, then y ghosts, then Oy closed south and on the YP row
  // except at tidal cells.
  double *arr[8] = {w.Vx, w.Vy, w.Zx, w.Zy, w.Nx, w.Oy, w.V, w.Z};
  double val[8] = {Vx, Vy, Zx, Zy, Nx, Oy, V, Zc};
  if (i == 0) {
    const long q = g.at(-1, j);
    for (int a = 0; a < 8; ++a) arr[a][q] = val[a];
    w.Nx[q] = 0;
  }
  if (i == g.nx - 1) {
    const long q = g.at(g.nx, j);
    for (int a = 0; a < 8; ++a) arr[a][q] = val[a];
    w.Nx[q] = 0;
    val[4] = 0;  // Nx[iPbd] = 0
  }
  if (j == 0) {
    const long q = g.at(i, -1);
    for (int a = 0; a < 8; ++a) arr[a][q] = val[a];
    w.Oy[q] = 0;
  }
  if (j == g.ny - 1) {
    const long q = g.at(i, g.ny);
    for (int a = 0; a < 8; ++a) arr[a][q] = val[a];
    if (!is_tidal(p, i, j)) {
      w.Oy[q] = 0;
      val[5] = 0;
    }
  }
  const long k = g.at(i, j);
  for (int a = 0; a < 8; ++a) arr[a][k] = val[a];
}

__global__ void __launch_bounds__(TBX *TBY, FREHD_GEO_MIN_BLOCKS) k_update_geo(View w) {
  if (*(volatile int *)&w.sc->status != FREHD_OK) return;
  update_geo_tile<false>(w, blockIdx.x, blockIdx.y);
}

// The geometry of the initial state (Init's computeSubArea + combineSubArea).
__global__ void __launch_bounds__(TBX *TBY, FREHD_GEO_MIN_BLOCKS) k_update_geo_init(View w) {
  update_geo_tile<true>(w, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------- k_update_vel
// Final velocity of the east face of (i, j): updateVelocitySub (subgrid.c:1084-1176),
// the dry-cell outflow and CFL-limiter zeroing, and waterfallCorrectionSub
// (subgrid.c:1400-1444) with detectWaterfallLocationSub's flag (subgrid.c:1335-1396;
// the XM pass runs after the XP pass, so +1 wins).
__device__ double face_u(const View &w, int i, int j) {
  const Params &p = w.p;
  const Grid &g = w.gr;
  const long k = g.at(i, j), kE = g.at(i + 1, j);
  const double Vx = w.Vx[k], Nx = w.Nx[k];
  const double hx = Vx > 0 ? Nx / Vx : 0;
  const double s = w.surf_nxt[k], sE = w.surf_nxt[kE];
  double u = w.EnXP[k] - (p.g * p.dt * hx) * (sE - s) / 1.0;
  const bool e = i + 1 < g.nx;
  if (Nx == 0) u = 0;
  if (w.depth_nxt[k] == 0 && u > 0) u = 0;
  if (e && w.depth_nxt[kE] == 0 && u < 0) u = 0;
  if (w.rmv[k] == 1 || (e && w.rmv[kE] == 1)) u = 0;
  const double b = w.bottomXP[k];
  double f = 0;
  if (s < b && sE - b >= p.wtfh) f = -1;
  if (e && sE < b && s - b >= p.wtfh) f = 1;
  if (f != 0) {
    const double CFLmax = 0.24 / p.subR;
    u = f * 0.7 * sqrt(2 * p.g * Nx / p.dy);
    if (fabs(u) > CFLmax * p.dx / p.dt) u = f * CFLmax * p.dx / p.dt;
  }
  return u;
}

__device__ double face_v(const View &w, int i, int j) {
  const Params &p = w.p;
  const Grid &g = w.gr;
  const long k = g.at(i, j), kN = g.at(i, j + 1);
  const double Vy = w.Vy[k], Oy = w.Oy[k];
  const double hy = Vy > 0 ? Oy / Vy : 0;
  const double s = w.surf_nxt[k], sN = w.surf_nxt[kN];
  double v = w.EnYP[k] - (p.g * p.dt * hy) * (sN - s) / 1.0;
  const bool n = j + 1 < g.ny;
  if (Oy == 0) v = 0;
  if (w.depth_nxt[k] == 0 && v > 0) v = 0;
  if (n && w.depth_nxt[kN] == 0 && v < 0) v = 0;
  if (w.rmv[k] == 1 || (n && w.rmv[kN] == 1)) v = 0;
  const double b = w.bottomYP[k];
  double f = 0;
  if (s < b && sN - b >= p.wtfh) f = -1;
  if (n && sN < b && s - b >= p.wtfh) f = 1;
  if (f != 0) {
    const double CFLmax = 0.24 / p.subR;
    v = f * 0.7 * sqrt(2 * p.g * Oy / p.dx);
    if (fabs(v) > CFLmax * p.dy / p.dt) v = f * CFLmax * p.dy / p.dt;
  }
  return v;
}

// Face flow rates as computeFaceFlowRateSub stores them (subgrid.c:1190-1212)
// for any face the TVD stencil reaches: interior faces recomputed, the ghost
// column/row faces from the boundary cell's velocity copied by enforceVelocityBC
// (nsfunctions.c:289-314) times the ghost's own face area.
__device__ double flux_u(const View &w, int i, int j) {
  const int ib = i < 0 ? 0 : (i >= w.gr.nx ? w.gr.nx - 1 : i);
  return face_u(w, ib, j) * w.Nx[w.gr.at(i, j)];
}

__device__ double flux_v(const View &w, int i, int j) {
  const int jb = j < 0 ? 0 : (j >= w.gr.ny ? w.gr.ny - 1 : j);
  return face_v(w, i, jb) * w.Oy[w.gr.at(i, j)];
}

// Superbee limiter (scalar.c:115-119).
__device__ __forceinline__ double superbee(double r) {
  double p1, p2, phi;
  if (2 * r > 1) p1 = 1; else p1 = 2 * r;
  if (r > 2) p2 = 2; else p2 = r;
  if (p1 > 0) phi = p1; else phi = 0;
  if (p2 > phi) phi = p2;
  return phi;
}

// TVD face values of cell (i, j) (scalarAdvection with scalarAdv = 2,
// scalar.c:99-249).  The two-cell maps are map.c:66-97's: iPPjc/iMMjc and icjPP
// stop at the ghost ring; icjMM of the second row (j = 1) is never assigned by
// the reference and reads 0 (cell (0, 0)) under the zero-filled allocation the
// parity build uses.  The YM Courant number uses dx, as the reference's does.
__device__ void tvd_faces(const View &w, const double *S, int i, int j, double FE, double FW,
                          double FN, double FS, double uE, double uW, double vst, double vS,
                          double *Sd_, double *Su_, double *Sr_, double *Sl_) {
  const Params &p = w.p;
  const Grid &g = w.gr;
  const double dSmin = 0.00001;
  const long k = g.at(i, j);
  const double Sc = S[k], SE = S[g.at(i + 1, j)], SW = S[g.at(i - 1, j)];
  const double SNn = S[g.at(i, j + 1)], SS = S[g.at(i, j - 1)];
  const int iee = i <= g.nx - 3 ? i + 2 : g.nx, iww = i >= 2 ? i - 2 : -1;
  const int jnn = j <= g.ny - 3 ? j + 2 : g.ny;
  const double SEE = S[g.at(iee, j)], SWW = S[g.at(iww, j)], SNN = S[g.at(i, jnn)];
  double SSS, Fss;
  if (j >= 2) { SSS = S[g.at(i, j - 2)]; Fss = flux_v(w, i, j - 2); }
  else if (j == 1) { SSS = S[g.at(0, 0)]; Fss = flux_v(w, 0, 0); }
  else { SSS = S[g.at(i, -1)]; Fss = flux_v(w, i, -1); }
  double Sd, Su, Sr, Sl, Cu, r;
  // XP face
  Cu = uE * p.dt / p.dx;
  if (FE > 0) {
    if (FW <= 0) Sd = Sc;
    else {
      if (fabs(SE - Sc) < dSmin) r = 0; else r = (Sc - SW) / (SE - Sc);
      Sd = Sc + 0.5 * superbee(r) * (SE - Sc) * Cu * (1 - Cu);
    }
  } else {
    if (flux_u(w, i + 1, j) >= 0) Sd = SE;
    else {
      if (fabs(SE - Sc) < dSmin) r = 0; else r = (SE - SEE) / (Sc - SE);
      Sd = SE + 0.5 * superbee(r) * (Sc - SE) * Cu * (1 - Cu);
    }
  }
  // XM face
  Cu = uW * p.dt / p.dx;
  if (FW > 0) {
    if (flux_u(w, iww, j) <= 0) Su = SW;
    else {
      if (fabs(Sc - SW) < dSmin) r = 0; else r = (SW - SWW) / (Sc - SW);
      Su = SW + 0.5 * superbee(r) * (Sc - SW) * Cu * (1 - Cu);
    }
  } else {
    if (FE >= 0) Su = Sc;
    else {
      if (fabs(Sc - SW) < dSmin) r = 0; else r = (Sc - SE) / (SW - Sc);
      Su = Sc + 0.5 * superbee(r) * (SW - Sc) * Cu * (1 - Cu);
    }
  }
  // YP face
  Cu = vst * p.dt / p.dy;
  if (FN > 0) {
    if (FS <= 0) Sr = Sc;
    else {
      if (fabs(SNn - Sc) < dSmin) r = 0; else r = (Sc - SS) / (SNn - Sc);
      Sr = Sc + 0.5 * superbee(r) * (SNn - Sc) * Cu * (1 - Cu);
    }
  } else {
    if (flux_v(w, i, j + 1) >= 0) Sr = SNn;
    else {
      if (fabs(SNn - Sc) < dSmin) r = 0; else r = (SNn - SNN) / (Sc - SNn);
      Sr = SNn + 0.5 * superbee(r) * (Sc - SNn) * Cu * (1 - Cu);
    }
  }
  // YM face
  Cu = vS * p.dt / p.dx;
  if (FS > 0) {
    if (Fss <= 0) Sl = SS;
    else {
      if (fabs(Sc - SS) < dSmin) r = 0; else r = (SS - SSS) / (Sc - SS);
      Sl = SS + 0.5 * superbee(r) * (Sc - SS) * Cu * (1 - Cu);
    }
  } else {
    if (FN >= 0) Sl = Sc;
    else {
      if (fabs(Sc - SS) < dSmin) r = 0; else r = (Sc - SNn) / (SS - Sc);
      Sl = Sc + 0.5 * superbee(r) * (SS - Sc) * Cu * (1 - Cu);
    }
  }
  *Sd_ = Sd;
  *Su_ = Su;
  *Sr_ = Sr;
  *Sl_ = Sl;
}

__device__ __forceinline__ unsigned long long dbits(double x) {
  return (unsigned long long)__double_as_longlong(x);
}

// What one cell's scalar update needs besides the scalar itself: the step's
// face flows and velocities, volumes and depth, and which neighbours the
// limiter may take its bounds from.
struct ScalarCell {
  double cv_old, cv, dep, FE, FW, FN, FS, uE, uW, vst, vS, NxW, OyS;
  bool inflow, wE, wW, wN, wS;
};

// scalarTransport (scalar.c:30-57) of one scalar in cell (i, j): upwind or TVD
// advection (scalar.c:72-249), scalarDiffusionSub (subgrid.c:1552-1567),
// updateScalarSub (subgrid.c:1570-1713), enforceScalarBC (scalar.c:419-471).
// `primary` is the reference's S: it stores Sm and, in the singularity branch
// (S outside [0, 100], subgrid.c:1700-1712), queues the cell for the surface and
// depth fix-up.  A tracer only takes the branch's zero, so the hydrodynamics
// stay those of S.
template <bool kTVD>
static __device__ __forceinline__ void transport_scalar(const View &w, const double *S, double *Snx,
                                                        bool primary, int i, int j, long k,
                                                        const ScalarCell &c) {
  const Params &p = w.p;
  const Grid &g = w.gr;
  const double Sc = S[k], SE = rd(S, g, i + 1, j), SW = rd(S, g, i - 1, j);
  const double SNn = rd(S, g, i, j + 1), SS = rd(S, g, i, j - 1);
  double Sm = Sc * c.cv_old;  // computeVolumeSub: Sm = S * cellV
  double Sd, Su, Sr, Sl;
  if (kTVD) {
    tvd_faces(w, S, i, j, c.FE, c.FW, c.FN, c.FS, c.uE, c.uW, c.vst, c.vS, &Sd, &Su, &Sr, &Sl);
  } else {
    Sd = c.FE > 0 ? Sc : SE;
    Su = c.FW > 0 ? SW : Sc;
    Sr = c.FN > 0 ? Sc : SNn;
    Sl = c.FS > 0 ? SS : Sc;
  }
  Sm = Sm + p.dt * (-c.FE * Sd + c.FW * Su - c.FN * Sr + c.FS * Sl);
  Sm = Sm + p.dt * ((p.Kx * w.Nx[k] / p.dx) * (SE - Sc) - (p.Kx * c.NxW / p.dx) * (Sc - SW) +
                    (p.Ky * w.Oy[k] / p.dy) * (SNn - Sc) - (p.Ky * c.OyS / p.dy) * (Sc - SS));
  // scalar from inflow (subgrid.c:1648-1654); inflow cells skip the limiter
  if (c.inflow) Sm = Sm + p.inflowS * inflow_value(w) * p.dt / p.inflowLen;
  int cnt = 0;
  double smax = 0, smin = 0;
#define FREHD_NB(cond, val)                                 \
  if (cond) {                                               \
    const double v_ = (val);                                \
    if (cnt == 0) { smax = v_; smin = v_; }                 \
    else { if (v_ > smax) smax = v_; if (v_ < smin) smin = v_; } \
    ++cnt;                                                  \
  }
  FREHD_NB(c.wE, SE);
  FREHD_NB(c.wW, SW);
  FREHD_NB(c.wN, SNn);
  FREHD_NB(c.wS, SS);
#undef FREHD_NB
  double Sn = c.cv > 0 ? Sm / c.cv : 0;
  if (cnt != 0 && Sn > smax && !c.inflow) Sn = smax;
  else if (cnt != 0 && Sn < smin && !c.inflow) Sn = smin;
  double depf = c.dep;
  if ((Sn > 100 || Sn < 0) && !(j == 0) && !(j == g.ny - 1 && i > 0)) {
    Sn = 0;
    if (primary) {
      depf = 0;
      const int slot = atomicAdd(&w.sc->n_fix, 1);
      w.fix_list[slot] = (int)k;
    }
  }
  if (i == 0) Snx[g.at(-1, j)] = Sn;
  if (i == g.nx - 1) Snx[g.at(g.nx, j)] = Sn;
  if (j == 0) Snx[g.at(i, -1)] = Sn;
  if (j == g.ny - 1) Snx[g.at(i, g.ny)] = Sn;
  if (is_tidal(p, i, j)) Sn = p.tidePS;
  if (depf <= 0) Sn = 0;
  Snx[k] = Sn;
  if (primary) w.Sm[k] = Sm;
}

// gx: the domain's tile-grid width (the block's partial-sum slot is by*gx + bx)
template <bool kTVD>
static __device__ __forceinline__ void update_vel_tile(const View &w, int bx, int by, int gx) {
  const Params &p = w.p;
  const Grid &g = w.gr;
  const int i = bx * TBX + threadIdx.x;
  const int j = by * TBY + threadIdx.y;
  double cflx = 0, cfly = 0, vol = 0;
  int nwarn = 0;
  // Each face velocity once: a cell's west face is its west neighbour's east
  // face (the lane before it) and its south face the north face of the cell
  // below (the row before it in the block); the block's first column and row
  // evaluate theirs.  The same function of the same inputs, so the same doubles.
  __shared__ double s_vN[TBY][TBX];
  const bool in = i < g.nx && j < g.ny;
  const double uE_ = in ? face_u(w, i, j) : 0.0;
  const double vN_ = in ? face_v(w, i, j) : 0.0;
  const double uW_lane = __shfl_up_sync(0xffffffffu, uE_, 1);
  s_vN[threadIdx.y][threadIdx.x] = vN_;
  __syncthreads();
  if (in) {
    const long k = g.at(i, j);
    const double uE = uE_;
    const double uW = i > 0 ? (threadIdx.x > 0 ? uW_lane : face_u(w, i - 1, j))
                            : uE;  // enforceVelocityBC ghost copy
    const double vN = vN_;
    const double vS = j > 0 ? (threadIdx.y > 0 ? s_vN[threadIdx.y - 1][threadIdx.x] : face_v(w, i, j - 1))
                            : vN;
    // computeFaceFlowRateSub (subgrid.c:1190-1212)
    const double NxW = rd(w.Nx, g, i - 1, j), OyS = rd(w.Oy, g, i, j - 1);
    const double FE = uE * w.Nx[k], FW = uW * NxW, FN = vN * w.Oy[k], FS = vS * OyS;
    double vstore = vN;
    const double sN = w.surf_nxt[k];
    if (is_tidal(p, i, j)) {
      // adjustTidalVelocitySub (subgrid.c:1295-1313)
      const double Fww = (sN - w.surf_cur[k]) * w.Z[k] / p.dt;
      const double all = FS + FW - FE - Fww;
      vstore = (all != 0 & w.Oy[k] > 0) ? all / w.Oy[k] : 0;
    }
    w.u[k] = uE;
    w.v[k] = vstore;
    w.Fuu[k] = FE;
    w.Fvv[k] = FN;
    // enforceVelocityBC ghosts (nsfunctions.c:289-314) and their face flows
    if (i == 0) {
      const long q = g.at(-1, j);
      w.u[q] = uE; w.v[q] = vN; w.Fuu[q] = uE * w.Nx[q]; w.Fvv[q] = vN * w.Oy[q];
    }
    if (i == g.nx - 1) {
      const long q = g.at(g.nx, j);
      w.u[q] = uE; w.v[q] = vN; w.Fuu[q] = uE * w.Nx[q]; w.Fvv[q] = vN * w.Oy[q];
    }
    if (j == 0) {
      const long q = g.at(i, -1);
      w.u[q] = uE; w.v[q] = vN; w.Fuu[q] = uE * w.Nx[q]; w.Fvv[q] = vN * w.Oy[q];
    }
    if (j == g.ny - 1) {
      const long q = g.at(i, g.ny);
      w.u[q] = uE; w.v[q] = vN; w.Fuu[q] = uE * w.Nx[q]; w.Fvv[q] = vN * w.Oy[q];
    }
    // corners: u from the jP/jM ghost rows, v from the iP/iM ghost columns
    if (i == g.nx - 1 && j == g.ny - 1) { w.u[g.at(g.nx, g.ny)] = uE; w.v[g.at(g.nx, g.ny)] = vN; }
    if (i == g.nx - 1 && j == 0) w.u[g.at(g.nx, -1)] = uE;
    if (i == 0 && j == g.ny - 1) { w.u[g.at(-1, g.ny)] = uE; w.v[g.at(g.nx, -1)] = vN; }
    if (i == 0 && j == 0) { w.u[g.at(-1, -1)] = uE; w.v[g.at(-1, -1)] = vN; }
    if (i == g.nx - 1 && j == 0) w.v[g.at(-1, g.ny)] = vN;
    // corner face flows (computeFaceFlowRateSub runs over all N2ct entries)
    if (i == g.nx - 1 && j == g.ny - 1) {
      const long q = g.at(g.nx, g.ny);
      w.Fuu[q] = w.u[q] * w.Nx[q]; w.Fvv[q] = w.v[q] * w.Oy[q];
    }
    // volumeByFluxSub (subgrid.c:1227-1263)
    const double cv_old = w.cellV[k];
    double cv = cv_old + p.dt * (FW - FE + FS - FN);
    const bool inflow_cell = is_inflow(p, i, j);
    if (inflow_cell) cv = cv + inflow_value(w) * p.dt;
    if (cv < 0) cv = 0;
    w.cellV[k] = cv;
    vol = cv;
    // updateCDSub, useSubDrag = 0 (subgrid.c:1521-1536), then thinLayerDrag
    // (nsfunctions.c:713-726) with the face depths of updateAllFaceDepth
    const double coeff = p.g * p.manningN * p.manningN;
    double CDX = w.CDXP[k], CDY = w.CDYP[k];
    if (w.V[k] > 0) {
      const double h = w.V[k] / w.Z[k];
      CDX = coeff / pow(h, 1.0 / 3.0);
      CDY = coeff / pow(h, 1.0 / 3.0);
    }
    const double dep = w.depth_nxt[k];
    if ((p.useThinLayer && dep > 0) || p.useWind) {
      double hxp = 0, hyp = 0;
      if (i < g.nx - 1) {
        const double a = sN, c = w.surf_nxt[g.at(i + 1, j)];
        hxp = (a > c ? a : c) - w.bottomXP[k];
        if (hxp < 0) hxp = 0;
      }
      if (j < g.ny - 1) {
        const double a = sN, c = w.surf_nxt[g.at(i, j + 1)];
        hyp = (a > c ? a : c) - w.bottomYP[k];
        if (hyp < 0) hyp = 0;
      }
      if (p.useThinLayer && dep > 0) {
        if (hxp <= p.hD) CDX = coeff / pow(dep, 2.0 / 3.0);
        if (hyp <= p.hD) CDY = coeff / pow(dep, 2.0 / 3.0);
      }
      if (p.useWind) {  // updateAllFaceDepth's interior faces, read by the next windTerm
        w.dXP[k] = hxp;
        w.dYP[k] = hyp;
      }
    }
    w.CDXP[k] = CDX;
    w.CDYP[k] = CDY;
    // scalarTransport for S and the tracers
    if (p.useScalar) {
      ScalarCell c;
      c.cv_old = cv_old; c.cv = cv; c.dep = dep;
      c.FE = FE; c.FW = FW; c.FN = FN; c.FS = FS;
      c.uE = uE; c.uW = uW; c.vst = vstore; c.vS = vS; c.NxW = NxW; c.OyS = OyS;
      c.inflow = inflow_cell;
      // connected wet neighbours of the limiter (updateScalarSub, subgrid.c:1582-1640)
      c.wE = w.Nx[k] > 0 && rd(w.surf_cur, g, i + 1, j) - rd(w.bottomZ, g, i + 1, j) > 0;
      c.wW = NxW > 0 && rd(w.surf_cur, g, i - 1, j) - rd(w.bottomZ, g, i - 1, j) > 0;
      c.wN = (j < g.ny - 1 || i == 0) && w.Oy[k] > 0 &&
             rd(w.surf_cur, g, i, j + 1) - rd(w.bottomZ, g, i, j + 1) > 0;
      c.wS = j > 0 && OyS > 0 && rd(w.surf_cur, g, i, j - 1) - rd(w.bottomZ, g, i, j - 1) > 0;
      transport_scalar<kTVD>(w, w.S_cur, w.S_nxt, true, i, j, k, c);
#pragma unroll
      for (int t = 0; t < FREHD_MAX_SCALARS - 1; ++t)
        if (t + 1 < p.nscalar) transport_scalar<kTVD>(w, w.Tr_cur[t], w.Tr_nxt[t], false, i, j, k, c);
    }
    // monitorCFL (nsfunctions.c:1196-1223)
    cflx = fabs(uE) * p.dt / p.dx;
    cfly = fabs(vstore) * p.dt / p.dy;
    w.CFLx[k] = cflx;
    w.CFLy[k] = cfly;
    nwarn = (cflx > 2) + (cfly > 2);
  }
  // block reductions: max CFL, warnings, volume partial
  cflx = warp_max(cflx);
  cfly = warp_max(cfly);
  nwarn = warp_sum_int(nwarn);
  vol = warp_sum(vol);
  __shared__ double sv[TBX * TBY / 32], sx[TBX * TBY / 32], sy[TBX * TBY / 32];
  __shared__ int sw[TBX * TBY / 32];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (lane == 0) { sv[wid] = vol; sx[wid] = cflx; sy[wid] = cfly; sw[wid] = nwarn; }
  __syncthreads();
  if (tid == 0) {
    double a = 0, mx = 0, my = 0;
    int nw = 0;
    for (int q = 0; q < TBX * TBY / 32; ++q) {
      a += sv[q];
      mx = fmax(mx, sx[q]);
      my = fmax(my, sy[q]);
      nw += sw[q];
    }
    w.partials[by * gx + bx] = a;
    if (mx > 0) atomicMax(&w.sc->max_cflx_bits, dbits(mx));
    if (my > 0) atomicMax(&w.sc->max_cfly_bits, dbits(my));
    if (nw) atomicAdd(&w.sc->n_cfl_warn, nw);
  }
}

// Four blocks per SM (64 registers): 1.78 -> 1.49 ms per step at 4096 x 4096
// against the unconstrained 72 registers and three blocks.
__global__ void __launch_bounds__(TBX *TBY, 4) k_update_vel(View w) {
  if (*(volatile int *)&w.sc->status != FREHD_OK) return;
  update_vel_tile<false>(w, blockIdx.x, blockIdx.y, gridDim.x);
}

// The same for decks with TVD scalar advection (scalarAdv = 2): a kernel of its
// own, so that the wider stencil's registers do not cost the upwind kernel
// occupancy.
__global__ void __launch_bounds__(TBX *TBY) k_update_vel_tvd(View w) {
  if (*(volatile int *)&w.sc->status != FREHD_OK) return;
  update_vel_tile<true>(w, blockIdx.x, blockIdx.y, gridDim.x);
}

// ---------------------------------------------------------------- k_finish
// The scalar singularity branch (subgrid.c:1700-1712) also lowers the surface
// of the cell by its depth; cells are queued by k_update_vel and fixed here so
// that no kernel reads a half-updated surface.  Then the step statistics.
static __device__ __forceinline__ bool finish_block(const View &w, int nblocks_vel, StepOut *out) {
  const int tid = threadIdx.x;
  if (*(volatile int *)&w.sc->status != FREHD_OK) {  // step skipped or aborted
    if (tid == 0) out->status = w.sc->status;
    return false;
  }
  const int nfix = w.sc->n_fix;
  for (int q = tid; q < nfix; q += blockDim.x) {
    const int k = w.fix_list[q];
    w.surf_nxt[k] = w.surf_nxt[k] - w.depth_nxt[k];
    w.depth_nxt[k] = 0;
  }
  // fixed-order volume sum
  __shared__ double sh[1024];
  double a = 0;
  for (int q = tid; q < nblocks_vel; q += blockDim.x) a += w.partials[q];
  sh[tid] = a;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (tid < s) sh[tid] += sh[tid + s];
    __syncthreads();
  }
  if (tid == 0) {
    Scratch *sc = w.sc;
    out->step = sc->tt;
    out->cg_iters = sc->cg_iters;
    out->cg_fallback = sc->cg_fallback;
    out->status = FREHD_OK;
    out->cg_rr = sc->cg_rr;
    out->cg_bb = sc->cg_bb;
    out->max_cflx = __longlong_as_double((long long)sc->max_cflx_bits);
    out->max_cfly = __longlong_as_double((long long)sc->max_cfly_bits);
    out->n_cfl_warn = sc->n_cfl_warn;
    out->volume = sh[0];
    out->n_fix = nfix;
    sc->cg_iters_total += sc->cg_iters;
    out->cg_iters_total = sc->cg_iters_total;
    // a solve that stopped at maxIter is reported, not fatal (laspack goes on, itersolv.c:399-418)
    out->cg_noconv = sc->cg_noconv;
    sc->cg_noconv_steps += sc->cg_noconv;
    out->cg_noconv_steps = sc->cg_noconv_steps;
    sc->cg_noconv = 0;
    // monitorCFL's exit condition (nsfunctions.c:1226-1231)
    if (fabs(out->max_cflx) > 20 || fabs(out->max_cfly) > 20) out->status = FREHD_ERR_CFL;
    // reset the per-step counters for the next step
    sc->n_fix = 0;
    sc->n_cfl_warn = 0;
    sc->max_cflx_bits = 0;
    sc->max_cfly_bits = 0;
    if (out->status != FREHD_OK) sc->status = out->status;
    sc->tt = sc->tt + 1;
  }
  return true;
}

__global__ void k_finish(View w, int nblocks_vel, StepOut *out) { finish_block(w, nblocks_vel, out); }

// ---------------------------------------------------------------- batched launches
// One block per table entry (domain slot, tile) over every domain of a batch.
// Each block stages its domain's view, at the domain's current ping-pong half
// (sc->cur, flipped by k_finish_batch), in shared memory.
static __device__ __forceinline__ void stage_view(const View *views2, int d, View *sv, int *s_cur, int tid,
                                           int nthr) {
  if (tid == 0) *s_cur = *(volatile int *)&views2[2 * d].sc->cur;
  __syncthreads();
  const unsigned long long *src = reinterpret_cast<const unsigned long long *>(views2 + 2 * d + *s_cur);
  unsigned long long *dst = reinterpret_cast<unsigned long long *>(sv);
  for (int e = tid; e < (int)(sizeof(View) / 8); e += nthr) dst[e] = src[e];
  __syncthreads();
}

// A block stages its domain's view once and runs the tile code on t.nt
// consecutive tiles of one tile row (the barrier between them frees the
// tile's shared memory for the next).
__global__ void __launch_bounds__(TBX *TBY, kExplicitMinBlocks)
    k_explicit_batch(const View *views2, const BatchTile *tiles) {
  __shared__ View sv;
  __shared__ int s_cur;
  const BatchTile t = tiles[blockIdx.x];
  stage_view(views2, t.d, &sv, &s_cur, threadIdx.y * TBX + threadIdx.x, TBX * TBY);
  if (*(volatile int *)&sv.sc->status != FREHD_OK) return;
  for (int q = 0; q < t.nt; ++q) {
    if (q) __syncthreads();
    explicit_tile(sv, t.bx + q, t.by);
  }
}

__global__ void __launch_bounds__(TBX *TBY, FREHD_GEO_MIN_BLOCKS)
    k_update_geo_batch(const View *views2, const BatchTile *tiles) {
  __shared__ View sv;
  __shared__ int s_cur;
  const BatchTile t = tiles[blockIdx.x];
  stage_view(views2, t.d, &sv, &s_cur, threadIdx.y * TBX + threadIdx.x, TBX * TBY);
  if (*(volatile int *)&sv.sc->status != FREHD_OK) return;
  for (int q = 0; q < t.nt; ++q) {
    if (q) __syncthreads();  // also: the window's mbarrier is re-armed only after every wait on it
    update_geo_tile<false>(sv, t.bx + q, t.by);
  }
}

// Upwind and TVD domains in kernels of their own (the batch orders its tiles
// upwind first), so that the TVD stencil's registers do not cost the upwind
// kernel its four blocks per SM.
__global__ void __launch_bounds__(TBX *TBY, 4) k_update_vel_batch(const View *views2, const BatchTile *tiles) {
  __shared__ View sv;
  __shared__ int s_cur;
  const BatchTile t = tiles[blockIdx.x];
  stage_view(views2, t.d, &sv, &s_cur, threadIdx.y * TBX + threadIdx.x, TBX * TBY);
  if (*(volatile int *)&sv.sc->status != FREHD_OK) return;
  for (int q = 0; q < t.nt; ++q) {
    if (q) __syncthreads();
    update_vel_tile<false>(sv, t.bx + q, t.by, t.gx);
  }
}

__global__ void __launch_bounds__(TBX *TBY) k_update_vel_tvd_batch(const View *views2, const BatchTile *tiles) {
  __shared__ View sv;
  __shared__ int s_cur;
  const BatchTile t = tiles[blockIdx.x];
  stage_view(views2, t.d, &sv, &s_cur, threadIdx.y * TBX + threadIdx.x, TBX * TBY);
  if (*(volatile int *)&sv.sc->status != FREHD_OK) return;
  for (int q = 0; q < t.nt; ++q) {
    if (q) __syncthreads();
    update_vel_tile<true>(sv, t.bx + q, t.by, t.gx);
  }
}

// One block per domain: k_finish's work, then the domain's ping-pong half flips.
// bsync (may be null): the barrier scratch of the batch's tile-list solve, which
// ran before this kernel; its counters start the next step's solve from zero,
// also after a solve that gave up waiting.
__global__ void k_finish_batch(const View *views2, const FinishJob *jobs, Scratch *bsync) {
  __shared__ View sv;
  __shared__ int s_cur;
  const FinishJob f = jobs[blockIdx.x];
  if (bsync && blockIdx.x == 0 && threadIdx.x == 0) {
    bsync->bar_count = 0;
    bsync->n_done = 0;
    bsync->status = FREHD_OK;
  }
  stage_view(views2, f.d, &sv, &s_cur, threadIdx.x, blockDim.x);
  const bool ran = finish_block(sv, f.nblocks_vel, f.out);
  if (ran && threadIdx.x == 0) sv.sc->cur = s_cur ^ 1;
  // the batch's owner sees a failed domain (CFL > 20, a wait that gave up) after
  // this step without reading the domain's statistics
  if (threadIdx.x == 0) *(volatile int *)f.status = *(volatile int *)&sv.sc->status;
}

// ---------------------------------------------------------------- layout
__global__ void k_ref_to_padded(double *dst, const double *src, long n, int nx, int ny, int pitch) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= n) return;
  int i, j;
  ref_to_ij(k, nx, ny, &i, &j);
  dst[(long)(j + 1) * pitch + (i + kXOff)] = src[k];
}

__global__ void k_padded_to_ref(double *dst, const double *src, long n, int nx, int ny, int pitch) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= n) return;
  int i, j;
  ref_to_ij(k, nx, ny, &i, &j);
  dst[k] = src[(long)(j + 1) * pitch + (i + kXOff)];
}

__global__ void k_ref_to_padded_int(int *dst, const int *src, long n, int nx, int ny, int pitch) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= n) return;
  int i, j;
  ref_to_ij(k, nx, ny, &i, &j);
  dst[(long)(j + 1) * pitch + (i + kXOff)] = src[k];
}

__global__ void k_padded_to_ref_int(int *dst, const int *src, long n, int nx, int ny, int pitch) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= n) return;
  int i, j;
  ref_to_ij(k, nx, ny, &i, &j);
  dst[k] = src[(long)(j + 1) * pitch + (i + kXOff)];
}

__global__ void k_fill(double *a, long n, double v) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k < n) a[k] = v;
}

// uuYP / vvXP of the current velocities (for downloads).
__global__ void k_interp_velocity(View w, double *uuYP, double *vvXP) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long N = (long)w.gr.nx * w.gr.ny;
  if (t >= N) return;
  const int i = (int)(t % w.gr.nx), j = (int)(t / w.gr.nx);
  uuYP[t] = uuYP_at(w, i, j);
  vvXP[t] = vvXP_at(w, i, j);
}

// Assembled system in the reference's terms (row-major Gn*, transposed z, x).
__global__ void k_system_to_ref(View w, double *GnCt, double *GnXP, double *GnXM, double *GnYP,
                                double *GnYM, double *z, double *xs) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const Grid &g = w.gr;
  const long N = (long)g.nx * g.ny;
  if (t >= N) return;
  const int i = (int)(t % g.nx), j = (int)(t / g.nx);
  const long k = g.at(i, j);
  const double ct = w.Ct[k];
  const bool iso = ct < 0;
  if (GnCt) GnCt[t] = iso ? -ct : ct;
  if (GnXP) GnXP[t] = (iso || i == g.nx - 1) ? 0.0 : w.Gx[k];
  if (GnXM) GnXM[t] = (iso || i == 0) ? 0.0 : w.Gx[g.at(i - 1, j)];
  if (GnYP) GnYP[t] = (iso || j == g.ny - 1) ? 0.0 : w.Gy[k];
  if (GnYM) GnYM[t] = (iso || j == 0) ? 0.0 : w.Gy[g.at(i, j - 1)];
  const long tr = (long)i * g.ny + j;  // sprt: transposed index of (i, j)
  if (z) z[tr] = w.b[k];
  if (xs) xs[tr] = w.x[k];
}

// Solution given in the transposed order into the padded x.
__global__ void k_solution_from_ref(View w, const double *xs) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const Grid &g = w.gr;
  const long N = (long)g.nx * g.ny;
  if (t >= N) return;
  const int i = (int)(t / g.ny), j = (int)(t % g.ny);  // trps
  w.x[g.at(i, j)] = xs[t];
}

}  // namespace frehd

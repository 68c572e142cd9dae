// Host pre-processing: subgrid tables and coarse bottoms of a deck from its fine
// bottoms.  Uses the same inline evaluation as the device (subgrid_levels.h), so a
// domain run from fine bottoms and a domain run from these tables see the same
// level values.  Parallelised over levels with std::thread; each value is computed
// by one thread with the fixed summation order of subgrid_levels.h.
#include <thread>
#include <vector>

#include "frehd_b200.h"
#include "frehd_internal.h"
#include "subgrid_levels.h"

extern "C" int frehd_build_tables_ex(const double *zf, long fpitch, int nx, int ny, int r,
                                     double dxf, double dyf, double surfmin, double dsurf, int Ne,
                                     int flags, double *tables) {
  if (!zf || !tables || nx <= 0 || ny <= 0 || r <= 0 || Ne <= 0 || fpitch < (long)nx * r ||
      (flags & ~FREHD_GEOM_BLOCK_CHECK))
    return frehd::fail(FREHD_ERR_INVALID, "frehd_build_tables: bad arguments");
  const int check_block = (flags & FREHD_GEOM_BLOCK_CHECK) && r > 1;
  if (check_block && r > 8)
    return frehd::fail(FREHD_ERR_UNSUPPORTED, "block check needs r <= 8 (r = %d)", r);
  const long N = (long)nx * ny;
  const double dA = dxf * dyf;
  unsigned nth = std::thread::hardware_concurrency();
  if (nth == 0) nth = 1;
  if (nth > (unsigned)Ne) nth = (unsigned)Ne;
  auto work = [&](int k0, int k1) {
    for (int k = k0; k < k1; ++k) {
      const double h = frehd_level(surfmin, dsurf, k);
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          frehd_cell_levels o;
          frehd_cell_levels_at(zf, fpitch, nx, ny, r, i, j, h, dA, dxf, check_block, &o);
          const long ii = (long)j * nx + i, base = N * k + ii, T = N * (long)Ne;
          tables[0 * T + base] = o.V;
          tables[1 * T + base] = o.Z;
          tables[2 * T + base] = o.Vxp;
          tables[3 * T + base] = o.Vxm;
          tables[4 * T + base] = o.Vyp;
          tables[5 * T + base] = o.Vym;
          tables[6 * T + base] = o.Np;
          tables[7 * T + base] = o.Nm;
          tables[8 * T + base] = o.Op;
          tables[9 * T + base] = o.Om;
        }
    }
  };
  std::vector<std::thread> pool;
  int per = (Ne + (int)nth - 1) / (int)nth;
  for (unsigned t = 0; t < nth; ++t) {
    int k0 = (int)t * per, k1 = k0 + per > Ne ? Ne : k0 + per;
    if (k0 < k1) pool.emplace_back(work, k0, k1);
  }
  for (auto &th : pool) th.join();
  return FREHD_OK;
}

extern "C" int frehd_build_tables(const double *zf, long fpitch, int nx, int ny, int r,
                                  double dxf, double dyf, double surfmin, double dsurf, int Ne,
                                  double *tables) {
  return frehd_build_tables_ex(zf, fpitch, nx, ny, r, dxf, dyf, surfmin, dsurf, Ne, 0, tables);
}

extern "C" int frehd_build_bottoms(const double *zf, long fpitch, int nx, int ny, int r,
                                   double *bottom, double *bottomXP, double *bottomYP) {
  if (!zf || !bottom || !bottomXP || !bottomYP || nx <= 0 || ny <= 0 || r <= 0 ||
      fpitch < (long)nx * r)
    return frehd::fail(FREHD_ERR_INVALID, "frehd_build_bottoms: bad arguments");
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      long ii = (long)j * nx + i;
      frehd_cell_bottoms(zf, fpitch, nx, ny, r, i, j, &bottom[ii], &bottomXP[ii], &bottomYP[ii]);
    }
  return FREHD_OK;
}

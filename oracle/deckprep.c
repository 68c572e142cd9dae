/*
 * deckprep.c -- TEST INFRASTRUCTURE: host pre-processing of synthetic decks for
 * runs of the reference program alone (bench.py's reference arm and CPU
 * baseline), so that those processes load no library of the product.
 *
 * The reference's own pre-processor is MATLAB (preProcessing/
 * script_CreateSubAreaWithBlockV16.m, ComputeSubgridFaceArea.m,
 * ComputeFaceAreaWithBlockCheck.m), which cannot run here.  Its formulas are
 * restated once, in the inline functions of subgrid_levels.h; this file
 * tabulates them exactly as the library's frehd_build_tables_ex and
 * frehd_build_bottoms do (same function per value, same order), so a deck
 * written with either builder holds the same doubles (a CPU test compares them).
 * Built with -ffp-contract=off like the rest of the oracle.
 */
#include "subgrid_levels.h"

/* tables: 10 * Ne * nx * ny doubles, V, Z, Vxp, Vxm, Vyp, Vym, Np, Nm, Op, Om,
 * each level-major (table[N*k + ii], subgrid.c:118-119). */
int oracle_build_tables(const double *zf, long fpitch, int nx, int ny, int r, double dxf,
                        double dyf, double surfmin, double dsurf, int Ne, int check_block,
                        double *tables) {
  if (!zf || !tables || nx <= 0 || ny <= 0 || r <= 0 || Ne <= 0 || fpitch < (long)nx * r) return 1;
  if (check_block && (r < 2 || r > 8)) return 2;
  const long N = (long)nx * ny, T = N * (long)Ne;
  const double dA = dxf * dyf;
#pragma omp parallel for schedule(dynamic, 1)
  for (int k = 0; k < Ne; ++k) {
    const double h = frehd_level(surfmin, dsurf, k);
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        frehd_cell_levels o;
        frehd_cell_levels_at(zf, fpitch, nx, ny, r, i, j, h, dA, dxf, check_block, &o);
        const long base = N * k + (long)j * nx + i;
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
  return 0;
}

/* Coarse bottom.dat / bottomXP.dat / bottomYP.dat (N doubles each). */
int oracle_build_bottoms(const double *zf, long fpitch, int nx, int ny, int r, double *bottom,
                         double *bottomXP, double *bottomYP) {
  if (!zf || !bottom || !bottomXP || !bottomYP || nx <= 0 || ny <= 0 || r <= 0 ||
      fpitch < (long)nx * r)
    return 1;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const long ii = (long)j * nx + i;
      frehd_cell_bottoms(zf, fpitch, nx, ny, r, i, j, &bottom[ii], &bottomXP[ii], &bottomYP[ii]);
    }
  return 0;
}

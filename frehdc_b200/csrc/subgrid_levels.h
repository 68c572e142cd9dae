/*
 * subgrid_levels.h -- the subgrid lookup-table values of one coarse cell at one
 * water level, computed from the cell's r x r fine bottom elevations.
 *
 * This is the single definition of the subgrid tables in this code base.  The
 * host deck writer calls it to produce the V.dat/Z.dat/Vxp.dat/... files that the
 * reference model reads (level-major, x fastest), and the device calls the very
 * same inline function to evaluate a level on the fly (no N x Ne tables are held
 * on the GPU for large domains).  Both sides therefore see identical doubles as
 * long as neither contracts a*b+c into an FMA: the host is built without -mfma and
 * the kernels that use this header are built with --fmad=false.
 *
 * Semantics follow the reference's MATLAB pre-processor (not runnable here):
 *   preProcessing/script_CreateSubAreaWithBlockV16.m:153      bottom = min of block
 *   preProcessing/script_CreateSubAreaWithBlockV16.m:159-175  bottomXP/YP
 *   preProcessing/script_CreateSubAreaWithBlockV16.m:221-259  V, Z, Vxp/Vxm/Vyp/Vym
 *   preProcessing/ComputeSubgridFaceArea.m:8-40               Np/Nm/Op/Om
 * MATLAB arrays there are (x, y, level) with x the first (fastest) index, which is
 * the reference C layout ii = j*nx + i.  Summation order is fixed here: MATLAB's
 * sum(A(:)) is a flat x-fastest sweep and sum(sum(A)) is a sum of column (x) sums.
 *
 * Block check (checkBlock = 1, script_CreateSubAreaWithBlockV16.m:27,214-216,
 * 262-283 and ComputeFaceAreaWithBlockCheck.m:14-171), for 1 < r <= 8:
 *   1. a block's wet pixels (level > bottom) are reduced to their largest
 *      4-connected cluster (bwlabel(.,4), :33-55; equal sizes: the cluster that
 *      bwlabel numbers first, i.e. whose first pixel comes first in MATLAB's
 *      column-major scan, x fastest); a cluster below 0.01*r*r pixels leaves the
 *      block dry;
 *   2. a face between two blocks gets sum over its pixel pairs of
 *      min(depth masked by one block's cluster, depth masked by the other's) * dx
 *      (:127-172), which is zero exactly where the blocks' clusters do not touch
 *      across the face, so the cross-cell blocking flags (:88-123) change nothing
 *      further;
 *   3. a face on the domain boundary keeps its unmasked edge sum (:140-145,
 *      :162-167) unless the block's cluster has no pixel on that edge (:61-76).
 * V, Z and the half volumes never use the clusters.
 *
 * Fine array layout: zf[fj * fpitch + fi], fi in [0, nx*r) along x, fj along y.
 */
#ifndef FREHD_SUBGRID_LEVELS_H
#define FREHD_SUBGRID_LEVELS_H

#ifdef __CUDACC__
#define FREHD_HD __host__ __device__ __forceinline__
#else
#define FREHD_HD static inline
#endif

typedef struct frehd_cell_levels {
  double V, Z, Vxp, Vxm, Vyp, Vym, Np, Nm, Op, Om;
} frehd_cell_levels;

/* max(h - z, 0) of the pre-processor (script_CreateSubAreaWithBlockV16.m:221). */
FREHD_HD double frehd_fine_depth(double h, double z) {
  double d = h - z;
  return d > 0.0 ? d : 0.0;
}

FREHD_HD double frehd_min2(double a, double b) { return b < a ? b : a; }

/* Half-block split round(r/2) of the pre-processor (MATLAB round: .5 away from 0). */
FREHD_HD int frehd_half(int r) { return (r + 1) / 2; }

/* Wet pixels (h > z) of the r x r block at b, bit fj*r + fi (r <= 8). */
FREHD_HD unsigned long long frehd_wet_bits(const double *b, long fpitch, int r, double h) {
  unsigned long long m = 0;
  for (int fj = 0; fj < r; ++fj)
    for (int fi = 0; fi < r; ++fi)
      if (frehd_fine_depth(h, b[(long)fj * fpitch + fi]) > 0.0) m |= 1ull << (fj * r + fi);
  return m;
}

FREHD_HD int frehd_popc64(unsigned long long v) {
#ifdef __CUDA_ARCH__
  return __popcll(v);
#else
  return __builtin_popcountll(v);
#endif
}

/* The largest 4-connected cluster of the wet bits m of an r x r block (bit
 * fj*r + fi).  Clusters are grown from their lowest bit in increasing order, so
 * among equal sizes the one whose first pixel comes first in MATLAB's
 * column-major (x fastest) scan is kept, as bwlabel numbers it first.  A cluster
 * below 0.01*r*r pixels leaves the block dry (ComputeFaceAreaWithBlockCheck.m:33-55). */
FREHD_HD unsigned long long frehd_cluster_bits(unsigned long long m, int r) {
  const unsigned long long all = r * r >= 64 ? ~0ull : ((1ull << (r * r)) - 1ull);
  unsigned long long first = 0, last = 0;
  for (int fj = 0; fj < r; ++fj) {
    first |= 1ull << (fj * r);
    last |= 1ull << (fj * r + r - 1);
  }
  unsigned long long best = 0, rem = m & all;
  int best_n = 0;
  while (rem) {
    unsigned long long c = rem & (~rem + 1ull);
    for (;;) {
      unsigned long long g = c | ((c << 1) & ~first) | ((c >> 1) & ~last) | (c << r) | (c >> r);
      g &= m & all;
      if (g == c) break;
      c = g;
    }
    const int n = frehd_popc64(c);
    if (n > best_n) {
      best = c;
      best_n = n;
    }
    rem &= ~c;
  }
  if ((double)best_n < 0.01 * r * r) return 0;
  return best;
}

/* Cluster of block (i, j) at level h. */
FREHD_HD unsigned long long frehd_block_cluster(const double *zf, long fpitch, int r, int i, int j,
                                                double h) {
  return frehd_cluster_bits(frehd_wet_bits(zf + (long)j * r * fpitch + (long)i * r, fpitch, r, h), r);
}

FREHD_HD double frehd_masked(double d, unsigned long long m, int bit) {
  return ((m >> bit) & 1ull) ? d : 0.0;
}

/*
 * All ten table values of cell (i, j) at level h (level in the deck's own datum,
 * i.e. without the model's bathymetry offset).
 *   zf      fine bottom elevations, pitch fpitch (elements)
 *   dA      fine pixel area dxf*dyf, dxf fine width (face areas use dxf, as in
 *           ComputeSubgridFaceArea.m:18,30 which multiplies both by dx)
 */
FREHD_HD void frehd_cell_levels_at(const double *zf, long fpitch, int nx, int ny, int r,
                                   int i, int j, double h, double dA, double dxf,
                                   int check_block, frehd_cell_levels *o) {
  const long fi0 = (long)i * r, fj0 = (long)j * r;
  const double *b = zf + fj0 * fpitch + fi0;
  if (r == 1) {
    /* script_CreateSubAreaWithBlockV16.m:246-255 (r == 1 branch) */
    double d = frehd_fine_depth(h, b[0]);
    o->V = dA * d;
    o->Z = dA * (d > 0.0 ? 1.0 : 0.0);
    o->Vxp = o->Vyp = o->Vxm = o->Vym = dA * d / 2.0;
    o->Np = o->Op = o->Nm = o->Om = dxf * d;
    return;
  }
  const int hf = frehd_half(r);
  double sV = 0.0, cnt = 0.0, sxp = 0.0, sxm = 0.0, syp = 0.0, sym = 0.0;
  for (int fj = 0; fj < r; ++fj) {
    const double *row = b + (long)fj * fpitch;
    double cxp = 0.0, cxm = 0.0, call = 0.0;
    for (int fi = 0; fi < r; ++fi) {
      double d = frehd_fine_depth(h, row[fi]);
      sV += d;                         /* sum(localDepth(:)), x fastest */
      if (d > 0.0) cnt += 1.0;         /* sum(sum(localDepth > 0)) */
      if (fi < hf) cxm += d; else cxp += d;
      call += d;                       /* column sum over x for this y */
    }
    sxp += cxp;                        /* sum(sum(localDepth(hf+1:r, :))) */
    sxm += cxm;
    if (fj < hf) sym += call; else syp += call;
  }
  o->V = dA * sV;
  o->Z = dA * cnt;
  o->Vxp = dA * sxp;
  o->Vxm = dA * sxm;
  o->Vyp = dA * syp;
  o->Vym = dA * sym;

  if (check_block) {
    const unsigned long long mo = frehd_block_cluster(zf, fpitch, r, i, j, h);
    unsigned long long edge_w = 0, edge_e = 0, edge_s = 0, edge_n = 0;
    for (int q = 0; q < r; ++q) {
      edge_w |= 1ull << (q * r);
      edge_e |= 1ull << (q * r + r - 1);
      edge_s |= 1ull << q;
      edge_n |= 1ull << ((r - 1) * r + q);
    }
    double s = 0.0;
    if (i < nx - 1) {
      const unsigned long long me = frehd_block_cluster(zf, fpitch, r, i + 1, j, h);
      for (int fj = 0; fj < r; ++fj) {
        const double *row = b + (long)fj * fpitch;
        s += frehd_min2(frehd_masked(frehd_fine_depth(h, row[r - 1]), mo, fj * r + r - 1),
                        frehd_masked(frehd_fine_depth(h, row[r]), me, fj * r));
      }
    } else {
      for (int fj = 0; fj < r; ++fj) s += frehd_fine_depth(h, b[(long)fj * fpitch + r - 1]);
    }
    o->Np = (mo & edge_e) ? s * dxf : 0.0;
    s = 0.0;
    if (i > 0) {
      const unsigned long long mw = frehd_block_cluster(zf, fpitch, r, i - 1, j, h);
      for (int fj = 0; fj < r; ++fj) {
        const double *row = b + (long)fj * fpitch;
        s += frehd_min2(frehd_masked(frehd_fine_depth(h, row[-1]), mw, fj * r + r - 1),
                        frehd_masked(frehd_fine_depth(h, row[0]), mo, fj * r));
      }
    } else {
      for (int fj = 0; fj < r; ++fj) s += frehd_fine_depth(h, b[(long)fj * fpitch]);
    }
    o->Nm = (mo & edge_w) ? s * dxf : 0.0;
    s = 0.0;
    if (j < ny - 1) {
      const unsigned long long mn = frehd_block_cluster(zf, fpitch, r, i, j + 1, h);
      const double *r0 = b + (long)(r - 1) * fpitch, *r1 = b + (long)r * fpitch;
      for (int fi = 0; fi < r; ++fi)
        s += frehd_min2(frehd_masked(frehd_fine_depth(h, r0[fi]), mo, (r - 1) * r + fi),
                        frehd_masked(frehd_fine_depth(h, r1[fi]), mn, fi));
    } else {
      const double *r0 = b + (long)(r - 1) * fpitch;
      for (int fi = 0; fi < r; ++fi) s += frehd_fine_depth(h, r0[fi]);
    }
    o->Op = (mo & edge_n) ? s * dxf : 0.0;
    s = 0.0;
    if (j > 0) {
      const unsigned long long ms = frehd_block_cluster(zf, fpitch, r, i, j - 1, h);
      const double *r0 = b - fpitch;
      for (int fi = 0; fi < r; ++fi)
        s += frehd_min2(frehd_masked(frehd_fine_depth(h, r0[fi]), ms, (r - 1) * r + fi),
                        frehd_masked(frehd_fine_depth(h, b[fi]), mo, fi));
    } else {
      for (int fi = 0; fi < r; ++fi) s += frehd_fine_depth(h, b[fi]);
    }
    o->Om = (mo & edge_s) ? s * dxf : 0.0;
    return;
  }

  /* Np: own last x-row against the east neighbour's first x-row. */
  double s = 0.0;
  if (i < nx - 1) {
    for (int fj = 0; fj < r; ++fj) {
      const double *row = b + (long)fj * fpitch;
      s += frehd_min2(frehd_fine_depth(h, row[r - 1]), frehd_fine_depth(h, row[r]));
    }
  } else {
    for (int fj = 0; fj < r; ++fj) s += frehd_fine_depth(h, b[(long)fj * fpitch + r - 1]);
  }
  o->Np = s * dxf;
  /* Nm: west neighbour's last x-row against own first x-row; the first column of
   * the domain uses its own first row (ComputeSubgridFaceArea.m:23-24). */
  s = 0.0;
  if (i > 0) {
    for (int fj = 0; fj < r; ++fj) {
      const double *row = b + (long)fj * fpitch;
      s += frehd_min2(frehd_fine_depth(h, row[-1]), frehd_fine_depth(h, row[0]));
    }
  } else {
    for (int fj = 0; fj < r; ++fj) s += frehd_fine_depth(h, b[(long)fj * fpitch]);
  }
  o->Nm = s * dxf;
  /* Op: own last y-row against the north neighbour's first y-row. */
  s = 0.0;
  if (j < ny - 1) {
    const double *r0 = b + (long)(r - 1) * fpitch, *r1 = b + (long)r * fpitch;
    for (int fi = 0; fi < r; ++fi)
      s += frehd_min2(frehd_fine_depth(h, r0[fi]), frehd_fine_depth(h, r1[fi]));
  } else {
    const double *r0 = b + (long)(r - 1) * fpitch;
    for (int fi = 0; fi < r; ++fi) s += frehd_fine_depth(h, r0[fi]);
  }
  o->Op = s * dxf;
  /* Om: south neighbour's last y-row against own first y-row. */
  s = 0.0;
  if (j > 0) {
    const double *r0 = b - fpitch;
    for (int fi = 0; fi < r; ++fi)
      s += frehd_min2(frehd_fine_depth(h, r0[fi]), frehd_fine_depth(h, b[fi]));
  } else {
    for (int fi = 0; fi < r; ++fi) s += frehd_fine_depth(h, b[fi]);
  }
  o->Om = s * dxf;
}

/* Parts of the table values frehd_cell_levels_r4 computes. */
enum { FREHD_LV_ALL = 0, FREHD_LV_WEST = 1, FREHD_LV_SOUTH = 2 };

/*
 * frehd_cell_levels_at for r == 4, with every fine depth evaluated once: the face
 * areas reuse the block's own edge depths instead of recomputing them.  Same
 * operations in the same order, so the same doubles.  `part` selects all ten
 * values, or only the west-face pair (Nm, Vxm) or the south-face pair (Om, Vym)
 * that the west or south neighbour's face combination needs.  b points at the
 * cell's first fine pixel in an array of row pitch fpitch that also holds the
 * neighbouring pixels the faces read (the whole domain, or a staged window).
 */
FREHD_HD void frehd_cell_levels_r4_at(const double *b, long fpitch, int nx, int ny, int i, int j,
                                      double h, double dA, double dxf, int part,
                                      frehd_cell_levels *o) {
  (void)nx;
  double d[4][4];
  if (part == FREHD_LV_ALL) {
    for (int fj = 0; fj < 4; ++fj)
      for (int fi = 0; fi < 4; ++fi) d[fj][fi] = frehd_fine_depth(h, b[(long)fj * fpitch + fi]);
    double sV = 0.0, cnt = 0.0, sxp = 0.0, sxm = 0.0, syp = 0.0, sym = 0.0;
    for (int fj = 0; fj < 4; ++fj) {
      double cxp = 0.0, cxm = 0.0, call = 0.0;
      for (int fi = 0; fi < 4; ++fi) {
        const double dd = d[fj][fi];
        sV += dd;
        if (dd > 0.0) cnt += 1.0;
        if (fi < 2) cxm += dd; else cxp += dd;
        call += dd;
      }
      sxp += cxp;
      sxm += cxm;
      if (fj < 2) sym += call; else syp += call;
    }
    o->V = dA * sV;
    o->Z = dA * cnt;
    o->Vxp = dA * sxp;
    o->Vxm = dA * sxm;
    o->Vyp = dA * syp;
    o->Vym = dA * sym;
    double s = 0.0;
    if (i < nx - 1) {
      for (int fj = 0; fj < 4; ++fj)
        s += frehd_min2(d[fj][3], frehd_fine_depth(h, b[(long)fj * fpitch + 4]));
    } else {
      for (int fj = 0; fj < 4; ++fj) s += d[fj][3];
    }
    o->Np = s * dxf;
    s = 0.0;
    if (j < ny - 1) {
      const double *r1 = b + 4 * fpitch;
      for (int fi = 0; fi < 4; ++fi) s += frehd_min2(d[3][fi], frehd_fine_depth(h, r1[fi]));
    } else {
      for (int fi = 0; fi < 4; ++fi) s += d[3][fi];
    }
    o->Op = s * dxf;
  } else if (part == FREHD_LV_WEST) {
    for (int fj = 0; fj < 4; ++fj)
      for (int fi = 0; fi < 2; ++fi) d[fj][fi] = frehd_fine_depth(h, b[(long)fj * fpitch + fi]);
    double sxm = 0.0;
    for (int fj = 0; fj < 4; ++fj) {
      double cxm = 0.0;
      cxm += d[fj][0];
      cxm += d[fj][1];
      sxm += cxm;
    }
    o->Vxm = dA * sxm;
  } else {
    for (int fj = 0; fj < 2; ++fj)
      for (int fi = 0; fi < 4; ++fi) d[fj][fi] = frehd_fine_depth(h, b[(long)fj * fpitch + fi]);
    double sym = 0.0;
    for (int fj = 0; fj < 2; ++fj) {
      double call = 0.0;
      for (int fi = 0; fi < 4; ++fi) call += d[fj][fi];
      sym += call;
    }
    o->Vym = dA * sym;
  }
  if (part != FREHD_LV_SOUTH) {  /* Nm: west neighbour's last x-row against own first */
    double s = 0.0;
    if (i > 0) {
      for (int fj = 0; fj < 4; ++fj)
        s += frehd_min2(frehd_fine_depth(h, b[(long)fj * fpitch - 1]), d[fj][0]);
    } else {
      for (int fj = 0; fj < 4; ++fj) s += d[fj][0];
    }
    o->Nm = s * dxf;
  }
  if (part != FREHD_LV_WEST) {  /* Om: south neighbour's last y-row against own first */
    double s = 0.0;
    if (j > 0) {
      const double *r0 = b - fpitch;
      for (int fi = 0; fi < 4; ++fi) s += frehd_min2(frehd_fine_depth(h, r0[fi]), d[0][fi]);
    } else {
      for (int fi = 0; fi < 4; ++fi) s += d[0][fi];
    }
    o->Om = s * dxf;
  }
}

/* The same with the fine bottoms zf[fj * fpitch + fi] of the whole domain. */
FREHD_HD void frehd_cell_levels_r4(const double *zf, long fpitch, int nx, int ny, int i, int j,
                                   double h, double dA, double dxf, int part,
                                   frehd_cell_levels *o) {
  frehd_cell_levels_r4_at(zf + (long)j * 4 * fpitch + (long)i * 4, fpitch, nx, ny, i, j, h, dA, dxf,
                          part, o);
}

/* Coarse bottom and face-bottom elevations of cell (i, j) (host pre-processing;
 * script_CreateSubAreaWithBlockV16.m:153,159-175). */
FREHD_HD void frehd_cell_bottoms(const double *zf, long fpitch, int nx, int ny, int r,
                                 int i, int j, double *bottom, double *bxp, double *byp) {
  const long fi0 = (long)i * r, fj0 = (long)j * r;
  const double *b = zf + fj0 * fpitch + fi0;
  double m = b[0];
  for (int fj = 0; fj < r; ++fj)
    for (int fi = 0; fi < r; ++fi) {
      double z = b[(long)fj * fpitch + fi];
      if (z < m) m = z;
    }
  *bottom = m;
  /* bottomXP = max over the two fine x-rows at the face of (min along y). */
  double m0 = b[r - 1];
  for (int fj = 1; fj < r; ++fj) m0 = frehd_min2(m0, b[(long)fj * fpitch + r - 1]);
  if (i < nx - 1) {
    double m1 = b[r];
    for (int fj = 1; fj < r; ++fj) m1 = frehd_min2(m1, b[(long)fj * fpitch + r]);
    *bxp = m1 > m0 ? m1 : m0;
  } else {
    *bxp = m0;
  }
  /* bottomYP = max over the two fine y-rows at the face of (min along x). */
  const double *r0 = b + (long)(r - 1) * fpitch;
  double n0 = r0[0];
  for (int fi = 1; fi < r; ++fi) n0 = frehd_min2(n0, r0[fi]);
  if (j < ny - 1) {
    const double *r1 = b + (long)r * fpitch;
    double n1 = r1[0];
    for (int fi = 1; fi < r; ++fi) n1 = frehd_min2(n1, r1[fi]);
    *byp = n1 > n0 ? n1 : n0;
  } else {
    *byp = n0;
  }
}

/* Level h_k of the reference's level vector before the offset is added
 * (subgrid.c:2118: allSurf[k] = surfmin + k*dsurf + offset, evaluated left to right). */
FREHD_HD double frehd_level(double surfmin, double dsurf, int k) {
  return surfmin + (double)k * dsurf;
}

#endif /* FREHD_SUBGRID_LEVELS_H */

"""Block-check face areas of the subgrid pre-processor, restated from the
reference's MATLAB.  Test infrastructure: the checker of frehd_build_tables_ex
and of the device evaluation with FREHD_GEOM_BLOCK_CHECK.

Follows preProcessing/ComputeFaceAreaWithBlockCheck.m:14-171 step by step:
  step 1 (:26-81)   each r x r block keeps its largest 4-connected wet cluster
                    (bwlabel(., 4), first maximum); intra-block blocking flags
                    for block edges without a wet pixel;
  step 2 (:83-124)  cross-block flags for faces whose cleaned edges share no wet
                    pixel pair (loops from the second block in both directions);
  step 3 (:126-173) face areas: sum of min(masked depths) over the face's pixel
                    pairs times dx, unmasked edge sums on the domain boundary;
and preProcessing/script_CreateSubAreaWithBlockV16.m:262-283, which sets every
flagged face area to zero.

MATLAB's arrays are (x, y) with x the first index; bathCenter is the fine
bottom field zf transposed.  bwlabel numbers clusters in column-major order (x
fastest); scipy.ndimage.label scans row-major, so it is given the block as
(y, x), which visits the pixels in the same order and numbers the clusters the
same way.  Sums run in index order (the order frehd_build_tables_ex fixes; the
MATLAB pre-processor itself cannot run here, so this restatement is the pin).
"""
from __future__ import annotations

import numpy as np
from scipy import ndimage

_FOUR = np.array([[0, 1, 0], [1, 1, 1], [0, 1, 0]])


def _seqsum(v) -> float:
    s = 0.0
    for x in v:
        s += float(x)
    return s


def _clean(cell_xy: np.ndarray, r: int) -> np.ndarray:
    """Step 1 for one block given as (x, y) booleans."""
    lab_yx, nw = ndimage.label(cell_xy.T, structure=_FOUR)
    if nw == 0:
        return np.zeros_like(cell_xy)
    lab = lab_yx.T
    sizes = [int(np.sum(lab == p)) for p in range(1, nw + 1)]
    best = 1 + int(np.argmax(sizes))          # MATLAB max: the first maximum
    bb = lab == best
    if bb.sum() < 0.01 * r * r:
        return np.zeros_like(cell_xy)
    return bb


def face_areas(zf: np.ndarray, nx: int, ny: int, r: int, dxf: float, h: float):
    """Np, Nm, Op, Om of every block at level h, each (nx, ny) indexed [i, j]."""
    B = np.asarray(zf, dtype=np.float64)[: ny * r, : nx * r].T   # bathCenter(x, y)
    depth = np.maximum(h - B, 0.0)
    binary = h > B
    blk = {k: np.zeros((nx, ny), dtype=bool) for k in ("Np", "Nm", "Op", "Om")}
    clean = np.zeros_like(binary)
    for ii in range(nx):
        for jj in range(ny):
            xs, ys = slice(ii * r, (ii + 1) * r), slice(jj * r, (jj + 1) * r)
            c = _clean(binary[xs, ys], r)
            if not c[0, :].any():
                blk["Nm"][ii, jj] = True
            if not c[-1, :].any():
                blk["Np"][ii, jj] = True
            if not c[:, 0].any():
                blk["Om"][ii, jj] = True
            if not c[:, -1].any():
                blk["Op"][ii, jj] = True
            clean[xs, ys] = c
    for ii in range(1, nx):
        for jj in range(1, ny):
            this = clean[ii * r:(ii + 1) * r, jj * r:(jj + 1) * r]
            west = clean[(ii - 1) * r:ii * r, jj * r:(jj + 1) * r]
            south = clean[ii * r:(ii + 1) * r, (jj - 1) * r:jj * r]
            if not np.any(this[0, :] & west[-1, :]):
                blk["Nm"][ii, jj] = True
                blk["Np"][ii - 1, jj] = True
            if not np.any(this[:, 0] & south[:, -1]):
                blk["Om"][ii, jj] = True
                blk["Op"][ii, jj - 1] = True
    A = {k: np.zeros((nx, ny)) for k in ("Np", "Nm", "Op", "Om")}
    X, Y = nx * r, ny * r
    for ii in range(nx):
        for jj in range(ny):
            i1, i2 = ii * r, (ii + 1) * r - 1
            j1, j2 = jj * r, (jj + 1) * r - 1
            if i2 != X - 1:
                dp = np.where(clean[i2, j1:j2 + 1], depth[i2, j1:j2 + 1], 0.0)
                dm = np.where(clean[i2 + 1, j1:j2 + 1], depth[i2 + 1, j1:j2 + 1], 0.0)
                s = _seqsum(np.minimum(dp, dm)) * dxf
                A["Np"][ii, jj] = s
                A["Nm"][ii + 1, jj] = s
            else:
                A["Np"][ii, jj] = _seqsum(depth[i2, j1:j2 + 1]) * dxf
                A["Nm"][0, jj] = _seqsum(depth[0, j1:j2 + 1]) * dxf
            if j2 != Y - 1:
                dp = np.where(clean[i1:i2 + 1, j2], depth[i1:i2 + 1, j2], 0.0)
                dm = np.where(clean[i1:i2 + 1, j2 + 1], depth[i1:i2 + 1, j2 + 1], 0.0)
                s = _seqsum(np.minimum(dp, dm)) * dxf
                A["Op"][ii, jj] = s
                A["Om"][ii, jj + 1] = s
            else:
                A["Op"][ii, jj] = _seqsum(depth[i1:i2 + 1, j2]) * dxf
                A["Om"][ii, 0] = _seqsum(depth[i1:i2 + 1, 0]) * dxf
    for k in A:
        A[k][blk[k]] = 0.0
    return A["Np"], A["Nm"], A["Op"], A["Om"]


def face_tables(zf: np.ndarray, nx: int, ny: int, r: int, dxf: float, surfmin: float,
                dsurf: float, Ne: int) -> np.ndarray:
    """(4, Ne, N) tables Np, Nm, Op, Om in the reference layout (level-major,
    ii = j*nx + i), at the levels surfmin + k*dsurf (subgrid.c:2118 before the
    offset)."""
    out = np.empty((4, Ne, nx * ny))
    for k in range(Ne):
        h = surfmin + float(k) * dsurf
        for q, a in enumerate(face_areas(zf, nx, ny, r, dxf, h)):
            out[q, k] = a.T.reshape(-1)            # [j, i] -> ii = j*nx + i
    return out

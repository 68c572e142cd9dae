"""Shared helpers of the parity tests (decks, phase comparison)."""
from __future__ import annotations

import os

import numpy as np

from frehdc_b200 import deck as D

# Arrays of one step's state, in the reference layout, compared between runs.
STATE = ["surf", "uuXP", "vvYP", "uuYP", "vvXP", "S", "depth", "CDXP", "CDYP", "CFLx", "CFLy",
         "V", "Z", "Nx", "Oy", "Vx", "Vy", "Zx", "Zy", "ind"]
TEMPS = ["surfOld", "EnXP", "EnYP", "DragXP", "DragYP", "Fuu", "Fvv", "cellV", "Sm", "rmvCFL",
         "wtfXP", "wtfYP", "advX", "advY", "depthXP", "depthYP", "GnCt", "GnXP", "GnXM", "GnYP",
         "GnYM", "z", "Vxp", "Vyp", "Vxm", "Vym", "Np", "Nm", "Op", "Om"]
EXPLICIT_OUT = ["EnXP", "EnYP", "DragXP", "DragYP", "advX", "advY", "GnCt", "GnXP", "GnXM",
                "GnYP", "GnYM", "z"]

# The small decks of the CPU parity suite.
SPECS = {
    "wet48x40": D.DeckSpec(nx=48, ny=40, steps=30, seed=3),
    "dry40x36": D.DeckSpec(nx=40, ny=36, steps=40, seed=5, dry_frac=0.3),
    "dry37x29": D.DeckSpec(nx=37, ny=29, steps=40, seed=9, dry_frac=0.35, dt=2.0, depth_max=3.0),
    # TVD (superbee) scalar advection, scalar.c:99-249
    "tvd44x36": D.DeckSpec(nx=44, ny=36, steps=40, seed=13, dry_frac=0.3, dt=2.0,
                           scalar_adv=2, scalar_sigma=60.0),
    # the same with fewer dry cells: its runs do not reach the scalar-singularity
    # branch, so whole runs compare to the solve's rounding (with 30 % dry cells
    # two converged CPU solves, SSOR and Jacobi, already differ by 1e-6 in eta)
    "tvdwet44x36": D.DeckSpec(nx=44, ny=36, steps=40, seed=13, dry_frac=0.15, dt=2.0,
                              scalar_adv=2, scalar_sigma=60.0),
    # inflow cells (configuration.c:53-60, subgrid.c:959-968,1236-1241,1648-1666)
    # and wind with the thin-layer decay (nsfunctions.c:609-648)
    "inflow36x30": D.DeckSpec(nx=36, ny=30, steps=30, seed=21, dry_frac=0.3,
                              inflow_cells=(4, 7, 2, 4), inflow_q=3.0, inflow_s=35.0),
    "wind40x32": D.DeckSpec(nx=40, ny=32, steps=30, seed=23, dry_frac=0.3,
                            wind_speed=9.0, wind_dir=60.0, north_angle=15.0),
}

_cache: dict = {}


def deck_for(name: str, root: str):
    """Generated deck (with tables) and its reference-format directory."""
    if name in _cache:
        return _cache[name]
    spec = SPECS[name]
    d = D.make_deck(spec, with_tables=True)
    path = os.path.join(root, name)
    D.write_reference_deck(d, path)
    _cache[name] = (d, path)
    return d, path


def mismatches(a: dict, b: dict, names, exact: bool = True, rtol: float = 0.0):
    """List of (name, count, first indices) where a[name] != b[name]."""
    out = []
    for n in names:
        x = np.asarray(a[n], dtype=np.float64)
        y = np.asarray(b[n], dtype=np.float64)
        if x.shape != y.shape:
            out.append((n, "shape", x.shape, y.shape))
            continue
        same = (x == y) | (np.isnan(x) & np.isnan(y))
        if not exact:
            scale = max(np.max(np.abs(y)), 1e-300)
            same = np.abs(x - y) <= rtol * scale
        bad = np.where(~same)[0]
        if len(bad):
            out.append((n, int(len(bad)), bad[:4].tolist(), x[bad[:2]].tolist(), y[bad[:2]].tolist()))
    return out


def inflow_source(d, tt: int) -> np.ndarray:
    """Volume each cell receives from the deck's inflow at step tt: every inflow
    cell gets the whole inflow times dt (subgrid.c:1236-1241), while the
    continuity equation shares it among them (subgrid.c:959-968)."""
    N = d.nx * d.ny
    src = np.zeros(N)
    if d.spec.inflow_cells:
        q = D.forcing_series(d)["inflow"]
        qt = q[tt] if tt < len(q) else 0.0
        i0, i1, j0, j1 = d.spec.inflow_cells
        for j in range(j0, j1):
            for i in range(i0, i1):
                src[j * d.nx + i] = qt * d.spec.dt
    return src


def max_rel(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = max(float(np.max(np.abs(b))), 1e-300)
    return float(np.max(np.abs(a - b))) / scale


def ledger_residual(V_old, cellV, Fuu, Fvv, nx: int, ny: int, dt: float, source=None) -> float:
    """Relative misclosure of one step's volume ledger (volumeByFluxSub,
    subgrid.c:1227-1263): the cell volumes after the flux update must add up to
    the volumes before it plus dt times the net inflow through the domain's
    outer faces, plus the volume the inflow cells receive (`source`, per cell,
    added before the clip), plus the water added where a negative volume was
    clipped to 0.  Arrays in the reference layout (ghost ring after the N
    interior cells)."""
    N = nx * ny
    ii = np.arange(N)
    i, j = ii % nx, ii // nx
    iM = np.where(i == 0, N + 2 * nx + ny + j, ii - 1)   # iMjc (map.c)
    jM = np.where(j == 0, N + nx + i, ii - nx)           # icjM
    raw = V_old[:N] + dt * (Fuu[iM] - Fuu[:N] + Fvv[jM] - Fvv[:N])
    src = np.zeros(N) if source is None else np.asarray(source, dtype=np.float64)
    raw = raw + src
    clip_added = float(np.sum(np.where(raw < 0, -raw, 0.0)))
    # outer faces: west (ghost column), east (i = nx-1), south (ghost row), north (j = ny-1)
    west = Fuu[N + 2 * nx + ny + np.arange(ny)]
    east = Fuu[np.arange(ny) * nx + nx - 1]
    south = Fvv[N + nx + np.arange(nx)]
    north = Fvv[(ny - 1) * nx + np.arange(nx)]
    inflow = float(np.sum(west) - np.sum(east) + np.sum(south) - np.sum(north))
    total = float(np.sum(cellV[:N]))
    want = float(np.sum(V_old[:N])) + dt * inflow + float(np.sum(src)) + clip_added
    return abs(total - want) / max(abs(total), 1e-300)

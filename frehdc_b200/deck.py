"""Synthetic FrehdC decks: seeded bathymetry, tide and initial fields, written in
the reference model's own input formats (``data.dat`` + ``input/`` folder).

The reference has no shipped benchmark deck for the subgrid configurations it is
measured on, so decks are generated from a seed.  The recipe (Gaussian random
field bathymetry, r x r fine roughness, sine tide on the tidal row, Gaussian
scalar plume) is deterministic: numpy ``default_rng`` streams keyed by the seed.

Orientation: the reference applies its tide on the YP row j = ny-1 (bcType = 1,
configuration.c:147-148).  The generator measures the along-basin coordinate
``xb`` from that row (xb = 0 at the tidal edge, growing landward), so the tidal
edge of a basin description sits on the reference's YP row.

File formats follow the reader code of the reference:
  data.dat          FREHD.c:30-63 (positional, ';' terminated, '#' comments)
  bottom*.dat       bathymetry.c:56-89 (N values, x fastest)
  subdata tables    subgrid.c:2089-2109 (Ne*N values, x fastest, then y, then level)
  tideP/inflow.dat  initialize.c:447-477 ("t,value" pairs, t in epoch seconds)
  surfic/scalaric   initialize.c:279-327 (N values)
Values are written with %.17g so fscanf("%lf") reads back the identical double.
"""
from __future__ import annotations

import calendar
import dataclasses
import math
import os
from dataclasses import dataclass, field

import numpy as np

# Order of the 10 subgrid tables in frehd_build_tables' output.
TABLE_NAMES = ("V", "Z", "Vxp", "Vxm", "Vyp", "Vym", "Np", "Nm", "Op", "Om")
DEFAULT_START = "2013-06-10"


@dataclass
class DeckSpec:
    """Parameters of one synthetic subgrid deck."""
    nx: int = 128
    ny: int = 128
    dx: float = 10.0
    r: int = 4                      # fine pixels per coarse cell edge
    dt: float = 1.0
    steps: int = 200
    manning_n: float = 0.03
    corr_len: float = 200.0         # correlation length of the bathymetry field [m]
    depth_min: float = 0.5          # shallowest / deepest coarse depth below datum [m]
    depth_max: float = 5.0
    slope: float = 1e-4             # bed rises landward by slope * xb
    roughness: float = 0.2          # fine pixels: +U(-roughness, roughness) [m]
    dry_frac: float | None = None   # if set: ~this fraction of cells above low tide
    tide_amp: float = 0.3
    tide_period: float = 44712.0    # 12.42 h
    eta0_amp: float = 0.05
    scalar_sigma: float = 100.0
    scalar_peak: float = 1.0
    scalar_in_window: bool = False  # plume at the centre of the (cropped) window, not the basin
    block_check: bool = False       # checkBlock = 1 face areas (largest wet cluster per block)
    scalar_adv: int = 1             # scalarAdv: 1 first-order upwind, 2 TVD (superbee)
    # inflow cells (i0, i1, j0, j1), half-open, 0-based; None = none.  The inflow
    # is inflow_q * (1 + 0.5 sin(2 pi t / 3 h)) m^3/s over all of them, carrying
    # scalar at concentration inflow_s
    inflow_cells: tuple | None = None
    inflow_q: float = 0.0
    inflow_s: float = 0.0
    # wind (useWind = 1 when wind_speed > 0): speed wind_speed * (1 + 0.3 sin(.)),
    # direction wind_dir + 20 sin(.) degrees from north, before north_angle
    wind_speed: float = 0.0
    wind_dir: float = 0.0
    north_angle: float = 0.0
    # scalars carried (nscalar): S plus n_scalars - 1 tracers, plumes like S's
    # placed around it (see _tracer_fields)
    n_scalars: int = 1
    # initial east-face velocity (uuic.dat, useConstU0 = 0): (i0, i1, j0, j1, value)
    # sets u = value on cells i in [i0, i1), j in [j0, j1); None = u starts at 0
    u0_block: tuple | None = None
    dsurf: float = 0.01
    eps: float = 1e-12
    max_iter: int = 100000
    use_thin_layer: int = 1
    seed: int = 1
    # open water along the tidal row: within sea_margin*L of it the bed is capped
    # at -(tide_amp + 1) m, relaxing quadratically to no cap at sea_margin*L
    sea_margin: float = 0.08
    # sub-window of a larger deck: (i0, j0, nx_full, ny_full); None = whole deck
    crop: tuple | None = None

    def replace(self, **kw) -> "DeckSpec":
        return dataclasses.replace(self, **kw)


@dataclass
class Deck:
    spec: DeckSpec
    nx: int
    ny: int
    r: int
    zf: np.ndarray          # (ny*r, nx*r) fine bottoms, deck datum
    bottom: np.ndarray      # (N,) coarse bottom.dat
    bottomXP: np.ndarray    # (N,)
    bottomYP: np.ndarray    # (N,)
    surf0: np.ndarray       # (N,) initial surface, deck datum
    S0: np.ndarray          # (N,) initial scalar
    surfmin: float
    surfmax: float
    dsurf: float
    Ne: int
    start: str
    tide_t: np.ndarray      # tideP.dat times (epoch s)
    tide_v: np.ndarray      # tideP.dat values (m)
    Nt: int                 # steps the data.dat allows (configuration.c:26)
    NT_days: float
    offset: float           # bathymetry offset the model adds (bathymetry.c:98-102)
    inflow_v: np.ndarray | None = None   # inflow.dat values at tide_t (m^3/s)
    wspd_v: np.ndarray | None = None     # windspd.dat values at tide_t (m/s)
    wdir_v: np.ndarray | None = None     # winddir.dat values at tide_t (degrees)
    tracers: list = field(default_factory=list)  # (N,) initial fields of tracers 1 ..
    u0: np.ndarray | None = None         # (N,) initial uuXP (uuic.dat); None = zero
    extra: dict = field(default_factory=dict)

    @property
    def N(self) -> int:
        return self.nx * self.ny


# --------------------------------------------------------------------------- fields
def _grf(ny: int, nx: int, dx: float, corr_len: float, seed: int) -> np.ndarray:
    """Gaussian random field on the coarse grid, min-max scaled to [0, 1]."""
    rng = np.random.default_rng([seed, 1])
    w = rng.standard_normal((ny, nx))
    ky = np.fft.fftfreq(ny, d=dx)
    kx = np.fft.fftfreq(nx, d=dx)
    k2 = ky[:, None] ** 2 + kx[None, :] ** 2
    filt = np.exp(-0.5 * (2.0 * np.pi) ** 2 * corr_len ** 2 * k2)
    f = np.real(np.fft.ifft2(np.fft.fft2(w) * filt))
    f -= f.min()
    mx = f.max()
    return f / mx if mx > 0 else f


def _xb(j: np.ndarray, ny: int, dy: float) -> np.ndarray:
    """Along-basin distance from the tidal (YP) row to cell centre j."""
    return (ny - 1 - j + 0.5) * dy


def _sea_cap(spec: DeckSpec, xb: np.ndarray, L: float) -> np.ndarray:
    """Upper bound of the bed near the tidal row (open water at the sea edge)."""
    zsea = -(spec.tide_amp + 1.0)
    m = max(spec.sea_margin * L, 1e-9)
    t = np.clip(xb / m, 0.0, 1.0)
    cap = zsea * (1.0 - t) ** 2
    return np.where(xb < m, cap, np.inf)


def _coarse_elevation(spec: DeckSpec, nxf: int, nyf: int) -> np.ndarray:
    """Coarse bed elevation (deck datum) of the full (uncropped) deck."""
    return np.minimum(_coarse_elevation_raw(spec, nxf, nyf),
                      _sea_cap(spec, _xb(np.arange(nyf)[:, None], nyf, spec.dx), nyf * spec.dx))


def _coarse_elevation_raw(spec: DeckSpec, nxf: int, nyf: int) -> np.ndarray:
    f = _grf(nyf, nxf, spec.dx, spec.corr_len, spec.seed)
    j = np.arange(nyf)[:, None]
    ramp = spec.slope * _xb(j, nyf, spec.dx)
    if spec.dry_frac is None:
        z = -(spec.depth_min + (spec.depth_max - spec.depth_min) * (1.0 - f))
        return z + ramp
    # z = -depth_max + span * f, span chosen so that ~dry_frac of the cells lie
    # above low tide (-tide_amp)
    base = -spec.depth_max + ramp
    lo, hi = 1e-3, 100.0
    for _ in range(80):
        span = 0.5 * (lo + hi)
        frac = np.mean(base + span * f > -spec.tide_amp)
        if frac > spec.dry_frac:
            hi = span
        else:
            lo = span
    return base + 0.5 * (lo + hi) * f


def _bilinear_rows(zc: np.ndarray, r: int, fj0: int, fj1: int, fi0: int, fi1: int) -> np.ndarray:
    """Bilinear interpolation of the coarse field at fine pixel centres."""
    nyc, nxc = zc.shape
    yc = np.clip((np.arange(fj0, fj1) + 0.5) / r - 0.5, 0.0, nyc - 1.0)
    xc = np.clip((np.arange(fi0, fi1) + 0.5) / r - 0.5, 0.0, nxc - 1.0)
    j0 = np.minimum(np.floor(yc).astype(np.int64), nyc - 2 if nyc > 1 else 0)
    i0 = np.minimum(np.floor(xc).astype(np.int64), nxc - 2 if nxc > 1 else 0)
    wy = (yc - j0)[:, None]
    wx = (xc - i0)[None, :]
    j1 = np.minimum(j0 + 1, nyc - 1)
    i1 = np.minimum(i0 + 1, nxc - 1)
    a = zc[j0][:, i0]
    b = zc[j0][:, i1]
    c = zc[j1][:, i0]
    d = zc[j1][:, i1]
    return (1 - wy) * ((1 - wx) * a + wx * b) + wy * ((1 - wx) * c + wx * d)


def _fine_noise(seed: int, fj: int, nxf_fine: int, lo: int, hi: int, rough: float) -> np.ndarray:
    rng = np.random.default_rng([seed, 7, fj])
    return rng.uniform(-rough, rough, size=nxf_fine)[lo:hi]


def _host(host):
    """The pre-processing builders (build_bottoms, build_tables): this library's
    by default; any module with the same two functions may stand in."""
    if host is None:
        from . import native as host
    return host


def make_deck(spec: DeckSpec, start: str = DEFAULT_START, with_tables: bool = False,
              host=None) -> Deck:
    """Generate a deck (fine bottoms, coarse bottoms, initial fields, tide series)."""
    r = spec.r
    if spec.crop is None:
        i0, j0, nxf, nyf = 0, 0, spec.nx, spec.ny
    else:
        i0, j0, nxf, nyf = spec.crop
    nx, ny = spec.nx, spec.ny
    zc = _coarse_elevation(spec, nxf, nyf)
    zf = _bilinear_rows(zc, r, j0 * r, (j0 + ny) * r, i0 * r, (i0 + nx) * r)
    for fj in range(ny * r):
        zf[fj] += _fine_noise(spec.seed, j0 * r + fj, nxf * r, i0 * r, (i0 + nx) * r, spec.roughness)
    zf = np.ascontiguousarray(zf)
    bottom, bxp, byp = _host(host).build_bottoms(zf, nx, ny, r)

    # initial surface: eta0 sine along the basin, scalar plume at the basin centre
    jj, ii = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    xb_full = _xb(jj + j0, nyf, spec.dx)
    L = nyf * spec.dx
    surf0 = spec.eta0_amp * np.sin(2.0 * np.pi * xb_full / L)
    if spec.scalar_in_window:
        xcen = (ii + 0.5) * spec.dx - 0.5 * nx * spec.dx
        ycen = (jj + 0.5) * spec.dx - 0.5 * ny * spec.dx
    else:
        xcen = ((ii + i0) + 0.5) * spec.dx - 0.5 * nxf * spec.dx
        ycen = ((jj + j0) + 0.5) * spec.dx - 0.5 * nyf * spec.dx
    S0 = spec.scalar_peak * np.exp(-(xcen ** 2 + ycen ** 2) / (2.0 * spec.scalar_sigma ** 2))
    W, H = (nx, ny) if spec.scalar_in_window else (nxf, nyf)
    tracers = _tracer_fields(spec, xcen, ycen, W * spec.dx, H * spec.dx)

    lo_eta = min(-spec.tide_amp, -spec.eta0_amp)
    hi_eta = max(spec.tide_amp, spec.eta0_amp)
    surfmin = round(lo_eta - 0.05, 6)
    surfmax = round(hi_eta + 0.05, 6)
    Ne = int(round((surfmax - surfmin) / spec.dsurf))     # subgrid.c:2115

    # time axis: Nt = NT_days*86400/dt truncated (configuration.c:26) must exceed steps
    NT_days = (spec.steps + 3) * spec.dt / 86400.0
    Nt = int(NT_days * 86400 / spec.dt)
    while Nt < spec.steps + 2:
        NT_days *= 1.0 + 1e-9
        Nt = int(NT_days * 86400 / spec.dt)
    t0 = float(calendar.timegm((int(start[0:4]), int(start[5:7]), int(start[8:10]), 0, 0, 0)))
    itval = 60.0
    M = int(math.ceil(Nt * spec.dt / itval)) + 4
    tide_t = t0 + itval * np.arange(M)
    tide_v = spec.tide_amp * np.sin(2.0 * np.pi * (tide_t - t0) / spec.tide_period)

    zmin = float(bottom.min())
    offset = 0.0 if zmin >= 0 else -zmin            # bathymetry.c:98-102
    ph = 2.0 * np.pi * (tide_t - t0) / 10800.0
    inflow_v = spec.inflow_q * (1.0 + 0.5 * np.sin(ph)) if spec.inflow_cells else None
    wspd_v = spec.wind_speed * (1.0 + 0.3 * np.sin(ph)) if spec.wind_speed > 0 else None
    wdir_v = spec.wind_dir + 20.0 * np.sin(0.7 * ph) if spec.wind_speed > 0 else None
    u0 = None
    if spec.u0_block is not None:
        bi0, bi1, bj0, bj1, uval = spec.u0_block
        u0 = np.zeros((ny, nx))
        u0[bj0:bj1, bi0:bi1] = uval
        u0 = u0.reshape(-1)
    deck = Deck(spec=spec, nx=nx, ny=ny, r=r, zf=zf, bottom=bottom, bottomXP=bxp, bottomYP=byp,
                surf0=surf0.reshape(-1).copy(), S0=S0.reshape(-1).copy(), surfmin=surfmin,
                surfmax=surfmax, dsurf=spec.dsurf, Ne=Ne, start=start, tide_t=tide_t,
                tide_v=tide_v, Nt=Nt, NT_days=NT_days, offset=offset, inflow_v=inflow_v,
                wspd_v=wspd_v, wdir_v=wdir_v, tracers=tracers, u0=u0)
    if with_tables:
        deck.extra["tables"] = build_tables(deck, host)
    return deck


def make_decks(specs, procs: int | None = None) -> list:
    """make_deck of every spec, on a pool of spawned worker processes when
    there are several (the generator is single-threaded numpy).  Spawned, not
    forked: a worker never inherits a CUDA context of the caller."""
    specs = list(specs)
    n = procs or min(16, os.cpu_count() or 1, len(specs))
    if n <= 1 or len(specs) < 4:
        return [make_deck(sp) for sp in specs]
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(n) as pool:
        return pool.map(make_deck, specs, chunksize=1)


def build_tables(deck: Deck, host=None) -> np.ndarray:
    """(10, Ne, N) subgrid tables of a deck (frehd_build_tables)."""
    return _host(host).build_tables(deck.zf, deck.nx, deck.ny, deck.r, deck.spec.dx / deck.r,
                                    deck.spec.dx / deck.r, deck.surfmin, deck.dsurf, deck.Ne,
                                    block_check=deck.spec.block_check)


# --------------------------------------------------------------------------- tide
def tide_series(deck: Deck) -> np.ndarray:
    """bc->tideP[0..Nt) as the reference computes it from tideP.dat."""
    return bc_series(deck, deck.tide_v)


def forcing_series(deck: Deck) -> dict:
    """bc->inflow / windspd / winddir[0..Nt) of the deck's forcing (only those
    its data.dat switches on)."""
    out = {}
    if deck.inflow_v is not None:
        out["inflow"] = bc_series(deck, deck.inflow_v)
    if deck.wspd_v is not None:
        out["windspd"] = bc_series(deck, deck.wspd_v)
        out["winddir"] = bc_series(deck, deck.wdir_v)
    return out


def bc_series(deck: Deck, v: np.ndarray) -> np.ndarray:
    """One BC array [0..Nt) as the reference computes it from a "t,value" file
    on the deck's time axis.

    Restates readOneBC/searchInd/dataInterp (initialize.c:447-477,
    utilities.c:65-86,129-148) with the same double arithmetic.
    """
    t = deck.tide_t
    dt = deck.spec.dt
    itval = int(t[1] - t[0])
    t_start = float(t[0])
    # searchInd: first index with |t - tNStart| <= itval/2
    ind = 0
    for c in range(len(t) + 1):
        if abs(t[c] - t_start) <= itval / 2:
            ind = c
            break
    y = np.empty(deck.Nt)
    kk = ind
    for ii in range(deck.Nt):
        tc = t_start + ii * dt
        if ii > 0 and tc > t[kk + 1]:
            kk += 1
        slope = (v[kk + 1] - v[kk]) / (t[kk + 1] - t[kk])
        intercept = v[kk] - slope * t[kk]
        y[ii] = slope * tc + intercept
    return y


# --------------------------------------------------------------------------- writer
def _fmt(x) -> str:
    return "%.17g" % x


def _write_column(path: str, arr: np.ndarray) -> None:
    arr = np.asarray(arr, dtype=np.float64).reshape(-1)
    with open(path, "w") as f:
        f.write("\n".join(map(_fmt, arr.tolist())))
        f.write("\n")


def data_dat_values(deck: Deck, out_hours: float | None = None) -> list:
    """The 88 positional values of data.dat (configuration.c:23-127).

    The default output interval lies beyond the last step (OutItvl must fit an
    int: configuration.c:27 truncates hours*3600/dt into one).
    """
    s = deck.spec
    if out_hours is None:
        out_hours = (deck.Nt + 1000) * s.dt / 3600.0
    nx, ny = deck.nx, deck.ny
    M = len(deck.tide_t)
    if s.inflow_cells:  # inflowLoc = jj*NX + ii - 1 for ii in [v27, v28), jj in [v29, v30)
        i0, i1, j0, j1 = s.inflow_cells
        inflow_vals = [(i1 - i0) * (j1 - j0), i0 + 1, i1 + 1, j0, j1]
    else:
        inflow_vals = [0, 1, 1, 0, 0]
    return [
        deck.start, "input/", "output/", "subdata/",
        s.dx, s.dx, nx, ny, s.dt, deck.NT_days, 0, out_hours,   # 4..11
        1, 1, 1, 1, 1, 0, 0,                                    # 12..18 save flags
        1,                                                      # 19 bcType: tide on YP
        nx, 0, M,                                               # 20..22 tideP: whole row
        1, 1, M,                                                # 23..25 tideM (unused)
        *inflow_vals, M,                                        # 26..31 inflow cells
        1 if s.wind_speed > 0 else 0, s.north_angle, M, M,      # 32..35 wind
        1, s.scalar_adv, 1, s.inflow_s, 1, 0.0, M, 1, 0.0, M,   # 36..45 scalar, tide S = 0
        0.0, 0.0, 0.0, 0.0, 0, 0 if deck.u0 is not None else 1, 1, 0,  # 46..53 IC files
        1, 0, s.dx / s.r, s.dx / s.r,                           # 54..57 subgrid
        deck.surfmax, deck.surfmin, deck.dsurf,                 # 58..60
        1, 0, 0.0, 3,                                           # 61..64 staggeredV, minA, beta, minV
        0, 1,                                                   # 65..66 no MPI
        9.81, 1e-4, 1e-4, 0, 0.01, 0.01, s.manning_n,           # 67..73
        s.use_thin_layer, 0.1, 1.0, 10.0, 1.25, 0.0013,         # 74..79
        1e-4, 1e-4, 1e-5, 1e-5, 0.5, 0.7, s.eps, s.max_iter,    # 80..87
    ]


DATA_DAT_LABELS = [
    "Model start date", "Input folder", "Output folder", "Subgrid folder",
    "dx(m)", "dy(m)", "NX", "NY", "dt(s)", "NT(days)", "If use cell edge",
    "Output interval(h)", "If save surface elevation", "If save u velocity",
    "If save v velocity", "If save depth", "If save scalar", "If save drag coefficient",
    "If save subgrid variables", "Type of boundary conditions", "Length of tideP boundary",
    "First cell of tideP boundary", "Size of tideP data", "Length of tideM boundary",
    "First cell of tideM boundary", "Size of tideM data", "Length of inflow boundary",
    "First i-index of inflow boundary", "Last i-index of inflow boundary",
    "First j-index of inflow boundary", "Last j-index of inflow boundary",
    "Size of inflow data", "If wind boundary condition exists", "North angle",
    "Size of wind speed data", "Size of wind direction data",
    "If scalar transport is modeled", "If scalar advection is modeled",
    "If inflow scalar is constant", "Inflow scalar", "If tideP scalar is constant",
    "TideP scalar", "Size of tideP scalar data", "If tideM scalar is constant",
    "TideM scalar", "Size of tideM scalar data", "Initial u velocity",
    "Initial v velocity", "Initial surface elevation", "Initial scalar concentration",
    "If initial u is constant", "If initial v is constant", "If initial surface is constant",
    "If initial scalar is constant", "If subgrid model is used", "The subgrid drag model used",
    "Subgrid dx", "Subgrid dy", "Max pre-defined surface elevation",
    "Min pre-defined surface elevation", "Increment of pre-defined surface",
    "If staggered volume is used", "If minimum face area is used",
    "Face area correction factor", "If effective volume is used", "If MPI is used",
    "Number of threads", "Gravity constant", "Eddy viscosity in x", "Eddy viscosity in y",
    "Use constant CD, not Manning's n", "Drag coefficient in x", "Drag coefficient in y",
    "Manning's n", "If thin-layer model is used", "Thin-layer thickness",
    "Max drag CD in the thin layer", "Wind decay rate in the thin layer", "Air density",
    "Wind drag coefficient", "Eddy diffusivity in x", "Eddy diffusivity in y",
    "Minimum depth allowed(m)", "Minimum waterfall depth(m)", "Low nonlinear cutoff",
    "High nonlinear cutoff", "Minimum CG residual", "Maximum CG iteration",
]


def write_reference_deck(deck: Deck, path: str, tables: np.ndarray | None = None,
                         binary_tables: bool = False, out_steps: int | None = None,
                         host=None) -> str:
    """Write data.dat + input/ for the reference model under ``path``.

    binary_tables additionally writes each subgrid table as raw little-endian
    doubles (``<name>.dat.bin``); the oracle harness reads those when present
    instead of parsing hundreds of millions of text values.  out_steps sets the
    output interval OutItvl in steps (default: beyond the last step).  host:
    the table builder when the deck carries no tables (see make_deck).
    """
    os.makedirs(os.path.join(path, "input", "subdata"), exist_ok=True)
    os.makedirs(os.path.join(path, "output"), exist_ok=True)
    out_hours = None
    if out_steps is not None:  # OutItvl = hours*3600/dt truncated (configuration.c:27)
        out_hours = (out_steps + 0.5) * deck.spec.dt / 3600.0
    vals = data_dat_values(deck, out_hours)
    with open(os.path.join(path, "data.dat"), "w") as f:
        f.write("# FrehdC input deck written by frehdc_b200.deck\n")
        for v, lab in zip(vals, DATA_DAT_LABELS):
            sv = v if isinstance(v, str) else (_fmt(v) if isinstance(v, float) else str(v))
            f.write("%-44s # %s\n" % (sv + ";", lab))
        f.write("# end\n")
    sub = os.path.join(path, "input", "subdata")
    _write_column(os.path.join(sub, "bottom.dat"), deck.bottom)
    _write_column(os.path.join(sub, "bottomXP.dat"), deck.bottomXP)
    _write_column(os.path.join(sub, "bottomYP.dat"), deck.bottomYP)
    if tables is None:
        tables = deck.extra.get("tables")
        if tables is None:
            tables = build_tables(deck, host)
    names = list(TABLE_NAMES)
    # useminV = 3 makes the reference load the minV* tables (subgrid.c:2186-2204)
    # without using them (subgrid.c:378,409); they repeat the half-cell volumes.
    extra = {"minVxp": 2, "minVxm": 3, "minVyp": 4, "minVym": 5}
    for k, name in enumerate(names):
        _write_table(os.path.join(sub, name + ".dat"), tables[k], binary_tables)
    for name, k in extra.items():
        _write_table(os.path.join(sub, name + ".dat"), tables[k], binary_tables)
    inp = os.path.join(path, "input")
    _write_column(os.path.join(inp, "surfic.dat"), deck.surf0)
    if deck.u0 is not None:
        _write_column(os.path.join(inp, "uuic.dat"), deck.u0)
    _write_column(os.path.join(inp, "scalaric.dat"), deck.S0)
    with open(os.path.join(inp, "tideP.dat"), "w") as f:
        for t, v in zip(deck.tide_t, deck.tide_v):
            f.write("%s,%s\n" % (_fmt(t), _fmt(v)))
    inflow = deck.inflow_v if deck.inflow_v is not None else np.zeros(len(deck.tide_t))
    with open(os.path.join(inp, "inflow.dat"), "w") as f:
        for t, v in zip(deck.tide_t, inflow):
            f.write("%s,%s\n" % (_fmt(t), _fmt(v)))
    if deck.wspd_v is not None:
        for name, vals in (("windspd.dat", deck.wspd_v), ("winddir.dat", deck.wdir_v)):
            with open(os.path.join(inp, name), "w") as f:
                for t, v in zip(deck.tide_t, vals):
                    f.write("%s,%s\n" % (_fmt(t), _fmt(v)))
    return path


def _write_table(path: str, tab: np.ndarray, binary: bool) -> None:
    tab = np.ascontiguousarray(tab, dtype="<f8").reshape(-1)
    if binary:
        tab.tofile(path + ".bin")
        # the text file must exist for the reference's fopen; keep it tiny
        with open(path, "w") as f:
            f.write("0\n")
    else:
        _write_column(path, tab)


def _tracer_fields(spec: DeckSpec, xcen, ycen, width: float, height: float) -> list:
    """Initial fields of the tracers: tracer t is S's plume moved a quarter of
    the basin from its centre, at angle 2 pi t / n_scalars, with peak
    scalar_peak * (1 - 0.2 t); all values stay inside [0, 100]."""
    out = []
    for t in range(1, spec.n_scalars):
        a = 2.0 * np.pi * t / spec.n_scalars
        cx, cy = 0.25 * width * np.cos(a), 0.25 * height * np.sin(a)
        peak = spec.scalar_peak * (1.0 - 0.2 * t)
        f = peak * np.exp(-((xcen - cx) ** 2 + (ycen - cy) ** 2) / (2.0 * spec.scalar_sigma ** 2))
        out.append(f.reshape(-1).copy())
    return out


def with_scalar(deck: Deck, S0: np.ndarray) -> Deck:
    """The same deck with S starting from another field: the reference run that a
    tracer with that initial field must reproduce."""
    return dataclasses.replace(deck, S0=np.asarray(S0, dtype=np.float64).copy(), tracers=[],
                               extra=dict(deck.extra))


def config_dict(deck: Deck) -> dict:
    """frehd_config fields of a deck, read back through the data.dat mapping."""
    from .config import config_from_values
    vals = data_dat_values(deck)
    # data.dat stores numbers as text; round-trip them the way the reference reads them
    txt = [v if isinstance(v, str) else (_fmt(v) if isinstance(v, float) else str(v)) for v in vals]
    from .config import _strtod
    parsed = txt[:4] + [_strtod(t) for t in txt[4:]]
    c = config_from_values(parsed, offset=deck.offset)
    c["nscalar"] = 1 + len(deck.tracers)
    return c

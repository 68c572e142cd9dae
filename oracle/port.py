"""ctypes wrapper of the C restatement oracle (oracle/frehd_oracle.c) and of
the deck pre-processing for runs of the reference program (oracle/deckprep.c).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__ (build/smoke) and
bench.py's cpu_baseline and reference legs.  build() compiles both with plain
gcc (no FMA contraction, IEEE doubles) into oracle/_build/libfrehd_oracle.so.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "libfrehd_oracle.so")
SRC = os.path.join(HERE, "frehd_oracle.c")
HDR = os.path.join(HERE, "frehd_oracle.h")
PREP = os.path.join(HERE, "deckprep.c")
# the pre-processor's formulas (one inline definition shared with the library)
LEVELS_DIR = os.path.join(os.path.dirname(HERE), "frehdc_b200", "csrc")
LEVELS = os.path.join(LEVELS_DIR, "subgrid_levels.h")

PRECOND_JACOBI, PRECOND_SSOR = 0, 1
X0_ZERO, X0_SURFACE = 0, 1

_lib = None


def build(force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    deps = (SRC, HDR, PREP, LEVELS)
    if force or not os.path.exists(LIB) or \
            max(os.path.getmtime(d) for d in deps) > os.path.getmtime(LIB):
        subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-fno-fast-math", "-ffp-contract=off",
                        "-fopenmp", "-I", LEVELS_DIR, "-o", LIB, SRC, PREP, "-lm"], check=True)
    return LIB


_dp = C.POINTER(C.c_double)


class OracleCfg(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("dt", C.c_double),
        ("g", C.c_double), ("NUx", C.c_double), ("NUy", C.c_double),
        ("Kx", C.c_double), ("Ky", C.c_double),
        ("CDx", C.c_double), ("CDy", C.c_double), ("manningN", C.c_double),
        ("CDmax", C.c_double), ("hD", C.c_double), ("CwT", C.c_double),
        ("CDnotN", C.c_int), ("useThinLayer", C.c_int),
        ("useSubgrid", C.c_int), ("useSubDrag", C.c_int), ("staggeredV", C.c_int),
        ("useminA", C.c_int), ("useminV", C.c_int),
        ("dxf", C.c_double), ("dyf", C.c_double), ("subR", C.c_double),
        ("surfmin", C.c_double), ("surfmax", C.c_double), ("dsurf", C.c_double),
        ("bcType", C.c_int), ("tideLocFirstP", C.c_int), ("tideLocLengthP", C.c_int),
        ("useScalar", C.c_int), ("scalarAdv", C.c_int), ("useConstTidePS", C.c_int),
        ("tidePS", C.c_double),
        ("useWind", C.c_int), ("useEvap", C.c_int), ("useRain", C.c_int),
        ("inflowLocLength", C.c_int), ("useSubStep", C.c_int), ("checkConservation", C.c_int),
        ("minDepth", C.c_double), ("wtfh", C.c_double), ("CFLl", C.c_double),
        ("CFLh", C.c_double), ("eps", C.c_double), ("maxIter", C.c_int),
        ("offset", C.c_double),
        ("inflowI0", C.c_int), ("inflowI1", C.c_int), ("inflowJ0", C.c_int), ("inflowJ1", C.c_int),
        ("inflowS", C.c_double), ("northAngle", C.c_double), ("rhoa", C.c_double),
        ("Cw", C.c_double),
    ]


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        L.oracle_create.restype = C.c_void_p
        L.oracle_create.argtypes = [C.POINTER(OracleCfg), C.c_char_p, C.c_int]
        L.oracle_destroy.argtypes = [C.c_void_p]
        L.oracle_error.restype = C.c_char_p
        L.oracle_error.argtypes = [C.c_void_p]
        L.oracle_set_tables.argtypes = [C.c_void_p, C.c_int, _dp]
        L.oracle_set_tide.argtypes = [C.c_void_p, C.c_int, _dp]
        L.oracle_set_series.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp]
        L.oracle_set_solver.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.oracle_init.argtypes = [C.c_void_p] + [_dp] * 7 + [C.c_int]
        L.oracle_explicit.argtypes = [C.c_void_p, C.c_int]
        L.oracle_solve.argtypes = [C.c_void_p]
        L.oracle_update.argtypes = [C.c_void_p, C.c_int, _dp]
        L.oracle_update.restype = C.c_double
        L.oracle_step.argtypes = [C.c_void_p, C.c_int]
        L.oracle_step.restype = C.c_double
        L.oracle_last_iters.argtypes = [C.c_void_p]
        L.oracle_last_accuracy.argtypes = [C.c_void_p]
        L.oracle_last_accuracy.restype = C.c_double
        L.oracle_field_len.argtypes = [C.c_void_p, C.c_char_p]
        L.oracle_field_len.restype = C.c_long
        L.oracle_get.argtypes = [C.c_void_p, C.c_char_p, _dp, C.c_long]
        L.oracle_set.argtypes = [C.c_void_p, C.c_char_p, _dp, C.c_long]
        L.oracle_build_tables.argtypes = [_dp, C.c_long, C.c_int, C.c_int, C.c_int, C.c_double,
                                          C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                          _dp]
        L.oracle_build_bottoms.argtypes = [_dp, C.c_long, C.c_int, C.c_int, C.c_int, _dp, _dp,
                                           _dp]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(_dp)


# ---- deck pre-processing (the same interface as frehdc_b200.native's builders)
def build_tables(zf: np.ndarray, nx: int, ny: int, r: int, dxf: float, dyf: float,
                 surfmin: float, dsurf: float, Ne: int, block_check: bool = False) -> np.ndarray:
    """(10, Ne, N) subgrid tables of fine bottoms zf ((ny*r, nx*r))."""
    zf = np.ascontiguousarray(zf, dtype=np.float64)
    out = np.empty((10, Ne, nx * ny), dtype=np.float64)
    rc = lib().oracle_build_tables(_p(zf), zf.shape[1], nx, ny, r, dxf, dyf, surfmin, dsurf, Ne,
                                   int(bool(block_check)), _p(out))
    if rc:
        raise ValueError(f"oracle_build_tables: bad arguments ({rc})")
    return out


def build_bottoms(zf: np.ndarray, nx: int, ny: int, r: int):
    """Coarse bottom, bottomXP and bottomYP (N doubles each) of fine bottoms zf."""
    zf = np.ascontiguousarray(zf, dtype=np.float64)
    N = nx * ny
    b, bx, by = np.empty(N), np.empty(N), np.empty(N)
    if lib().oracle_build_bottoms(_p(zf), zf.shape[1], nx, ny, r, _p(b), _p(bx), _p(by)):
        raise ValueError("oracle_build_bottoms: bad arguments")
    return b, bx, by


class Oracle:
    """One domain of the restatement oracle."""

    def __init__(self, cfg: dict, tables: np.ndarray, tideP: np.ndarray,
                 precond: int = PRECOND_SSOR, x0: int = X0_ZERO):
        L = lib()
        c = OracleCfg()
        for name, _ in OracleCfg._fields_:
            setattr(c, name, cfg[name])
        err = C.create_string_buffer(256)
        h = L.oracle_create(C.byref(c), err, 256)
        if not h:
            raise RuntimeError("oracle_create: " + err.value.decode())
        self.h = h
        self.cfg = dict(cfg)
        self.nx, self.ny = cfg["nx"], cfg["ny"]
        tables = np.ascontiguousarray(tables, dtype=np.float64)
        self.Ne = tables.shape[1]
        self._chk(L.oracle_set_tables(h, self.Ne, _p(tables)))
        tideP = np.ascontiguousarray(tideP, dtype=np.float64)
        self._chk(L.oracle_set_tide(h, len(tideP), _p(tideP)))
        L.oracle_set_solver(h, precond, x0)

    def set_series(self, kind: str, values: np.ndarray) -> None:
        """bc->inflow / windspd / winddir by step."""
        v = np.ascontiguousarray(values, dtype=np.float64)
        k = {"inflow": 1, "windspd": 2, "winddir": 3}[kind]
        self._chk(lib().oracle_set_series(self.h, k, len(v), _p(v)))

    def _chk(self, rc):
        if rc != 0:
            raise RuntimeError("oracle: " + lib().oracle_error(self.h).decode())

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_destroy(self.h)
            self.h = None

    def init(self, bottom, bottomXP, bottomYP, surf0, u0=None, v0=None, S0=None,
             round_trip_output=True):
        N = self.nx * self.ny
        z = np.zeros(N)
        arrs = [np.ascontiguousarray(a if a is not None else z, dtype=np.float64)
                for a in (bottom, bottomXP, bottomYP, surf0, u0, v0, S0)]
        self._chk(lib().oracle_init(self.h, *[_p(a) for a in arrs], int(round_trip_output)))

    def get(self, name: str) -> np.ndarray:
        n = lib().oracle_field_len(self.h, name.encode())
        if n < 0:
            raise KeyError(name)
        out = np.empty(n)
        self._chk(lib().oracle_get(self.h, name.encode(), _p(out), n))
        return out

    def set(self, name: str, a: np.ndarray) -> None:
        a = np.ascontiguousarray(a, dtype=np.float64)
        self._chk(lib().oracle_set(self.h, name.encode(), _p(a), a.size))

    def explicit(self, tt: int) -> None:
        lib().oracle_explicit(self.h, tt)

    def solve(self) -> None:
        lib().oracle_solve(self.h)

    def update(self, tt: int, x: np.ndarray | None = None) -> float:
        if x is None:
            x = self.get("x")
        x = np.ascontiguousarray(x, dtype=np.float64)
        return lib().oracle_update(self.h, tt, _p(x))

    def step(self, tt: int) -> float:
        return lib().oracle_step(self.h, tt)

    @property
    def last_iters(self) -> int:
        return lib().oracle_last_iters(self.h)

    @property
    def last_accuracy(self) -> float:
        return lib().oracle_last_accuracy(self.h)


def from_deck(deck, precond: int = PRECOND_SSOR, x0: int = X0_ZERO) -> Oracle:
    """Oracle domain initialised from a generated deck (frehdc_b200.deck)."""
    from frehdc_b200 import deck as D
    cfg = D.config_dict(deck)
    tables = deck.extra.get("tables")
    if tables is None:
        tables = D.build_tables(deck)
        deck.extra["tables"] = tables
    o = Oracle(cfg, tables, D.tide_series(deck), precond=precond, x0=x0)
    for kind, series in D.forcing_series(deck).items():
        o.set_series(kind, series)
    o.init(deck.bottom, deck.bottomXP, deck.bottomYP, deck.surf0, deck.u0, None, deck.S0)
    return o

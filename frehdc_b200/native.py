"""ctypes binding of the C ABI in include/frehd_b200.h.

The library is loaded from the package directory (libfrehd_b200.so, built in
tree by frehdc_b200.build).  There is no fallback: if the library is missing or
a call fails, a FrehdError is raised.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfrehd_b200.so")

_lib = None


class FrehdError(RuntimeError):
    def __init__(self, status: int, where: str, message: str):
        super().__init__(f"{where}: {message} (status {status})")
        self.status = status


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FrehdError(-1, "load", f"{LIB_PATH} is not built; run frehdc_b200.build")
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class Config(C.Structure):
    """Mirror of frehd_config (include/frehd_b200.h)."""
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
    ]


STATE_FIELDS = [
    "surf", "uuXP", "vvYP", "S", "depth", "CDXP", "CDYP", "CFLx", "CFLy",
    "V", "Z", "Nx", "Oy", "Vx", "Vy", "Zx", "Zy", "ind",
    "bottomZ", "bottomXP", "bottomYP",
    "surfOld", "uuYP", "vvXP", "EnXP", "EnYP", "cellV", "Sm", "Fuu", "Fvv",
]
# arrays carrying the ghost ring (N2ct) vs interior only (N)
STATE_N = {"depth", "uuYP", "vvXP", "EnXP", "EnYP", "cellV", "Sm"}


class State(C.Structure):
    _fields_ = [(n, _ip if n == "ind" else _dp) for n in STATE_FIELDS]


class StepStats(C.Structure):
    _fields_ = [
        ("step", C.c_int), ("cg_iters", C.c_int), ("status", C.c_int),
        ("cg_rel_residual", C.c_double), ("max_cflx", C.c_double), ("max_cfly", C.c_double),
        ("n_cfl_warn", C.c_int), ("volume", C.c_double),
    ]


def _declare(L: C.CDLL) -> None:
    L.frehd_status_string.restype = C.c_char_p
    L.frehd_last_error.restype = C.c_char_p
    L.frehd_version.restype = C.c_char_p
    L.frehd_build_tables.argtypes = [_dp, C.c_long, C.c_int, C.c_int, C.c_int, C.c_double,
                                     C.c_double, C.c_double, C.c_double, C.c_int, _dp]
    L.frehd_build_bottoms.argtypes = [_dp, C.c_long, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp]
    L.frehd_config_defaults.argtypes = [C.POINTER(Config)]
    L.frehd_config_defaults.restype = None


def check(status: int, where: str) -> None:
    if status != 0:
        L = lib()
        msg = L.frehd_last_error().decode() or L.frehd_status_string(status).decode()
        raise FrehdError(status, where, msg)


def as_dp(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def build_tables(zf: np.ndarray, nx: int, ny: int, r: int, dxf: float, dyf: float,
                 surfmin: float, dsurf: float, Ne: int) -> np.ndarray:
    zf = np.ascontiguousarray(zf, dtype=np.float64)
    out = np.empty((10, Ne, nx * ny), dtype=np.float64)
    check(lib().frehd_build_tables(as_dp(zf), zf.shape[1], nx, ny, r, dxf, dyf, surfmin, dsurf,
                                   Ne, as_dp(out)), "frehd_build_tables")
    return out


def build_bottoms(zf: np.ndarray, nx: int, ny: int, r: int):
    zf = np.ascontiguousarray(zf, dtype=np.float64)
    N = nx * ny
    b = np.empty(N)
    bx = np.empty(N)
    by = np.empty(N)
    check(lib().frehd_build_bottoms(as_dp(zf), zf.shape[1], nx, ny, r, as_dp(b), as_dp(bx),
                                    as_dp(by)), "frehd_build_bottoms")
    return b, bx, by

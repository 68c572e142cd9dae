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
# the in-tree build; FREHD_B200_LIB names another build of the same library
LIB_PATH = os.environ.get("FREHD_B200_LIB") or os.path.join(HERE, "libfrehd_b200.so")

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
        ("inflowI0", C.c_int), ("inflowI1", C.c_int), ("inflowJ0", C.c_int), ("inflowJ1", C.c_int),
        ("inflowS", C.c_double), ("northAngle", C.c_double), ("rhoa", C.c_double),
        ("Cw", C.c_double), ("nscalar", C.c_int),
    ]


STATE_FIELDS = [
    "surf", "uuXP", "vvYP", "S", "depth", "CDXP", "CDYP", "CFLx", "CFLy",
    "V", "Z", "Nx", "Oy", "Vx", "Vy", "Zx", "Zy", "ind",
    "bottomZ", "bottomXP", "bottomYP",
    "surfOld", "uuYP", "vvXP", "EnXP", "EnYP", "cellV", "Sm", "Fuu", "Fvv",
    "depthXP", "depthYP",   # held only with useWind = 1
]
WIND_FIELDS = ("depthXP", "depthYP")
# arrays carrying the ghost ring (N2ct) vs interior only (N)
STATE_N = {"depth", "uuYP", "vvXP", "cellV", "Sm"}


class State(C.Structure):
    _fields_ = [(n, _ip if n == "ind" else _dp) for n in STATE_FIELDS]


class StepStats(C.Structure):
    _fields_ = [
        ("step", C.c_int), ("cg_iters", C.c_int), ("status", C.c_int),
        ("cg_rel_residual", C.c_double), ("max_cflx", C.c_double), ("max_cfly", C.c_double),
        ("n_cfl_warn", C.c_int), ("volume", C.c_double), ("cg_fallback", C.c_int),
        ("cg_noconverge", C.c_int),
    ]


def _declare(L: C.CDLL) -> None:
    L.frehd_status_string.restype = C.c_char_p
    L.frehd_last_error.restype = C.c_char_p
    L.frehd_version.restype = C.c_char_p
    L.frehd_build_tables.argtypes = [_dp, C.c_long, C.c_int, C.c_int, C.c_int, C.c_double,
                                     C.c_double, C.c_double, C.c_double, C.c_int, _dp]
    L.frehd_build_tables_ex.argtypes = [_dp, C.c_long, C.c_int, C.c_int, C.c_int, C.c_double,
                                        C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, _dp]
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


GEOM_BLOCK_CHECK = 1


def build_tables(zf: np.ndarray, nx: int, ny: int, r: int, dxf: float, dyf: float,
                 surfmin: float, dsurf: float, Ne: int, block_check: bool = False) -> np.ndarray:
    zf = np.ascontiguousarray(zf, dtype=np.float64)
    out = np.empty((10, Ne, nx * ny), dtype=np.float64)
    check(lib().frehd_build_tables_ex(as_dp(zf), zf.shape[1], nx, ny, r, dxf, dyf, surfmin, dsurf,
                                      Ne, GEOM_BLOCK_CHECK if block_check else 0, as_dp(out)),
          "frehd_build_tables")
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


_vp = C.c_void_p

PHASE_EXPLICIT, PHASE_SOLVE, PHASE_UPDATE = 1, 2, 3
X0_ZERO, X0_SURFACE = 0, 1
CG_SINGLE_SWEEP, CG_TWO_PHASE = 0, 1
DECOUPLED_AS_ASSEMBLED, DECOUPLED_ELIMINATED = 0, 1
PRECISION_FP64, PRECISION_MIXED = 0, 1
SERIES_TIDE, SERIES_INFLOW, SERIES_WIND_SPEED, SERIES_WIND_DIR = 0, 1, 2, 3
BATCH_TILE_LIST, BATCH_CTA_GROUPS = 0, 1
STATUS = {0: "ok", 1: "invalid", 2: "unsupported", 3: "cuda", 4: "nomem", 5: "cg_noconverge",
          6: "cfl", 7: "timeout", 8: "state"}


class KernelTimes(C.Structure):
    _fields_ = [("explicit_ms", C.c_double), ("cg_ms", C.c_double), ("update_geo_ms", C.c_double),
                ("update_vel_ms", C.c_double), ("finish_ms", C.c_double), ("steps", C.c_int),
                ("cg_iters", C.c_longlong)]


def _declare_domain(L: C.CDLL) -> None:
    L.frehd_domain_set_profiling.argtypes = [_vp, C.c_int]
    L.frehd_domain_kernel_times.argtypes = [_vp, C.POINTER(KernelTimes)]
    L.frehd_domain_stream.argtypes = [_vp, C.POINTER(_vp)]
    L.frehd_domain_create.argtypes = [C.POINTER(Config), C.c_int, C.POINTER(_vp)]
    L.frehd_domain_destroy.argtypes = [_vp]
    L.frehd_domain_set_tables.argtypes = [_vp, C.c_int, _dp]
    L.frehd_domain_set_fine_bottoms.argtypes = [_vp, C.c_int, _dp, C.c_long]
    L.frehd_domain_set_fine_bottoms_ex.argtypes = [_vp, C.c_int, _dp, C.c_long, C.c_int]
    L.frehd_domain_set_tide.argtypes = [_vp, C.c_int, _dp]
    L.frehd_domain_set_series.argtypes = [_vp, C.c_int, C.c_int, _dp]
    L.frehd_domain_update_series.argtypes = [_vp, C.c_int, C.c_int, C.c_int, _vp]
    L.frehd_domain_set_solver.argtypes = [_vp, C.c_int]
    L.frehd_domain_set_cg_schedule.argtypes = [_vp, C.c_int]
    L.frehd_domain_set_decoupled.argtypes = [_vp, C.c_int]
    L.frehd_domain_set_precision.argtypes = [_vp, C.c_int, C.c_double]
    L.frehd_domain_upload_state.argtypes = [_vp, C.POINTER(State)]
    L.frehd_domain_download_state.argtypes = [_vp, C.POINTER(State)]
    L.frehd_domain_init.argtypes = [_vp] + [_dp] * 7 + [C.c_int]
    L.frehd_domain_upload_scalar.argtypes = [_vp, C.c_int, _dp]
    L.frehd_domain_download_scalar.argtypes = [_vp, C.c_int, _dp]
    L.frehd_domain_init_scalar.argtypes = [_vp, C.c_int, _dp]
    L.frehd_domain_step.argtypes = [_vp, C.c_int]
    L.frehd_domain_run.argtypes = [_vp, C.c_int, C.c_int]
    L.frehd_domain_set_wait_test.argtypes = [_vp, C.c_longlong, C.c_int]
    L.frehd_domain_phase.argtypes = [_vp, C.c_int, C.c_int, _dp]
    L.frehd_domain_download_system.argtypes = [_vp] + [_dp] * 6
    L.frehd_domain_download_solution.argtypes = [_vp, _dp]
    L.frehd_domain_stats.argtypes = [_vp, C.POINTER(StepStats)]
    L.frehd_domain_sync.argtypes = [_vp]
    L.frehd_device_count.argtypes = [_ip]
    L.frehd_domain_write_output.argtypes = [_vp, C.c_char_p, C.c_int, C.c_int]
    L.frehd_domain_write_restart.argtypes = [_vp, C.c_char_p, C.c_int, C.c_double]
    L.frehd_format_fixed4.argtypes = [_dp, C.c_long, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]
    L.frehd_cg_solve_noalloc.argtypes = [C.c_int, C.c_int] + [_vp] * 5 + \
        [C.c_double, C.c_int, C.c_int, _vp, _ip, C.POINTER(C.c_double)]


OUT_SURFACE, OUT_U, OUT_V, OUT_DEPTH, OUT_CD, OUT_SCALAR, OUT_SUB = 1, 2, 4, 8, 16, 32, 64


def format_fixed4(values) -> bytes:
    """The reference's "%4.4f \n" lines of the values, formatted on the GPU."""
    L = lib()
    if not hasattr(L, "_domain_declared"):
        _declare_domain(L)
        L._domain_declared = True
    v = np.ascontiguousarray(values, dtype=np.float64)
    n = C.c_size_t(0)
    check(L.frehd_format_fixed4(as_dp(v), v.size, None, 0, C.byref(n)), "format_fixed4")
    buf = C.create_string_buffer(n.value + 1)
    check(L.frehd_format_fixed4(as_dp(v), v.size, buf, n.value, C.byref(n)), "format_fixed4")
    return buf.raw[:n.value]


def device_count() -> int:
    n = C.c_int(0)
    lib().frehd_device_count(C.byref(n))
    return n.value


class Domain:
    """One domain resident on a GPU, driven through the C ABI."""

    def __init__(self, cfg: dict, device: int = 0):
        L = lib()
        if not hasattr(L, "_domain_declared"):
            _declare_domain(L)
            L._domain_declared = True
        c = Config()
        from .config import fill_struct
        fill_struct(c, cfg)
        h = _vp()
        check(L.frehd_domain_create(C.byref(c), device, C.byref(h)), "frehd_domain_create")
        self.h = h
        self.cfg = dict(cfg)
        self.nx, self.ny = cfg["nx"], cfg["ny"]
        self.N = self.nx * self.ny
        self.T = (self.nx + 2) * (self.ny + 2)
        self._keep = []

    def close(self):
        if getattr(self, "h", None):
            lib().frehd_domain_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # geometry / forcing
    def set_tables(self, tables: np.ndarray):
        t = np.ascontiguousarray(tables, dtype=np.float64)
        check(lib().frehd_domain_set_tables(self.h, t.shape[1], as_dp(t)), "set_tables")

    def set_fine_bottoms(self, zf: np.ndarray, r: int, block_check: bool = False):
        z = np.ascontiguousarray(zf, dtype=np.float64)
        check(lib().frehd_domain_set_fine_bottoms_ex(self.h, r, as_dp(z), z.shape[1],
                                                     GEOM_BLOCK_CHECK if block_check else 0),
              "set_fine_bottoms")

    def set_tide(self, tideP: np.ndarray):
        t = np.ascontiguousarray(tideP, dtype=np.float64)
        check(lib().frehd_domain_set_tide(self.h, len(t), as_dp(t)), "set_tide")

    def update_series(self, kind: int, t0: int, n: int, ptr: int):
        """Overwrite entries t0..t0+n-1 of a series from host memory at address
        ptr (queued on the domain's stream; from pinned memory the values must
        stay untouched until the next synchronisation)."""
        check(lib().frehd_domain_update_series(self.h, kind, t0, n, C.c_void_p(ptr)),
              "update_series")

    def set_series(self, kind: int, values: np.ndarray):
        """bc->inflow / windspd / winddir by step (SERIES_*)."""
        v = np.ascontiguousarray(values, dtype=np.float64)
        check(lib().frehd_domain_set_series(self.h, kind, len(v), as_dp(v)), "set_series")

    def set_solver(self, x0: int):
        check(lib().frehd_domain_set_solver(self.h, x0), "set_solver")

    def set_cg_schedule(self, schedule: int):
        check(lib().frehd_domain_set_cg_schedule(self.h, schedule), "set_cg_schedule")

    def set_decoupled(self, mode: int):
        check(lib().frehd_domain_set_decoupled(self.h, mode), "set_decoupled")

    def set_precision(self, mode: int, eps_inner: float = 1e-5):
        check(lib().frehd_domain_set_precision(self.h, mode, eps_inner), "set_precision")

    def init(self, bottom, bottomXP, bottomYP, surf0, u0=None, v0=None, S0=None,
             round_trip_output: bool = True):
        z = np.zeros(self.N)
        arrs = [np.ascontiguousarray(a if a is not None else z, dtype=np.float64)
                for a in (bottom, bottomXP, bottomYP, surf0, u0, v0, S0)]
        check(lib().frehd_domain_init(self.h, *[as_dp(a) for a in arrs], int(round_trip_output)),
              "init")

    def init_scalar(self, s: int, S0=None):
        """Init's setup of scalar s (a tracer for s >= 1) from its initial field (N values)."""
        a = None if S0 is None else np.ascontiguousarray(S0, dtype=np.float64)
        assert a is None or a.size == self.N
        check(lib().frehd_domain_init_scalar(self.h, s, None if a is None else as_dp(a)),
              "init_scalar")

    def upload_scalar(self, s: int, values: np.ndarray):
        a = np.ascontiguousarray(values, dtype=np.float64)
        assert a.size == self.T
        check(lib().frehd_domain_upload_scalar(self.h, s, as_dp(a)), "upload_scalar")

    def download_scalar(self, s: int) -> np.ndarray:
        a = np.empty(self.T)
        check(lib().frehd_domain_download_scalar(self.h, s, as_dp(a)), "download_scalar")
        return a

    # state
    def _len(self, name: str) -> int:
        return self.N if name in STATE_N else self.T

    def upload(self, arrays: dict):
        st = State()
        keep = []
        for name, a in arrays.items():
            if name not in STATE_FIELDS:
                continue
            if name == "ind":
                b = np.ascontiguousarray(a, dtype=np.int32)
                assert b.size == self.T
                setattr(st, name, b.ctypes.data_as(_ip))
            else:
                b = np.ascontiguousarray(a, dtype=np.float64)
                assert b.size == self._len(name), (name, b.size)
                setattr(st, name, as_dp(b))
            keep.append(b)
        check(lib().frehd_domain_upload_state(self.h, C.byref(st)), "upload_state")

    def download(self, names=None) -> dict:
        names = [n for n in STATE_FIELDS if n not in WIND_FIELDS] if names is None else names
        st = State()
        out = {}
        for name in names:
            if name == "ind":
                a = np.empty(self.T, dtype=np.int32)
                setattr(st, name, a.ctypes.data_as(_ip))
            else:
                a = np.empty(self._len(name))
                setattr(st, name, as_dp(a))
            out[name] = a
        check(lib().frehd_domain_download_state(self.h, C.byref(st)), "download_state")
        return out

    def system(self) -> dict:
        names = ["GnCt", "GnXP", "GnXM", "GnYP", "GnYM", "z"]
        arrs = {n: np.empty(self.N) for n in names}
        check(lib().frehd_domain_download_system(self.h, *[as_dp(arrs[n]) for n in names]),
              "download_system")
        return arrs

    def solution(self) -> np.ndarray:
        x = np.empty(self.N)
        check(lib().frehd_domain_download_solution(self.h, as_dp(x)), "download_solution")
        return x

    # stepping
    def phase(self, phase: int, tt: int, x_ext: np.ndarray | None = None) -> int:
        if x_ext is not None:
            x = np.ascontiguousarray(x_ext, dtype=np.float64)
            rc = lib().frehd_domain_phase(self.h, phase, tt, as_dp(x))
        else:
            rc = lib().frehd_domain_phase(self.h, phase, tt, None)
        if rc not in (0, 6):
            check(rc, "phase")
        return rc

    # statuses a step returns without raising: FREHD_OK, FREHD_ERR_CG_NOCONVERGE
    # (a warning: the solve stopped at maxIter) and FREHD_ERR_CFL (the reference
    # stops there)
    STEP_STATUSES = (0, 5, 6)

    def step(self, tt: int) -> int:
        rc = lib().frehd_domain_step(self.h, tt)
        if rc not in self.STEP_STATUSES:
            check(rc, "step")
        return rc

    def run(self, t0: int, nsteps: int) -> int:
        rc = lib().frehd_domain_run(self.h, t0, nsteps)
        if rc not in self.STEP_STATUSES:
            check(rc, "run")
        return rc

    def set_wait_test(self, wait_limit_ns: int, skip_barrier_rank: int = -1):
        """Failure-path testing (frehd_domain_set_wait_test): bounded grid-barrier
        waits of wait_limit_ns, and one CTA that skips the next solve's first
        barrier so that the others' wait runs out."""
        check(lib().frehd_domain_set_wait_test(self.h, int(wait_limit_ns), int(skip_barrier_rank)),
              "frehd_domain_set_wait_test")

    def stats(self) -> dict:
        s = StepStats()
        check(lib().frehd_domain_stats(self.h, C.byref(s)), "stats")
        return {n: getattr(s, n) for n, _ in StepStats._fields_}

    def sync(self):
        check(lib().frehd_domain_sync(self.h), "sync")

    def write_output(self, prefix: str, tt: int, fields: int):
        """DataOutput/SubOutput files of the current state (OUT_* flags)."""
        check(lib().frehd_domain_write_output(self.h, prefix.encode(), tt, fields), "write_output")

    def write_restart(self, prefix: str, tt: int, tNEnd: float):
        check(lib().frehd_domain_write_restart(self.h, prefix.encode(), tt, tNEnd), "write_restart")

    def set_profiling(self, on: bool):
        check(lib().frehd_domain_set_profiling(self.h, int(on)), "set_profiling")

    def kernel_times(self) -> dict:
        t = KernelTimes()
        check(lib().frehd_domain_kernel_times(self.h, C.byref(t)), "kernel_times")
        return {n: getattr(t, n) for n, _ in KernelTimes._fields_}

    def stream(self) -> int:
        s = _vp()
        check(lib().frehd_domain_stream(self.h, C.byref(s)), "stream")
        return s.value or 0


class BatchInfo(C.Structure):
    _fields_ = [("domains", C.c_int), ("cg_ctas", C.c_int), ("cg_capacity", C.c_int),
                ("tiles", C.c_long), ("graph", C.c_int), ("bytes_used", C.c_longlong),
                ("bytes_budget", C.c_longlong), ("steps", C.c_longlong)]


def _declare_batch(L: C.CDLL) -> None:
    if hasattr(L, "_batch_declared"):
        return
    if not hasattr(L, "_domain_declared"):
        _declare_domain(L)
        L._domain_declared = True
    L.frehd_domain_footprint.argtypes = [C.POINTER(Config), C.c_int, C.POINTER(C.c_longlong)]
    L.frehd_batch_create.argtypes = [C.c_int, C.c_longlong, C.c_double, C.POINTER(_vp)]
    L.frehd_batch_destroy.argtypes = [_vp]
    L.frehd_batch_admit.argtypes = [_vp, _vp, C.c_int, _ip]
    L.frehd_batch_release.argtypes = [_vp, C.c_int, C.POINTER(_vp)]
    L.frehd_batch_step.argtypes = [_vp]
    L.frehd_batch_sync.argtypes = [_vp]
    L.frehd_batch_info.argtypes = [_vp, C.POINTER(BatchInfo)]
    L.frehd_batch_stream.argtypes = [_vp, C.POINTER(_vp)]
    L.frehd_batch_set_graph.argtypes = [_vp, C.c_int]
    L.frehd_batch_set_cg_packing.argtypes = [_vp, C.c_int]
    L.frehd_batch_set_stencil_tiles.argtypes = [_vp, C.c_int]
    L.frehd_server_create.argtypes = [C.c_int, C.c_longlong, C.c_double, C.POINTER(_vp)]
    L.frehd_server_submit.argtypes = [_vp, _vp, C.c_int, C.c_int, C.POINTER(C.c_longlong)]
    L.frehd_server_poll.argtypes = [_vp, C.POINTER(ServerDone), C.c_int, C.c_int, _ip]
    L.frehd_server_info.argtypes = [_vp, C.POINTER(ServerInfo)]
    L.frehd_server_destroy.argtypes = [_vp]
    L._batch_declared = True


class ServerDone(C.Structure):
    """Mirror of frehd_server_done."""
    _fields_ = [("ticket", C.c_longlong), ("domain", _vp), ("status", C.c_int), ("steps", C.c_int),
                ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double)]


class ServerInfo(C.Structure):
    """Mirror of frehd_server_info_t."""
    _fields_ = [("submitted", C.c_longlong), ("completed", C.c_longlong), ("waiting", C.c_int),
                ("active", C.c_int), ("max_active", C.c_int), ("batch_steps", C.c_longlong),
                ("cell_steps", C.c_longlong), ("clock", C.c_double), ("status", C.c_int)]


def footprint(cfg: dict, r: int) -> int:
    """Device bytes one domain of this configuration holds (frehd_domain_footprint)."""
    L = lib()
    _declare_batch(L)
    from .config import fill_struct
    c = Config()
    fill_struct(c, cfg)
    out = C.c_longlong(0)
    check(L.frehd_domain_footprint(C.byref(c), r, C.byref(out)), "frehd_domain_footprint")
    return out.value


class Batch:
    """Many resident domains stepped together (frehd_batch_*): each admitted
    Domain advances one step per step() call; release() hands it back."""

    def __init__(self, budget_bytes: int, cells_per_cta: float, device: int = 0):
        L = lib()
        _declare_batch(L)
        h = _vp()
        check(L.frehd_batch_create(device, int(budget_bytes), float(cells_per_cta), C.byref(h)),
              "frehd_batch_create")
        self.h = h
        self.members: dict[int, "Domain"] = {}

    def admit(self, dom: "Domain", t0: int = 1) -> int:
        slot = C.c_int(-1)
        check(lib().frehd_batch_admit(self.h, dom.h, t0, C.byref(slot)), "frehd_batch_admit")
        self.members[slot.value] = dom
        return slot.value

    def try_admit(self, dom: "Domain", t0: int = 1):
        """The slot, or None when the budget or the CTA capacity is exhausted."""
        try:
            return self.admit(dom, t0)
        except FrehdError as e:
            if e.status == 4:
                return None
            raise

    def release(self, slot: int) -> "Domain":
        out = _vp()
        check(lib().frehd_batch_release(self.h, slot, C.byref(out)), "frehd_batch_release")
        return self.members.pop(slot)

    def step(self):
        check(lib().frehd_batch_step(self.h), "frehd_batch_step")

    def sync(self):
        check(lib().frehd_batch_sync(self.h), "frehd_batch_sync")

    def info(self) -> dict:
        i = BatchInfo()
        check(lib().frehd_batch_info(self.h, C.byref(i)), "frehd_batch_info")
        return {n: getattr(i, n) for n, _ in BatchInfo._fields_}

    @staticmethod
    def capacity(device: int = 0) -> int:
        """Co-resident CTAs of the batched CG on this device."""
        b = Batch(1 << 20, 1.0, device)
        try:
            return int(b.info()["cg_capacity"])
        finally:
            b.close()

    def stream(self) -> int:
        s = _vp()
        check(lib().frehd_batch_stream(self.h, C.byref(s)), "frehd_batch_stream")
        return s.value or 0

    def set_graph(self, on: bool):
        check(lib().frehd_batch_set_graph(self.h, int(on)), "frehd_batch_set_graph")

    def set_cg_packing(self, packing: int):
        """BATCH_CTA_GROUPS (default) or BATCH_TILE_LIST (frehd_batch_set_cg_packing)."""
        check(lib().frehd_batch_set_cg_packing(self.h, int(packing)), "frehd_batch_set_cg_packing")

    def set_stencil_tiles(self, tiles_per_block: int):
        """32 x 8 stencil tiles per block of the batched stencil kernels, 1..8
        (frehd_batch_set_stencil_tiles)."""
        check(lib().frehd_batch_set_stencil_tiles(self.h, int(tiles_per_block)),
              "frehd_batch_set_stencil_tiles")

    def close(self):
        if getattr(self, "h", None):
            lib().frehd_batch_destroy(self.h)
            self.h = None
            self.members.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """frehd_server_*: a native continuous-batching loop on its own host thread.
    Submitted domains stay owned by the caller (and by this object's table
    until polled back)."""

    def __init__(self, budget_bytes: int, cells_per_cta: float, device: int = 0):
        L = lib()
        _declare_batch(L)
        h = _vp()
        check(L.frehd_server_create(device, int(budget_bytes), float(cells_per_cta), C.byref(h)),
              "frehd_server_create")
        self.h = h
        self.held: dict[int, "Domain"] = {}

    def submit(self, dom: "Domain", nsteps: int, t0: int = 1) -> int:
        t = C.c_longlong()
        check(lib().frehd_server_submit(self.h, dom.h, t0, nsteps, C.byref(t)), "frehd_server_submit")
        self.held[t.value] = dom
        return t.value

    def poll(self, timeout_ms: int = 0, cap: int = 64) -> list:
        """Completed requests: dicts with ticket, domain (the Domain object),
        status, steps and the server-clock times."""
        arr = (ServerDone * cap)()
        n = C.c_int()
        check(lib().frehd_server_poll(self.h, arr, cap, int(timeout_ms), C.byref(n)),
              "frehd_server_poll")
        out = []
        for k in range(n.value):
            r = {f: getattr(arr[k], f) for f, _ in ServerDone._fields_}
            r["domain"] = self.held.pop(r["ticket"])
            out.append(r)
        return out

    def info(self) -> dict:
        i = ServerInfo()
        check(lib().frehd_server_info(self.h, C.byref(i)), "frehd_server_info")
        return {n: getattr(i, n) for n, _ in ServerInfo._fields_}

    def clock(self) -> float:
        return self.info()["clock"]

    def close(self):
        if getattr(self, "h", None):
            lib().frehd_server_destroy(self.h)
            self.h = None
            self.held.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def cg_solve_noalloc(nx: int, ny: int, Ct: int, Gx: int, Gy: int, b: int, x: int, eps: float,
                     max_iter: int, x0_from_x: bool = False, stream: int = 0,
                     wait: bool = True):
    """frehd_cg_solve_noalloc on device pointers (ints) the caller owns.

    Row-major nx*ny doubles each; at most 512*512 cells.  With wait=True the
    call blocks until the solve ends and returns (iterations, ||r||/||b||);
    otherwise it only queues the solve on `stream` and returns None."""
    L = lib()
    if not hasattr(L, "_domain_declared"):
        _declare_domain(L)
        L._domain_declared = True
    if wait:
        it, rel = C.c_int(0), C.c_double(0.0)
        check(L.frehd_cg_solve_noalloc(nx, ny, Ct, Gx, Gy, b, x, eps, max_iter, int(x0_from_x),
                                       stream or None, C.byref(it), C.byref(rel)),
              "frehd_cg_solve_noalloc")
        return it.value, rel.value
    check(L.frehd_cg_solve_noalloc(nx, ny, Ct, Gx, Gy, b, x, eps, max_iter, int(x0_from_x),
                                   stream or None, None, None), "frehd_cg_solve_noalloc")
    return None


def domain_from_deck(deck, device: int = 0, geometry: str = "fine", x0: int = X0_ZERO,
                     schedule: int = CG_SINGLE_SWEEP, decoupled: int = DECOUPLED_AS_ASSEMBLED,
                     precision: int = PRECISION_FP64, eps_inner: float = 1e-5):
    """A Domain initialised from a generated deck (frehdc_b200.deck)."""
    from . import deck as D
    d = Domain(D.config_dict(deck), device)
    if geometry == "fine":
        d.set_fine_bottoms(deck.zf, deck.r, block_check=deck.spec.block_check)
    else:
        tabs = deck.extra.get("tables")
        if tabs is None:
            tabs = D.build_tables(deck)
            deck.extra["tables"] = tabs
        d.set_tables(tabs)
    d.set_tide(D.tide_series(deck))
    for kind, series in D.forcing_series(deck).items():
        d.set_series({"inflow": SERIES_INFLOW, "windspd": SERIES_WIND_SPEED,
                      "winddir": SERIES_WIND_DIR}[kind], series)
    d.set_solver(x0)
    d.set_cg_schedule(schedule)
    d.set_decoupled(decoupled)
    if precision != PRECISION_FP64:
        d.set_precision(precision, eps_inner)
    d.init(deck.bottom, deck.bottomXP, deck.bottomYP, deck.surf0, deck.u0, None, deck.S0)
    for s, field in enumerate(deck.tracers, start=1):
        d.init_scalar(s, field)
    return d

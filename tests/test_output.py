"""Output files written from the device (DataOutput/SubOutput/writeRestartFile
formats, fileio.c:62-242).

The device formatter must print every value exactly as the reference's
fprintf("%4.4f \\n") does (glibc: round to nearest, ties to even, on the exact
binary value); the comparison is byte for byte against the C library's own
snprintf, through ctypes, on values chosen to hit exact ties, negative zeros,
tiny and large magnitudes and the values the device hands back to the host
(non-finite or |x| >= 1e15).  A domain's files must be the same bytes the
reference's writers produce from the downloaded state, and the surface must be
left round-tripped through the output datum as DataOutput leaves it.
"""
import ctypes
import os

import numpy as np
import pytest

from frehdc_b200 import deck as D
from frehdc_b200 import native

pytestmark = pytest.mark.gpu

_libc = ctypes.CDLL(None)
_libc.snprintf.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p, ctypes.c_double]


def c_fixed4(values) -> bytes:
    out = []
    buf = ctypes.create_string_buffer(512)
    for x in values:
        n = _libc.snprintf(buf, 512, b"%4.4f \n", float(x))
        out.append(buf.raw[:n])
    return b"".join(out)


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if native.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")


def _hard_values() -> np.ndarray:
    rng = np.random.default_rng(11)
    v = [0.0, -0.0, 1.0, -1.0, 0.5, 1e-300, -1e-300, 5e-324, 0.00005, -0.00005, 0.99995,
         9.99995, 123.45675, 1e14, -1e14, 999999999999999.9, 0.03125, -0.03125, 1.03125,
         2.5e-5, 7.5e-5, -7.5e-5, 1e-4, 3e-5, 4.99999999999e-5]
    v += list(np.arange(-64, 65) / 32.0)                # exact ties at the 4th decimal
    v += list(np.arange(-200, 201) / 2 ** 14)           # dyadic values near 0
    v += list(rng.normal(0, 3, 2000))
    v += list(rng.normal(0, 1e-3, 2000))
    v += list(10.0 ** rng.uniform(-8, 14, 2000) * rng.choice([-1, 1], 2000))
    v += list(np.nextafter(np.round(rng.uniform(-50, 50, 1000), 4) + 0.00005, np.inf))
    v += list(np.nextafter(np.round(rng.uniform(-50, 50, 1000), 4) + 0.00005, -np.inf))
    return np.array(v, dtype=np.float64)


def test_formatter_matches_printf():
    v = _hard_values()
    assert native.format_fixed4(v) == c_fixed4(v)


def test_formatter_host_path_values():
    # non-finite and very large values are printed by the host's snprintf
    v = np.array([1.0, np.inf, -np.inf, 1e15, -3.5e20, 1e300, 2.0])
    assert native.format_fixed4(v) == c_fixed4(v)
    assert native.format_fixed4(np.array([])) == b""


def test_domain_files_match_reference_writer(tmp_path):
    d = D.make_deck(D.DeckSpec(nx=40, ny=36, steps=6, seed=5, dry_frac=0.3))
    g = native.domain_from_deck(d)
    assert g.run(1, 5) == 0
    names = ["surf", "uuXP", "vvYP", "depth", "CDXP", "CDYP", "S", "Nx", "Oy", "Vx", "Vy", "V", "Z"]
    st = g.download(names)
    N = d.nx * d.ny
    off = d.offset
    prefix = str(tmp_path) + "/"
    g.write_output(prefix, 5, native.OUT_U | native.OUT_V | native.OUT_SURFACE | native.OUT_DEPTH |
                   native.OUT_CD | native.OUT_SCALAR | native.OUT_SUB)
    expect = {"uVelocity": st["uuXP"][:N], "vVelocity": st["vvYP"][:N],
              "surfaceZ": st["surf"][:N] - off, "depth": st["depth"][:N],
              "cdxp": st["CDXP"][:N], "cdyp": st["CDYP"][:N], "scalar": st["S"][:N],
              "SubNx": st["Nx"][:N], "SubOy": st["Oy"][:N], "SubVx": st["Vx"][:N],
              "SubVy": st["Vy"][:N], "SubV": st["V"][:N], "SubZ": st["Z"][:N]}
    for name, vals in expect.items():
        got = open(os.path.join(tmp_path, f"{name}_5.dat"), "rb").read()
        assert got == c_fixed4(vals), name
    # DataOutput's in-place round trip of the interior surface (fileio.c:65-66,120-121)
    after = g.download(["surf"])["surf"]
    assert np.array_equal(after[:N], (st["surf"][:N] - off) + off)
    assert np.array_equal(after[N:], st["surf"][N:])
    # restart file: tNEnd, dx, dy, surf - offset, uu, vv, S (fileio.c:217-238)
    st2 = g.download(["surf", "uuXP", "vvYP", "S"])
    g.write_restart(prefix, 5, 123.25)
    got = open(os.path.join(tmp_path, "restart_5.dat"), "rb").read()
    vals = np.concatenate([[123.25, d.spec.dx, d.spec.dx], st2["surf"][:N] - off, st2["uuXP"][:N],
                           st2["vvYP"][:N], st2["S"][:N]])
    assert got == c_fixed4(vals)

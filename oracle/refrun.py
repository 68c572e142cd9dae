"""Helpers around the reference oracle binaries in oracle/_ref (test
infrastructure: only tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline/reference legs use this module).

oracle/_ref is built from the reference's own sources by oracle/ref/Makefile
when the reference tree is present; the built binaries travel with the
repository snapshot, the sources do not.
"""
from __future__ import annotations

import os
import shutil
import struct
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
RECIPE = os.path.join(HERE, "ref")
# The reference checkout: $FREHD_REFERENCE, else a directory named "reference"
# beside this repository's root (where the build machine keeps it).
REF_SRC = os.environ.get("FREHD_REFERENCE") or os.path.join(
    os.path.dirname(os.path.dirname(HERE)), "reference")

PARITY_BIN = os.path.join(REF_DIR, "frehd_ref")
# the parity build with laspack's JacobiPrecond in place of SSORPrecond
JACOBI_BIN = os.path.join(REF_DIR, "frehd_ref_jacobi")
TIMING_BIN = os.path.join(REF_DIR, "frehd_ref_timing")
MLSTEST_BIN = os.path.join(REF_DIR, "mlstest")


def available() -> bool:
    return all(os.path.exists(b) for b in (PARITY_BIN, JACOBI_BIN, TIMING_BIN))


def build(quiet: bool = True) -> bool:
    """Build oracle/_ref from the reference sources when they are present."""
    if not os.path.isdir(os.path.join(REF_SRC, "frehdc5+")):
        return available()
    cmd = ["make", "-C", RECIPE, "-j8", f"REF={REF_SRC}", "OUT=../_ref"]
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL if quiet else None)
    return available()


def read_dump(path: str) -> dict:
    """Read a FRHDDUMP file written by oracle/ref/harness.c."""
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:8] != b"FRHDDUMP":
        raise ValueError(f"{path}: not a FRHDDUMP file")
    ver, count = struct.unpack_from("<ii", buf, 8)
    off = 16
    out = {}
    for _ in range(count):
        name = buf[off:off + 24].split(b"\0", 1)[0].decode()
        n, ty, _pad = struct.unpack_from("<qii", buf, off + 24)
        off += 40
        dt = np.float64 if ty == 0 else np.int32
        nb = n * (8 if ty == 0 else 4)
        out[name] = np.frombuffer(buf, dtype=dt, count=n, offset=off).copy()
        off += nb
    return out


def run(deck_dir: str, steps: int, out_path: str, timing: bool = False,
        precond: str = "ssor") -> dict:
    """Run the reference for `steps` steps and return its final state.

    precond "ssor" is the reference as shipped (SSORPrecond, nsfunctions.c:1016);
    "jacobi" hands laspack's JacobiPrecond to the same CGIter call."""
    binary = TIMING_BIN if timing else (JACOBI_BIN if precond == "jacobi" else PARITY_BIN)
    mode = "time" if timing else "run"
    r = subprocess.run([binary, mode, os.path.abspath(deck_dir), str(steps),
                        os.path.abspath(out_path)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"frehd_ref failed ({r.returncode}): {r.stderr[-2000:]}\n{r.stdout[-2000:]}")
    st = read_dump(out_path)
    if timing:
        import json
        for line in r.stdout.splitlines():
            if line.startswith("{"):
                st["timing"] = json.loads(line)
    return st


def time_run(deck_dir: str, steps: int) -> dict:
    """Wall time of the reference's step loop (stock allocator build)."""
    r = subprocess.run([TIMING_BIN, "time", os.path.abspath(deck_dir), str(steps)],
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"frehd_ref_timing failed: {r.stderr[-2000:]}")
    import json
    for line in r.stdout.splitlines():
        if line.startswith("{"):
            return json.loads(line)
    raise RuntimeError("frehd_ref_timing printed no timing line")


def phases(deck_dir: str, steps: int, out_dir: str, at=None) -> None:
    os.makedirs(out_dir, exist_ok=True)
    cmd = [PARITY_BIN, "phases", os.path.abspath(deck_dir), str(steps), os.path.abspath(out_dir)]
    if at:
        cmd += ["--at", ",".join(str(a) for a in at)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"frehd_ref phases failed: {r.stderr[-2000:]}")


def phase_dump(out_dir: str, tt: int, p: int) -> dict:
    return read_dump(os.path.join(out_dir, f"step{tt:04d}_p{p}.bin"))


def copy_deck(src: str, dst: str) -> str:
    if os.path.exists(dst):
        shutil.rmtree(dst)
    shutil.copytree(src, dst)
    return dst


def write_dump(path: str, arrays: dict) -> None:
    """Write a FRHDDUMP file (the harness's inject mode reads it)."""
    with open(path, "wb") as f:
        f.write(b"FRHDDUMP")
        f.write(struct.pack("<ii", 1, len(arrays)))
        for name, a in arrays.items():
            a = np.asarray(a)
            ty = 1 if a.dtype.kind in "iu" else 0
            a = np.ascontiguousarray(a, dtype="<i4" if ty else "<f8")
            nm = name.encode()[:23].ljust(24, b"\0")
            f.write(nm)
            f.write(struct.pack("<qii", a.size, ty, 0))
            f.write(a.tobytes())


def inject(deck_dir: str, tt: int, out_dir: str, state: dict) -> None:
    """Run step tt of the reference from an injected state, with phase dumps."""
    os.makedirs(out_dir, exist_ok=True)
    sp = os.path.abspath(os.path.join(out_dir, "injected_state.bin"))
    write_dump(sp, state)
    r = subprocess.run([PARITY_BIN, "inject", os.path.abspath(deck_dir), str(tt),
                        os.path.abspath(out_dir), sp], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"frehd_ref inject failed ({r.returncode}): {r.stderr[-2000:]}")

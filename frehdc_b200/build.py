"""Build of the in-tree native library ``frehdc_b200/libfrehd_b200.so``.

All device code is compiled for sm_100a only.  The plain FP64 kernels are built
with --fmad=false so that a*b+c is never contracted: together with an unchanged
evaluation order this keeps their doubles identical to the host restatement of
the reference step.  Objects are cached under ``frehdc_b200/_build`` and rebuilt
when a source or header is newer.

Each .cu file is compiled whole-program (no relocatable device code; no device
symbol crosses files).  With -rdc the device linker lays out the function-scope
__shared__ variables of all files in one range, and a kernel's static shared
memory becomes the end of that range: k_cg1 grew from 3.9 KB to 32 KB and
k_update_vel from 0.2 KB to 13 KB, which shrank the L1 carve-out and cost the
CG 12 % at 4096 x 4096 (16.0 -> 14.3 ms per solve once removed).
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(REPO, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfrehd_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2,-fno-fast-math",
          "-I", INCLUDE, "-I", CSRC]
# Per-source extra flags: files whose kernels must reproduce host doubles exactly
# are built without FMA contraction; the mixed-precision kernels keep FMA.
EXTRA = {
    "default": ["--fmad=false"],
    "cg.cu": ["--fmad=true"],
    "noalloc.cu": ["--fmad=true"],
    "cg1.cu": ["--fmad=true"],
}


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers() -> list[str]:
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_library(verbose: bool = False, force: bool = False) -> str:
    """Compile every CUDA/C++ source under csrc/ and link the shared library."""
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    hdrs = _headers()
    objs = []
    for src in srcs:
        base = os.path.basename(src)
        obj = os.path.join(BUILD, base + ".o")
        objs.append(obj)
        if not force and not _stale(obj, [src] + hdrs + [__file__]):
            continue
        extra = EXTRA.get(base, EXTRA["default"])
        cmd = [nvcc] + ARCH + COMMON + extra + ["-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd = [shutil.which("g++") or "g++", "-O2", "-fPIC", "-std=c++17", "-fno-fast-math",
                   "-I", INCLUDE, "-I", CSRC, "-I", "/usr/local/cuda/include", "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", LIB] + objs + \
            ["-lcudart", "-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB



DROPIN = os.path.join(HERE, "dropin")
DROPIN_BIN = os.path.join(DROPIN, "_build", "frehd_dropin")


def build_dropin(ref_src: str, quiet: bool = True) -> str | None:
    """Build the drop-in host (the reference's host program with nssolve_b200.c
    in place of nssolve.c, linked against the library) from the reference
    sources under ref_src.  Without those sources an existing binary is kept;
    returns its path, or None when there is none."""
    if os.path.isdir(os.path.join(ref_src, "frehdc5+")):
        build_library(verbose=False)
        subprocess.run(["make", "-C", DROPIN, "-j8", f"REF={ref_src}"], check=True,
                       stdout=subprocess.DEVNULL if quiet else None)
    return DROPIN_BIN if os.path.exists(DROPIN_BIN) else None


if __name__ == "__main__":
    build_library(verbose=True, force="--force" in sys.argv)

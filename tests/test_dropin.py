"""The drop-in host: the reference's own host program (FREHD.c main, Init,
DataOutput, monitorCFL, all unchanged) with nssolve_b200.c in place of
nssolve.c, stepping on the GPU through the C ABI.

CPU: the binary is linked against the library, defines the nssolve.h entry
points and the frehd_dropin.h API, and fails loudly when no device is present
(there is no host fallback).  GPU: on the same deck it writes the same output
files as the reference program (Jacobi-preconditioned build), whether the
reference's DataOutput prints them from copied-back state or the device formats
them (FREHD_DEVICE_OUTPUT=1), and its
full-precision state at the output steps matches the reference's to the
rounding level of two Jacobi-PCG solves.
"""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from frehdc_b200 import build as fb
from frehdc_b200 import deck as D
from frehdc_b200 import native
from oracle import refrun
from tests.helpers import SPECS, max_rel

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "frehd_dropin.h")
ENTRY_POINTS = ["SolveAll", "oneCompleteStep", "solveSourceTerm", "solveFreeSurface", "updateData"]
OUT_STEPS = 10


def _binary() -> str:
    b = fb.build_dropin(refrun.REF_SRC)
    if b is None:
        pytest.fail("drop-in host not built (frehdc_b200/dropin/Makefile needs the reference sources)")
    return b


def _declared() -> list[str]:
    text = re.sub(r"/\*.*?\*/", " ", open(HEADER).read(), flags=re.S)
    return sorted(set(re.findall(r"\b(frehd_gpu_[a-z0-9_]+)\s*\(", text)))


def _deck_dir(name: str, root: str) -> tuple:
    d = D.make_deck(SPECS[name], with_tables=True)
    path = os.path.join(root, name)
    D.write_reference_deck(d, path, out_steps=OUT_STEPS)
    return d, path


def test_dropin_links_library_and_defines_entry_points():
    b = _binary()
    dyn = subprocess.run(["readelf", "-d", b], capture_output=True, text=True, check=True).stdout
    assert "libfrehd_b200.so" in dyn
    syms = subprocess.run(["nm", "--defined-only", b], capture_output=True, text=True,
                          check=True).stdout
    defined = {ln.split()[-1] for ln in syms.splitlines() if ln.split()[-2:-1] in (["T"], ["t"])}
    for name in ENTRY_POINTS + _declared():
        assert name in defined, name
    # the library's step is what the program calls
    undef = subprocess.run(["nm", "--undefined-only", b], capture_output=True, text=True,
                           check=True).stdout
    for name in ["frehd_domain_create", "frehd_domain_run", "frehd_domain_set_tables"]:
        assert name in undef


def test_header_declares_the_gpu_api():
    assert {"frehd_gpu_init", "frehd_gpu_run", "frehd_gpu_sync_to_host",
            "frehd_gpu_finalize", "frehd_gpu_status"} <= set(_declared())


def test_dropin_fails_loudly_without_a_device(tmp_path):
    if native.device_count() > 0:
        pytest.skip("a CUDA device is visible")
    b = _binary()
    _, path = _deck_dir("wet48x40", str(tmp_path))
    r = subprocess.run([b], cwd=path, capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert "frehd_b200: frehd_gpu_init failed" in r.stderr
    # Init and the tt = 0 output ran on the host before the device was needed
    assert os.path.exists(os.path.join(path, "output", "surfaceZ_0.dat"))
    assert not os.path.exists(os.path.join(path, "output", f"surfaceZ_{OUT_STEPS}.dat"))


def _read_outputs(folder: str) -> dict:
    out = {}
    for f in sorted(os.listdir(folder)):
        if f.endswith(".dat"):
            out[f] = np.loadtxt(os.path.join(folder, f))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("output", ["host", "device"])
@pytest.mark.parametrize("name", ["wet48x40", "dry40x36", "inflow36x30", "wind40x32"])
def test_dropin_matches_reference_program(name, output, tmp_path):
    if native.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")
    if not os.path.exists(refrun.JACOBI_BIN):
        pytest.fail("oracle/_ref/frehd_ref_jacobi missing (built with the oracle recipe)")
    b = _binary()
    d, ref_deck = _deck_dir(name, str(tmp_path / "ref"))
    gpu_deck = str(tmp_path / "gpu" / name)
    shutil.copytree(ref_deck, gpu_deck)
    steps = SPECS[name].steps                      # a multiple of OUT_STEPS, < Nt
    assert steps % OUT_STEPS == 0 and steps < d.Nt
    ref = refrun.run(ref_deck, steps, str(tmp_path / "ref.bin"), precond="jacobi")
    env = dict(os.environ, FREHD_DUMP=str(tmp_path / "gpu_%d.bin"),
               FREHD_DEVICE_OUTPUT="1" if output == "device" else "0")
    r = subprocess.run([b], cwd=gpu_deck, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:] + r.stdout[-2000:]
    assert "Time stepping completed" in r.stdout
    got = refrun.read_dump(str(tmp_path / f"gpu_{steps}.bin"))
    assert got["meta"][4] == steps
    # the state at the reference's last step (after its DataOutput); face
    # velocities amplify the CG's eta error on thin-water faces, so they get the
    # whole-run velocity bound of the device parity tests
    for field, tol in [("surf", 1e-9), ("S", 1e-9), ("uuXP", 3e-9), ("vvYP", 3e-9),
                       ("depth", 1e-9), ("cellV", 1e-9)]:
        assert max_rel(got[field], ref[field]) < tol, field
    assert np.array_equal(got["ind"], ref["ind"])
    # the output files both programs wrote (4 decimals, fileio.c:186-189)
    ro = _read_outputs(os.path.join(ref_deck, "output"))
    go = _read_outputs(os.path.join(gpu_deck, "output"))
    common = [f for f in ro if f in go]
    expect = {f"{v}_{t}.dat" for v in ("surfaceZ", "uVelocity", "vVelocity", "depth", "scalar")
              for t in range(0, steps + 1, OUT_STEPS)}
    assert expect <= set(common)
    for f in common:
        diff = np.abs(go[f] - ro[f])
        # values that agree to 1e-12 print the same 4 decimals except at a tie
        assert diff.max() <= 1.0001e-4, f
        assert np.count_nonzero(diff) <= 2, f


@pytest.mark.gpu
def test_dropin_exits_like_the_reference_on_cfl(tmp_path):
    """CFL > 20 (an initial 100 m/s jet, uuic.dat): like the reference program,
    whose monitorCFL writes the state and exits (nsfunctions.c:1225-1231), the
    drop-in host stops at the same step with a failure status, the same message
    and the same output files of that step."""
    if native.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")
    b = _binary()
    spec = D.DeckSpec(nx=48, ny=40, steps=30, seed=3, u0_block=(20, 28, 16, 24, 100.0))
    d = D.make_deck(spec, with_tables=True)
    ref_deck, gpu_deck = str(tmp_path / "ref"), str(tmp_path / "gpu")
    D.write_reference_deck(d, ref_deck, out_steps=OUT_STEPS)
    shutil.copytree(ref_deck, gpu_deck)
    r_ref = subprocess.run([refrun.JACOBI_BIN, "run", os.path.abspath(ref_deck), str(spec.steps),
                            str(tmp_path / "ref.bin")], capture_output=True, text=True, timeout=300)
    r_gpu = subprocess.run([b], cwd=gpu_deck, capture_output=True, text=True, timeout=300)
    msg = "Max CFL exceeds 20, program forced to quit!"
    assert r_ref.returncode == 1 and msg in r_ref.stdout
    assert r_gpu.returncode == 1 and msg in r_gpu.stdout, r_gpu.stderr[-2000:]
    ro = _read_outputs(os.path.join(ref_deck, "output"))
    go = _read_outputs(os.path.join(gpu_deck, "output"))
    # the step the reference stopped at: its DataOutput files beyond step 0
    stopped = {f for f in ro if not f.endswith("_0.dat")}
    assert stopped and stopped <= set(go)
    assert {f for f in go if not f.endswith("_0.dat")} == stopped
    for f in stopped:
        diff = np.abs(go[f] - ro[f])
        assert diff.max() <= 1.0001e-4, f
        assert np.count_nonzero(diff) <= 2, f

"""The C restatement oracle pinned against the reference itself (CPU only).

oracle/_ref/frehd_ref is the unchanged reference (frehdc5+ + laspack) built by
oracle/ref/Makefile.  Its phase dumps of one oneCompleteStep are compared with
the restatement array by array: bit for bit for every stencil phase, and to the
CG tolerance for the linear solve.
"""
import os
import subprocess

import numpy as np
import pytest

from frehdc_b200 import deck as D
from oracle import port, refrun
from tests.helpers import EXPLICIT_OUT, STATE, TEMPS, deck_for, max_rel, mismatches

pytestmark = pytest.mark.skipif(not refrun.build(), reason="reference oracle not built")


def _load(o, dump):
    for n in STATE + TEMPS:
        o.set(n, dump[n].astype(np.float64))


def test_laspack_known_answer():
    """laspack's own check (laspack/check/check): mlstest over 132 solver set-ups."""
    chk = os.path.join(refrun.REF_SRC, "laspack", "check")
    if not os.path.exists(os.path.join(chk, "mlstest.org")):
        pytest.skip("laspack/check golden not present")
    out = []
    for solver in ["mg", "mgpcg", "bpxpcg"]:
        tpl = open(os.path.join(chk, solver + ".tpl")).read()
        for sm in [1, 2, 3, 4, 6, 7, 8, 9, 10, 11, 12]:
            for pc in [0, 1, 2, 3]:
                out.append(f"Testing ... solver = {solver}, smoother = {sm}, preconditioner = {pc}")
                inp = tpl.replace("SMOOTHER_ID", str(sm)).replace("PRECOND_ID", str(pc))
                r = subprocess.run([refrun.MLSTEST_BIN], input=inp, capture_output=True, text=True)
                out += [ln for ln in r.stdout.split("\n") if "=" in ln]
    golden = open(os.path.join(chk, "mlstest.org")).read().rstrip("\n").split("\n")
    assert out == golden


@pytest.mark.parametrize("name", ["wet48x40", "dry40x36"])
def test_tide_series_bitwise(name, scratch):
    d, path = deck_for(name, str(scratch))
    st = refrun.run(path, 2, os.path.join(path, "t.bin"))
    assert np.array_equal(D.tide_series(d), st["tideP"])


@pytest.mark.parametrize("name", ["wet48x40", "dry40x36", "dry37x29"])
def test_init_bitwise(name, scratch):
    d, path = deck_for(name, str(scratch))
    ph = os.path.join(path, "ph_init")
    refrun.phases(path, 1, ph)
    p0 = refrun.phase_dump(ph, 1, 0)
    o = port.from_deck(d)
    got = {n: o.get(n) for n in STATE + ["bottomZ", "bottomXP", "bottomYP", "cellV", "Sm",
                                         "depthXP", "depthYP"]}
    assert mismatches(got, p0, list(got)) == []


@pytest.mark.parametrize("name,steps", [("wet48x40", 8), ("dry40x36", 30), ("dry37x29", 40),
                                        ("tvd44x36", 40), ("inflow36x30", 30),
                                        ("wind40x32", 30)])
def test_phases_bitwise(name, steps, scratch):
    """Each phase of each step from the reference's own pre-phase state."""
    d, path = deck_for(name, str(scratch))
    ph = os.path.join(path, "ph")
    refrun.phases(path, steps, ph)
    o = port.from_deck(d, precond=port.PRECOND_SSOR, x0=port.X0_ZERO)
    for tt in range(1, steps + 1):
        p0, p1, p2, p3 = (refrun.phase_dump(ph, tt, k) for k in range(4))
        _load(o, p0)
        o.explicit(tt)
        assert mismatches({n: o.get(n) for n in EXPLICIT_OUT}, p1, EXPLICIT_OUT) == [], tt
        _load(o, p1)
        o.solve()
        assert max_rel(o.get("x"), p2["x"]) < 1e-12, tt
        o.update(tt, p2["x"])
        got = {n: o.get(n) for n in STATE + TEMPS}
        assert mismatches(got, p3, STATE + TEMPS) == [], tt


def test_injected_branches_bitwise(scratch):
    """Branches a smooth run rarely reaches, driven by injected states: the CFL
    limiter (incl. the CFLx test in the y branch), scalar singularities (S > 100
    and S < 0 blocks) and closed dry cells."""
    d, path = deck_for("dry40x36", str(scratch))
    ph = os.path.join(path, "ph_base")
    refrun.phases(path, 6, ph, at=[6])
    base = refrun.phase_dump(ph, 6, 0)
    rng = np.random.default_rng(17)
    st = {n: base[n].copy() for n in STATE + TEMPS}
    T = st["CFLx"].size
    st["CFLx"] = rng.uniform(0.0, 1.0, T)
    st["CFLy"] = rng.uniform(0.0, 1.0, T)
    nx = d.nx
    S = st["S"]
    for j in range(10, 14):
        S[j * nx + 10:j * nx + 14] = 150.0
        S[j * nx + 25:j * nx + 29] = -3.0
    out = os.path.join(path, "inj")
    refrun.inject(path, 6, out, st)
    p0, p1, p2, p3 = (refrun.phase_dump(out, 6, k) for k in range(4))
    o = port.from_deck(d)
    _load(o, p0)
    o.explicit(6)
    assert mismatches({n: o.get(n) for n in EXPLICIT_OUT}, p1, EXPLICIT_OUT) == []
    _load(o, p1)
    o.update(6, p2["x"])
    got = {n: o.get(n) for n in STATE + TEMPS}
    assert mismatches(got, p3, STATE + TEMPS) == []
    # the injected blocks must have reached the singularity branch
    assert np.any((p0["S"] > 100) & (p3["S"] == 0))


def test_full_run_jacobi_matches_reference(scratch):
    """Whole runs: reference (SSOR-PCG from x=0) vs oracle with the device's
    solver choice (Jacobi-PCG from the current surface), both to eps = 1e-12."""
    d, path = deck_for("dry40x36", str(scratch))
    steps = 40
    ref = refrun.run(path, steps, os.path.join(path, "full.bin"))
    o = port.from_deck(d, precond=port.PRECOND_JACOBI, x0=port.X0_SURFACE)
    for tt in range(1, steps + 1):
        o.step(tt)
    for n in ["surf", "uuXP", "vvYP", "S"]:
        assert max_rel(o.get(n), ref[n]) <= 1e-9, n


@pytest.mark.parametrize("block_check", [False, True])
def test_oracle_deck_builders_match_library(block_check):
    """The deck pre-processing of runs of the reference program alone
    (oracle/deckprep.c, used by bench.py's reference arm so that it loads no
    library of the product) gives the library's tables and bottoms bit for bit."""
    from frehdc_b200 import deck as D
    spec = D.DeckSpec(nx=40, ny=36, steps=5, seed=3, dry_frac=0.3, block_check=block_check)
    a, b = D.make_deck(spec), D.make_deck(spec, host=port)
    for f in ("bottom", "bottomXP", "bottomYP"):
        assert getattr(a, f).tobytes() == getattr(b, f).tobytes(), f
    assert D.build_tables(a).tobytes() == D.build_tables(a, host=port).tobytes()

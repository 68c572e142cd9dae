"""CUDA step parity (needs a B200): the device path against the C oracle,
which the CPU suite pins bit for bit to the reference itself.

Stencil phases must match the oracle's doubles exactly; the drag coefficients
go through pow(), where CUDA and glibc may differ in the last place, so they
are compared to a few ulp.  The linear solve is compared to the CG tolerance.

Whole runs: the surface and the scalar to 1e-9 relative (max norm).  Face
velocities are compared to 6e-9.  Two solves that both meet ||r|| < 1e-12 ||b||
(the reference's own SSOR-PCG and a Jacobi-PCG, both on the CPU) already differ
in the velocities: by 1.2e-9 on the 30%-dry deck and 3.3e-9 after 40 steps of
the 15%-dry TVD deck.  u = En - g dt (Nx/Vx) d(eta) amplifies the solver's eta
error on thin-water faces; the surface itself agrees to ~1e-11.
"""
import os

import numpy as np
import pytest

from frehdc_b200 import deck as D
from frehdc_b200 import native
from oracle import port, refrun
from tests.helpers import SPECS, deck_for, max_rel, mismatches

pytestmark = pytest.mark.gpu

EXACT = ["surf", "uuXP", "vvYP", "S", "depth", "V", "Z", "Nx", "Oy", "Vx", "Vy", "Zx", "Zy", "ind",
         "surfOld", "cellV", "Sm", "Fuu", "Fvv", "CFLx", "CFLy", "uuYP", "vvXP"]
POW = ["CDXP", "CDYP"]
RUN_TOL = {"surf": 1e-9, "S": 1e-9, "uuXP": 6e-9, "vvYP": 6e-9}
UPLOAD = ["surf", "uuXP", "vvYP", "S", "depth", "CDXP", "CDYP", "CFLx", "CFLy", "V", "Z", "Nx",
          "Oy", "Vx", "Vy", "Zx", "Zy", "ind", "bottomZ", "bottomXP", "bottomYP"]


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if native.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")


def _oracle_state(o, names):
    return {n: o.get(n) for n in names}


@pytest.mark.parametrize("name", ["wet48x40", "dry40x36"])
@pytest.mark.parametrize("geometry", ["fine", "tables"])
def test_init_bitwise(name, geometry, scratch):
    d, _ = deck_for(name, str(scratch))
    o = port.from_deck(d)
    g = native.domain_from_deck(d, geometry=geometry)
    got = g.download(UPLOAD)
    ref = _oracle_state(o, UPLOAD)
    assert mismatches(got, ref, [n for n in UPLOAD if n not in POW]) == []
    assert mismatches(got, ref, POW, exact=False, rtol=1e-15) == []


@pytest.mark.parametrize("name,steps", [("wet48x40", 6), ("dry40x36", 25), ("dry37x29", 25),
                                        ("tvd44x36", 25), ("inflow36x30", 20)])
def test_phases_bitwise(name, steps, scratch):
    """Each step: the oracle's state is uploaded, then the device's explicit
    phase and update phase (fed the oracle's x) must give the oracle's doubles."""
    d, _ = deck_for(name, str(scratch))
    o = port.from_deck(d, precond=port.PRECOND_JACOBI, x0=port.X0_ZERO)
    g = native.domain_from_deck(d, geometry="fine")
    for tt in range(1, steps + 1):
        g.upload(_oracle_state(o, UPLOAD))
        o.explicit(tt)
        g.phase(native.PHASE_EXPLICIT, tt)
        sysg = g.system()
        en = g.download(["EnXP", "EnYP"])
        sysr = _oracle_state(o, ["GnCt", "GnXP", "GnXM", "GnYP", "GnYM", "z", "EnXP", "EnYP"])
        assert mismatches({**sysg, **en}, sysr, list(sysr)) == [], tt
        o.solve()
        x = o.get("x")
        o.update(tt, x)
        g.phase(native.PHASE_UPDATE, tt, x_ext=x)
        got = g.download(EXACT + POW)
        ref = _oracle_state(o, EXACT + POW)
        assert mismatches(got, ref, EXACT) == [], tt
        assert mismatches(got, ref, POW, exact=False, rtol=1e-15) == [], tt


def test_phases_with_wind(scratch):
    """Wind (nsfunctions.c:609-648): the direction's cosine and sine are taken on
    the host as the reference takes them, so only the thin-layer decay's exp()
    may differ from glibc's in the last place; the phases match to 1e-15."""
    d, _ = deck_for("wind40x32", str(scratch))
    o = port.from_deck(d, precond=port.PRECOND_JACOBI, x0=port.X0_ZERO)
    g = native.domain_from_deck(d, geometry="fine")
    up = UPLOAD + ["depthXP", "depthYP"]
    names = ["GnCt", "GnXP", "GnXM", "GnYP", "GnYM", "z", "EnXP", "EnYP"]
    for tt in range(1, 16):
        g.upload(_oracle_state(o, up))
        o.explicit(tt)
        g.phase(native.PHASE_EXPLICIT, tt)
        sysg = {**g.system(), **g.download(["EnXP", "EnYP"])}
        assert mismatches(sysg, _oracle_state(o, names), names, exact=False, rtol=1e-15) == [], tt
        o.solve()
        x = o.get("x")
        o.update(tt, x)
        g.phase(native.PHASE_UPDATE, tt, x_ext=x)
        got = g.download(EXACT + POW + ["depthXP", "depthYP"])
        ref = _oracle_state(o, EXACT + POW + ["depthXP", "depthYP"])
        assert mismatches(got, ref, EXACT + POW, exact=False, rtol=1e-13) == [], tt
        # the face depths the next wind term reads are the update's own doubles
        N = d.nx * d.ny
        assert np.array_equal(got["depthXP"][:N], ref["depthXP"][:N]), tt
        assert np.array_equal(got["depthYP"][:N], ref["depthYP"][:N]), tt


def test_update_series_equals_set_series(scratch):
    """Forcing streamed in while the model runs (frehd_domain_update_series,
    queued before each step) gives the doubles of the same series set up front."""
    d, _ = deck_for("wind40x32", str(scratch))
    alt_tide = D.tide_series(d) + 0.03 * np.sin(np.arange(d.Nt))
    alt_dir = D.forcing_series(d)["winddir"] + 25.0
    whole = native.domain_from_deck(d)
    whole.set_tide(alt_tide)
    whole.set_series(native.SERIES_WIND_DIR, alt_dir)
    streamed = native.domain_from_deck(d)
    for tt in range(1, 9):
        for kind, arr in ((native.SERIES_TIDE, alt_tide), (native.SERIES_WIND_DIR, alt_dir)):
            streamed.update_series(kind, tt, 1, arr.ctypes.data + 8 * tt)
        assert streamed.step(tt) == 0
    assert whole.run(1, 8) == 0
    a = whole.download(["surf", "uuXP", "vvYP", "S"])
    b = streamed.download(["surf", "uuXP", "vvYP", "S"])
    for n in a:
        assert np.array_equal(a[n], b[n]), n
    with pytest.raises(native.FrehdError):
        streamed.update_series(native.SERIES_TIDE, d.Nt, 1, alt_tide.ctypes.data)


SCHEDULES = {"single_sweep": native.CG_SINGLE_SWEEP, "two_phase": native.CG_TWO_PHASE}


@pytest.mark.parametrize("schedule", list(SCHEDULES))
@pytest.mark.parametrize("name", ["wet48x40", "dry40x36"])
def test_solve_matches_oracle(name, schedule, scratch):
    d, _ = deck_for(name, str(scratch))
    o = port.from_deck(d, precond=port.PRECOND_JACOBI, x0=port.X0_ZERO)
    g = native.domain_from_deck(d, geometry="fine", schedule=SCHEDULES[schedule])
    for tt in range(1, 4):
        g.upload(_oracle_state(o, UPLOAD))
        o.explicit(tt)
        o.solve()
        g.phase(native.PHASE_EXPLICIT, tt)
        g.phase(native.PHASE_SOLVE, tt)
        xg = g.solution()
        # both solves meet ||r|| < 1e-12 ||b||; x agrees to the conditioning of A
        assert max_rel(xg, o.get("x")) < 1e-10
        o.update(tt, o.get("x"))


def _true_residual(sysm: dict, x_t: np.ndarray, nx: int, ny: int) -> float:
    """||z - A x|| / ||z|| of the assembled 5-point system (setupMatrix,
    nsfunctions.c:927-1001: row entries -GnXM, -GnYM, GnCt, -GnYP, -GnXP; z and x
    in the transposed order k = i*ny + j, the coefficients row-major)."""
    def rm(v):  # transposed -> row-major (ny, nx)
        return v.reshape(nx, ny).T
    x = rm(x_t)
    z = rm(sysm["z"])
    c = {n: sysm[n].reshape(ny, nx) for n in ("GnCt", "GnXP", "GnXM", "GnYP", "GnYM")}
    ax = c["GnCt"] * x
    ax[:, :-1] -= c["GnXP"][:, :-1] * x[:, 1:]
    ax[:, 1:] -= c["GnXM"][:, 1:] * x[:, :-1]
    ax[:-1, :] -= c["GnYP"][:-1, :] * x[1:, :]
    ax[1:, :] -= c["GnYM"][1:, :] * x[:-1, :]
    return float(np.linalg.norm(z - ax) / np.linalg.norm(z))


def test_true_residual_of_the_solution(scratch):
    """The device's x meets the stopping rule on the true residual z - A x of the
    assembled system, not only on the residual the CG recurrence carries (the
    scaled solve updates x~ apart from r~), over several stopping tolerances and
    iteration counts of both parities."""
    parities = set()
    for name in ("dry40x36", "tvdwet44x36"):
        for eps in (1e-12, 3e-12, 1e-11, 3e-11):
            d = D.make_deck(SPECS[name].replace(eps=eps))
            g = native.domain_from_deck(d, geometry="fine")
            for tt in range(1, 9):
                g.phase(native.PHASE_EXPLICIT, tt)
                g.phase(native.PHASE_SOLVE, tt)
                res = _true_residual(g.system(), g.solution(), d.nx, d.ny)
                g.phase(native.PHASE_UPDATE, tt)
                st = g.stats()
                if st["cg_fallback"]:
                    continue
                assert res < 2 * eps, (name, eps, tt, res, st["cg_iters"])
                parities.add(st["cg_iters"] % 2)
    assert parities == {0, 1}


@pytest.mark.parametrize("schedule", list(SCHEDULES))
@pytest.mark.parametrize("name", ["wet48x40", "dry40x36", "dry37x29", "tvdwet44x36",
                                  "inflow36x30", "wind40x32"])
def test_full_run_matches_oracle(name, schedule, scratch):
    """Whole run against the oracle in the reference's own solver set-up (SSOR-PCG
    from x = 0, which tracks the reference program to ~1e-13)."""
    d, _ = deck_for(name, str(scratch))
    steps = SPECS[name].steps
    o = port.from_deck(d, precond=port.PRECOND_SSOR, x0=port.X0_ZERO)
    for tt in range(1, steps + 1):
        o.step(tt)
    g = native.domain_from_deck(d, geometry="fine", schedule=SCHEDULES[schedule])
    assert g.run(1, steps) == 0
    st = g.stats()
    assert st["step"] == steps
    got = g.download(["surf", "uuXP", "vvYP", "S", "cellV"])
    for n in ["surf", "uuXP", "vvYP", "S"]:
        assert max_rel(got[n], o.get(n)) <= RUN_TOL[n], n
    # volume ledger: the device's fixed-order sum of cellV equals the host sum
    assert abs(st["volume"] - got["cellV"].sum()) <= 1e-12 * abs(got["cellV"].sum())


@pytest.mark.skipif(not refrun.available(), reason="reference oracle binaries not present")
@pytest.mark.parametrize("name", ["wet48x40", "dry40x36"])
def test_full_run_matches_reference(name, scratch):
    """Whole run against the reference program itself (SSOR-PCG from x = 0)."""
    d, path = deck_for(name, str(scratch))
    steps = SPECS[name].steps
    ref = refrun.run(path, steps, os.path.join(path, "gpu_full.bin"))
    g = native.domain_from_deck(d, geometry="fine")
    assert g.run(1, steps) == 0
    got = g.download(["surf", "uuXP", "vvYP", "S"])
    for n in ["surf", "uuXP", "vvYP", "S"]:
        assert max_rel(got[n], ref[n]) <= RUN_TOL[n], n


def test_warm_start_option(scratch):
    """The warm-started solve (FREHD_X0_SURFACE) meets the same residual test."""
    d, _ = deck_for("wet48x40", str(scratch))
    g = native.domain_from_deck(d, geometry="fine", x0=native.X0_SURFACE)
    assert g.run(1, 10) == 0
    st = g.stats()
    assert st["cg_rel_residual"] < d.spec.eps
    o = port.from_deck(d, precond=port.PRECOND_SSOR, x0=port.X0_ZERO)
    for tt in range(1, 11):
        o.step(tt)
    got = g.download(["surf"])
    assert max_rel(got["surf"], o.get("surf")) <= 1e-9


def test_run_is_bit_reproducible(scratch):
    d, _ = deck_for("dry40x36", str(scratch))
    a = native.domain_from_deck(d, geometry="fine")
    b = native.domain_from_deck(d, geometry="tables")
    a.run(1, 15)
    b.run(1, 15)
    da = a.download(["surf", "uuXP", "vvYP", "S"])
    db = b.download(["surf", "uuXP", "vvYP", "S"])
    assert mismatches(da, db, list(da)) == []


@pytest.mark.parametrize("decoupled", [native.DECOUPLED_AS_ASSEMBLED, native.DECOUPLED_ELIMINATED])
@pytest.mark.parametrize("name", ["wet48x40", "dry37x29"])
def test_schedules_agree(name, decoupled, scratch):
    """The single-sweep and two-phase schedules solve the same system to the CG
    tolerance; without a stall fallback their iteration counts are within one."""
    d, _ = deck_for(name, str(scratch))
    a = native.domain_from_deck(d, geometry="fine", schedule=native.CG_SINGLE_SWEEP,
                                decoupled=decoupled)
    b = native.domain_from_deck(d, geometry="fine", schedule=native.CG_TWO_PHASE,
                                decoupled=decoupled)
    for g in (a, b):
        g.phase(native.PHASE_EXPLICIT, 1)
        g.phase(native.PHASE_SOLVE, 1)
        g.phase(native.PHASE_UPDATE, 1)
    sa, sb = a.stats(), b.stats()
    assert sa["cg_fallback"] == sb["cg_fallback"]
    if not sa["cg_fallback"]:
        assert abs(sa["cg_iters"] - sb["cg_iters"]) <= 1
    assert sa["cg_rel_residual"] < d.spec.eps and sb["cg_rel_residual"] < d.spec.eps
    assert max_rel(a.solution(), b.solution()) < 1e-10


@pytest.mark.parametrize("schedule", list(SCHEDULES))
def test_stalled_solve_falls_back(schedule, scratch):
    """On the wet deck the assembled (non-symmetric) matrix stalls near 4e-12
    relative residual, where laspack's CGIter runs on to maxIter.  The device
    notices (no halving of ||r|| in 400 iterations), solves the step again with
    the decoupled rows eliminated, and reports it; the solve then meets eps."""
    d, _ = deck_for("wet48x40", str(scratch))
    g = native.domain_from_deck(d, geometry="fine", schedule=SCHEDULES[schedule])
    e = native.domain_from_deck(d, geometry="fine", schedule=SCHEDULES[schedule],
                                decoupled=native.DECOUPLED_ELIMINATED)
    for h in (g, e):
        h.phase(native.PHASE_EXPLICIT, 1)
        h.phase(native.PHASE_SOLVE, 1)
        h.phase(native.PHASE_UPDATE, 1)
    st, se = g.stats(), e.stats()
    assert st["cg_fallback"] == 1 and se["cg_fallback"] == 0
    assert st["cg_rel_residual"] < d.spec.eps
    assert 400 < st["cg_iters"] < 2000
    # the fallback solve is the eliminated solve
    assert max_rel(g.solution(), e.solution()) < 1e-12

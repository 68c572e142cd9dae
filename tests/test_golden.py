"""Golden fixtures of the plain FP64 step (tests/golden/*.npz, made by
tests/golden/make_golden.py from runs of the reference program itself).

Two reference runs per case: `jacobi` is the reference program with laspack's
JacobiPrecond handed to its CGIter call -- the solver the device runs -- and
`ssor` is the reference as shipped (SSORPrecond).

CPU: the deck generator still produces the fixtures' decks (fingerprint), and
the C oracle reproduces both reference runs of the 128 x 128 case.

GPU, default solver set-up (FREHD_DECOUPLED_AS_ASSEMBLED): against the Jacobi
runs every field agrees to 1e-9 relative to its max magnitude and the total
water volume to 1e-12, also after the 512 x 512 case's 1000 steps.  Against the SSOR runs the surface, scalar, depth and
cell volumes agree to 1e-9 as well; the face velocities differ by what the two
preconditioners leave in the solution: both solves stop at ||r|| < 1e-12 ||b||,
b carries eta*Z with the datum offset, so eta may differ by ~1e-11 m, and
u - En is proportional to the eta gradient.  The C oracle with Jacobi shows the
same gap to the SSOR runs (3.5e-8 on u of the 512 x 512 case), hence 1e-7.
With FREHD_DECOUPLED_ELIMINATED the device solves a symmetric rearrangement of
the same system; its iterates differ from laspack's at the CG tolerance, which
shows as up to ~7e-9 on u and v (1e-8 bound) and ~3e-11 on eta.
"""
import numpy as np
import pytest

from tests.golden import make_golden as G

_BASE = {"surf": 1e-9, "S": 1e-9, "depth": 1e-9, "cellV": 1e-9}
# The volume bound of a run against a different solver (another preconditioner,
# or the eliminated form) covers the ledgers of two converged solves drifting
# apart: 3.3e-11 and 3.8e-11 relative after the 512 x 512 case's 1000 steps.
TOL = {  # (decoupled-row mode, reference preconditioner) -> field bounds, volume bound
    ("assembled", "jacobi"): ({**_BASE, "uuXP": 1e-9, "vvYP": 1e-9}, 1e-12),
    ("assembled", "ssor"): ({**_BASE, "uuXP": 1e-7, "vvYP": 1e-7}, 1e-10),
    ("eliminated", "jacobi"): ({**_BASE, "uuXP": 1e-8, "vvYP": 1e-8}, 1e-10),
    ("eliminated", "ssor"): ({**_BASE, "uuXP": 1e-7, "vvYP": 1e-7}, 1e-10),
}
_decks: dict = {}


def deck(case):
    if case not in _decks:
        from frehdc_b200 import deck as D
        _decks[case] = D.make_deck(G.CASES[case]())
    return _decks[case]


def rel_err(got_full: np.ndarray, fx: dict, field: str) -> float:
    """Max error at the sampled cells, relative to the field's max magnitude
    (absolute for a field that is zero everywhere)."""
    got = np.asarray(got_full, dtype=np.float64)[fx["idx"]]
    scale = max(abs(fx[field + "_sums"][2]), abs(fx[field + "_sums"][3]))
    err = float(np.max(np.abs(got - fx[field])))
    return err / scale if scale > 0 else err


@pytest.mark.parametrize("case", list(G.CASES))
def test_fixture_deck_fingerprint(case):
    d = deck(case)
    for pc in G.PRECONDS:
        assert str(G.load(case, pc)["fingerprint"]) == G.fingerprint(d)


@pytest.mark.parametrize("precond", G.PRECONDS)
def test_oracle_reproduces_reference_c1(precond):
    from oracle import port
    fx = G.load("c1_128", precond)
    d = deck("c1_128")
    pre = port.PRECOND_JACOBI if precond == "jacobi" else port.PRECOND_SSOR
    o = port.from_deck(d, precond=pre, x0=port.X0_ZERO)
    for tt in range(1, int(fx["steps"]) + 1):
        o.step(tt)
    N = d.spec.nx * d.spec.ny
    for f in G.FIELDS:
        assert rel_err(o.get(f)[:N], fx, f) <= 1e-11, f
    vol = float(np.sum(o.get("cellV")[:N]))
    assert abs(vol - fx["cellV_sums"][0]) <= 1e-12 * abs(fx["cellV_sums"][0])


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["assembled", "eliminated"])
@pytest.mark.parametrize("precond", G.PRECONDS)
@pytest.mark.parametrize("case", list(G.CASES))
def test_device_reproduces_reference(case, precond, mode):
    from frehdc_b200 import native
    if native.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")
    fx = G.load(case, precond)
    d = deck(case)
    dec = native.DECOUPLED_AS_ASSEMBLED if mode == "assembled" else native.DECOUPLED_ELIMINATED
    g = native.domain_from_deck(d, geometry="fine", decoupled=dec)
    tol, vol_tol = TOL[(mode, precond)]
    assert g.run(1, int(fx["steps"])) == 0
    st = g.stats()
    got = g.download(G.FIELDS)
    N = d.spec.nx * d.spec.ny
    errs = {f: rel_err(got[f][:N], fx, f) for f in G.FIELDS}
    for f in G.FIELDS:
        assert errs[f] <= tol[f], (f, errs)
    # total water volume (sum of cellV over the domain) against the reference's
    ref_vol = fx["cellV_sums"][0]
    assert abs(st["volume"] - ref_vol) <= vol_tol * abs(ref_vol), (st["volume"], ref_vol)

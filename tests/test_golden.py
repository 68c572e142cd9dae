"""Golden fixtures of the plain FP64 step (tests/golden/*.npz, made by
tests/golden/make_golden.py from runs of the reference program itself).

CPU: the deck generator still produces the fixtures' decks (fingerprint), and
the C oracle in the reference's own solver set-up (SSOR-PCG from x = 0)
reproduces the reference's final state on the 128 x 128 case.
GPU: the device step reproduces both cases within the whole-run tolerances
(surface and scalar 1e-9, face velocities 3e-9, relative to the field's max).
"""
import numpy as np
import pytest

from tests.golden import make_golden as G

RUN_TOL = {"surf": 1e-9, "S": 1e-9, "uuXP": 3e-9, "vvYP": 3e-9, "depth": 1e-9, "cellV": 1e-9}
_decks: dict = {}


def deck(case):
    if case not in _decks:
        from frehdc_b200 import deck as D
        _decks[case] = D.make_deck(G.CASES[case]())
    return _decks[case]


def rel_err(got_full: np.ndarray, fx: dict, field: str) -> float:
    """Max error at the sampled cells, relative to the field's max magnitude."""
    got = np.asarray(got_full, dtype=np.float64)[fx["idx"]]
    scale = max(abs(fx[field + "_sums"][2]), abs(fx[field + "_sums"][3]), 1e-300)
    return float(np.max(np.abs(got - fx[field]))) / scale


@pytest.mark.parametrize("case", list(G.CASES))
def test_fixture_deck_fingerprint(case):
    fx = G.load(case)
    assert str(fx["fingerprint"]) == G.fingerprint(deck(case))


def test_oracle_reproduces_reference_c1():
    from oracle import port
    fx = G.load("c1_128")
    d = deck("c1_128")
    o = port.from_deck(d, precond=port.PRECOND_SSOR, x0=port.X0_ZERO)
    for tt in range(1, int(fx["steps"]) + 1):
        o.step(tt)
    N = d.spec.nx * d.spec.ny
    for f in G.FIELDS:
        assert rel_err(o.get(f)[:N], fx, f) <= 1e-12, f
    vol = float(np.sum(o.get("cellV")[:N]))
    assert abs(vol - fx["cellV_sums"][0]) <= 1e-12 * abs(fx["cellV_sums"][0])


@pytest.mark.gpu
@pytest.mark.parametrize("case", list(G.CASES))
def test_device_reproduces_reference(case):
    from frehdc_b200 import native
    if native.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")
    fx = G.load(case)
    d = deck(case)
    g = native.domain_from_deck(d, geometry="fine")
    assert g.run(1, int(fx["steps"])) == 0
    st = g.stats()
    got = g.download(G.FIELDS)
    N = d.spec.nx * d.spec.ny
    for f in G.FIELDS:
        assert rel_err(got[f][:N], fx, f) <= RUN_TOL[f], (f, rel_err(got[f][:N], fx, f))
    # the water volume (sum of cellV) against the reference's
    ref_vol = fx["cellV_sums"][0]
    assert abs(st["volume"] - ref_vol) <= 1e-10 * abs(ref_vol)

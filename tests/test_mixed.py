"""Mixed precision (FREHD_PRECISION_MIXED): FP32 inner CG iterations inside
FP64 iterative refinement, against the FP64 solve.

The refinement stops on the same FP64 residual test ||r|| < 1e-12 ||b||, so a
solve agrees with the FP64 solve to the CG tolerance; over a whole run the
surface must stay within 1e-6 m of the FP64 run and the water volume within
1e-10 relative (the targets of the mixed form); the measured errors are far
smaller.
"""
import numpy as np
import pytest

from frehdc_b200 import native
from tests.golden import make_golden as G
from tests.helpers import deck_for, max_rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if native.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")


@pytest.mark.parametrize("decoupled", [native.DECOUPLED_AS_ASSEMBLED, native.DECOUPLED_ELIMINATED])
@pytest.mark.parametrize("name", ["dry40x36", "dry37x29"])
def test_mixed_solve_matches_fp64(name, decoupled, scratch):
    d, _ = deck_for(name, str(scratch))
    a = native.domain_from_deck(d, decoupled=decoupled)
    b = native.domain_from_deck(d, decoupled=decoupled, precision=native.PRECISION_MIXED)
    for g in (a, b):
        g.phase(native.PHASE_EXPLICIT, 1)
        g.phase(native.PHASE_SOLVE, 1)
        g.phase(native.PHASE_UPDATE, 1)
    sa, sb = a.stats(), b.stats()
    assert sb["cg_fallback"] == 0
    assert sb["cg_rel_residual"] < d.spec.eps
    assert max_rel(b.solution(), a.solution()) < 1e-10


def test_mixed_run_error_c1():
    from frehdc_b200 import deck as D
    d = D.make_deck(G.c1_spec())
    steps = 200
    a = native.domain_from_deck(d)
    b = native.domain_from_deck(d, precision=native.PRECISION_MIXED)
    assert a.run(1, steps) == 0 and b.run(1, steps) == 0
    N = d.spec.nx * d.spec.ny
    fa = a.download(["surf", "uuXP", "vvYP", "S"])
    fb = b.download(["surf", "uuXP", "vvYP", "S"])
    eta_err = float(np.max(np.abs(fb["surf"][:N] - fa["surf"][:N])))
    assert eta_err <= 1e-6, eta_err
    for f in ("uuXP", "vvYP", "S"):
        assert max_rel(fb[f][:N], fa[f][:N]) < 1e-6, f
    va, vb = a.stats()["volume"], b.stats()["volume"]
    assert abs(vb - va) <= 1e-10 * abs(va)
    assert b.stats()["cg_fallback"] == 0


def test_mixed_in_batch(scratch):
    """A mixed-precision domain in a batch gives its single-domain result."""
    d, _ = deck_for("dry40x36", str(scratch))
    g = native.domain_from_deck(d, precision=native.PRECISION_MIXED)
    ref = native.domain_from_deck(d, precision=native.PRECISION_MIXED)
    bt = native.Batch(8 << 30, 1)
    slot = bt.admit(g, 1)
    for _ in range(8):
        bt.step()
    bt.release(slot)
    assert ref.run(1, 8) == 0
    fa, fb = g.download(["surf", "uuXP"]), ref.download(["surf", "uuXP"])
    assert np.array_equal(fa["surf"], fb["surf"]) and np.array_equal(fa["uuXP"], fb["uuXP"])
    bt.close()

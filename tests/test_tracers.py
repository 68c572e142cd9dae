"""Several scalars per domain (frehd_config.nscalar): S and up to three passive
tracers, each transported like the reference's S.

The reference carries one scalar and its hydrodynamics do not read it while it
stays inside [0, 100] (scalar.c:403-415), so k scalars are k reference runs that
differ only in the initial S.  GPU: a domain with tracers keeps the single-scalar
run's hydrodynamics and S bit for bit; tracer t equals, bit for bit, the
single-scalar run whose S starts from tracer t's field, and that run matches the
C oracle to the whole-run tolerance; this holds for upwind and TVD advection,
with inflow cells, in a batch, and for the tracer output files.
"""
import os

import numpy as np
import pytest

from frehdc_b200 import deck as D
from frehdc_b200 import native
from tests.helpers import SPECS, max_rel, mismatches

pytestmark = pytest.mark.gpu
HYDRO = ["surf", "uuXP", "vvYP", "depth", "cellV", "CDXP", "CDYP", "ind", "S"]


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if native.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")


def _deck(name: str, n_scalars: int = 3):
    return D.make_deck(SPECS[name].replace(n_scalars=n_scalars), with_tables=False)


def _single_runs(deck, steps):
    """The single-scalar run of each scalar's initial field (S first)."""
    out = []
    for field in [deck.S0] + list(deck.tracers):
        g = native.domain_from_deck(D.with_scalar(deck, field))
        assert g.run(1, steps) == 0
        out.append((g.download(HYDRO), g.stats()))
    return out


@pytest.mark.parametrize("name", ["dry40x36", "tvd44x36", "inflow36x30"])
def test_tracers_equal_single_scalar_runs(name):
    deck = _deck(name)
    assert len(deck.tracers) == 2 and D.config_dict(deck)["nscalar"] == 3
    steps = 20
    g = native.domain_from_deck(deck)
    assert g.run(1, steps) == 0
    got = g.download(HYDRO)
    single = _single_runs(deck, steps)
    # S and the hydrodynamics are those of the run without tracers
    assert mismatches(got, single[0][0], HYDRO) == []
    assert g.stats()["volume"] == single[0][1]["volume"]
    for t in (1, 2):
        tr = g.download_scalar(t)
        assert np.array_equal(tr, single[t][0]["S"]), t
        assert not np.array_equal(tr, got["S"])     # a different field, really transported
    assert np.array_equal(g.download_scalar(0), got["S"])


def test_tracer_matches_oracle_run():
    from oracle import port
    deck = _deck("inflow36x30", n_scalars=2)
    steps = SPECS["inflow36x30"].steps
    g = native.domain_from_deck(deck)
    assert g.run(1, steps) == 0
    o = port.from_deck(D.with_scalar(deck, deck.tracers[0]), precond=port.PRECOND_SSOR,
                       x0=port.X0_ZERO)
    for tt in range(1, steps + 1):
        o.step(tt)
    assert max_rel(g.download_scalar(1), o.get("S")) <= 1e-9
    assert max_rel(g.download(["surf"])["surf"], o.get("surf")) <= 1e-9


def test_tracers_in_a_batch_equal_alone():
    names = ["dry40x36", "tvd44x36"]
    decks = {n: _deck(n, n_scalars=2 + k) for k, n in enumerate(names)}
    steps = 10
    alone = {}
    for n, deck in decks.items():
        g = native.domain_from_deck(deck)
        assert g.run(1, steps) == 0
        alone[n] = [g.download_scalar(s) for s in range(1 + len(deck.tracers))]
    b = native.Batch(8 << 30, 1)
    doms = {n: native.domain_from_deck(deck) for n, deck in decks.items()}
    slots = {n: b.admit(g, 1) for n, g in doms.items()}
    for _ in range(steps):
        b.step()
    for n, g in doms.items():
        b.release(slots[n])
        for s, ref in enumerate(alone[n]):
            assert np.array_equal(g.download_scalar(s), ref), (n, s)
    b.close()


def test_tracer_output_files(tmp_path):
    from tests.test_output import c_fixed4
    deck = _deck("dry40x36", n_scalars=3)
    g = native.domain_from_deck(deck)
    assert g.run(1, 5) == 0
    g.write_output(str(tmp_path) + "/", 5, native.OUT_SCALAR)
    N = deck.nx * deck.ny
    for s, name in enumerate(["scalar", "scalar1", "scalar2"]):
        got = open(os.path.join(tmp_path, f"{name}_5.dat"), "rb").read()
        assert got == c_fixed4(g.download_scalar(s)[:N]), name


def test_scalar_index_checked():
    g = native.domain_from_deck(_deck("dry40x36", n_scalars=2))
    with pytest.raises(native.FrehdError):
        g.download_scalar(2)
    with pytest.raises(native.FrehdError):
        g.upload_scalar(-1, np.zeros(g.T))

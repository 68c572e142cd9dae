"""Why tracers can be checked as separate reference runs (CPU, C oracle).

The reference's hydrodynamics do not read S while it stays inside [0, 100]
(the singularity branch of updateScalarSub, subgrid.c:1700-1712, is the only
place that writes the surface or depth from S): two oracle runs that differ
only in the initial S end with the same surface, velocities and volumes, bit
for bit.  The generated tracer fields are different plumes inside [0, 1].
"""
import numpy as np
import pytest

from frehdc_b200 import deck as D
from oracle import port


def test_tracer_fields_are_distinct_plumes():
    deck = D.make_deck(D.DeckSpec(nx=24, ny=20, steps=3, seed=4, n_scalars=4))
    assert len(deck.tracers) == 3
    fields = [deck.S0] + deck.tracers
    for k, f in enumerate(fields):
        assert f.shape == (deck.N,) and f.min() >= 0 and f.max() <= 1.0
        for g in fields[k + 1:]:
            assert not np.array_equal(f, g)
    assert D.config_dict(deck)["nscalar"] == 4
    assert D.config_dict(D.with_scalar(deck, deck.tracers[0]))["nscalar"] == 1
    assert D.make_deck(D.DeckSpec(nx=24, ny=20, steps=3, seed=4)).tracers == []


@pytest.mark.parametrize("extra", [dict(), dict(scalar_adv=2),
                                   dict(inflow_cells=(3, 5, 2, 4), inflow_q=2.0, inflow_s=30.0)],
                         ids=["upwind", "tvd", "inflow"])
def test_hydrodynamics_do_not_read_the_scalar(extra):
    deck = D.make_deck(D.DeckSpec(nx=20, ny=16, steps=8, seed=6, dry_frac=0.3, n_scalars=2,
                                  **extra), with_tables=True)
    runs = []
    for field in (deck.S0, deck.tracers[0]):
        o = port.from_deck(D.with_scalar(deck, field), precond=port.PRECOND_JACOBI,
                           x0=port.X0_ZERO)
        for tt in range(1, 9):
            o.step(tt)
        runs.append({n: o.get(n).copy() for n in ("surf", "uuXP", "vvYP", "cellV", "S")})
    for n in ("surf", "uuXP", "vvYP", "cellV"):
        assert np.array_equal(runs[0][n], runs[1][n]), n
    assert not np.array_equal(runs[0]["S"], runs[1]["S"])

"""The per-cell level-value cache of the fine geometry (needs a B200).

With fine bottoms, k_update_geo keeps each cell's values of the last even and
the last odd level it evaluated and reuses them while the cell's surface stays
between the same two levels.  A level's values depend on the fine bottoms
alone, so a run through the cache must give, at every step, the doubles of a
run that reads the host-built tables (no cache).  The decks here push the
surface through several levels per step (a fast, large tide; a bore from an
injected velocity), so entries are replaced in most steps, in single-domain
runs and in a batch where block halos read other blocks' entries.
"""
import numpy as np
import pytest

from frehdc_b200 import deck as D
from frehdc_b200 import native
from tests.helpers import mismatches

pytestmark = pytest.mark.gpu

FIELDS = ["surf", "uuXP", "vvYP", "S", "depth", "V", "Z", "Nx", "Oy", "Vx", "Vy", "Zx", "Zy", "ind"]
FAST_TIDE = dict(nx=96, ny=72, dx=10.0, dt=1.0, tide_amp=1.2, tide_period=900.0, dry_frac=0.35,
                 roughness=0.3, seed=21)
BORE = dict(nx=80, ny=64, dx=10.0, dt=1.0, dry_frac=0.25, seed=4, u0_block=(10, 30, 20, 44, 2.0))


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if native.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")


@pytest.mark.parametrize("kw", [FAST_TIDE, BORE], ids=["fast_tide", "bore"])
def test_cache_equals_tables_every_step(kw):
    steps = 40
    d = D.make_deck(D.DeckSpec(steps=steps + 5, **kw), with_tables=True)
    gf = native.domain_from_deck(d, geometry="fine")
    gt = native.domain_from_deck(d, geometry="tables")
    moved = 0
    prev = gf.download(["ind"])["ind"]
    for t in range(1, steps + 1):
        assert gf.run(t, 1) == 0 and gt.run(t, 1) == 0
        a, b = gf.download(FIELDS), gt.download(FIELDS)
        assert mismatches(a, b, FIELDS) == [], f"step {t}"
        moved += int(np.count_nonzero(a["ind"] != prev))
        prev = a["ind"]
    # the level index of a good share of the cells moved: entries were replaced
    assert moved > steps * kw["nx"] * kw["ny"] // 20
    gf.close()
    gt.close()


def test_cache_in_batch_equals_tables():
    """Two fast-tide domains and a bore batched together (32 x 8 stencil tiles of
    several domains per launch, whose halos read other blocks' entries): the
    final state equals the table-geometry runs stepped alone."""
    steps = 25
    decks = [D.make_deck(D.DeckSpec(steps=steps + 5, **kw), with_tables=True)
             for kw in (FAST_TIDE, dict(FAST_TIDE, seed=22, nx=64, ny=100), BORE)]
    fine = [native.domain_from_deck(dk, geometry="fine") for dk in decks]
    # CTA groups at one cell per CTA: every solve on the CTAs its single-domain
    # run uses, so the batch reproduces those runs bit for bit
    b = native.Batch(8 << 30, 1.0)
    b.set_cg_packing(native.BATCH_CTA_GROUPS)
    slots = [b.admit(g, 1) for g in fine]
    for _ in range(steps):
        b.step()
    b.sync()
    for sl in slots:
        b.release(sl)
    b.close()
    for g, dk in zip(fine, decks):
        h = native.domain_from_deck(dk, geometry="tables")
        assert h.run(1, steps) == 0
        assert mismatches(g.download(FIELDS), h.download(FIELDS), FIELDS) == []
        g.close()
        h.close()

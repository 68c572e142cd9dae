"""The autotuner (CPU): its capacity pre-check follows the batch's CTA rule, and
its two-stage search runs against a fake device."""
from frehdc_b200 import autotune


def test_ctas_needed_rule():
    # two 1024 x 1024 domains and three small ones at 262144 cells per CTA:
    # groups of 4 CTAs each, the small domains share one CTA
    sizes = [(1024, 1024), (1024, 1024), (64, 64), (64, 128), (96, 96)]
    assert autotune.ctas_needed(sizes, 262144.0) == 4 + 4 + 1
    # a group never exceeds the domain's CG tiles (128 x 16) nor the capacity
    assert autotune.ctas_needed([(256, 32)], 1.0) == 4
    assert autotune.ctas_needed([(4096, 4096)], 1.0, capacity=148) == 148
    # only single-CTA domains: one CTA
    assert autotune.ctas_needed([(64, 64)] * 300, 65536.0) == 1


class _Deck:
    def __init__(self, nx, ny):
        self.nx, self.ny = nx, ny


class _Dom:
    closed = 0

    def close(self):
        _Dom.closed += 1


def test_tune_two_stages(monkeypatch):
    """The search on a fake device: candidates whose CG would exceed the CTA
    capacity are never timed; the stencil stage runs at the best solve setting
    only, and the overall fastest wins; every domain built is closed."""
    timed = []

    def fake_time(doms, cpc, steps, warmup, budget, precision, eps, device, packing, tpb=4):
        timed.append((packing, cpc, eps, tpb))
        ms = 60.0 if packing == autotune.native.BATCH_TILE_LIST else 50.0 + abs(cpc - 393216.0) / 1e5
        ms += {1e-4: 0.0, 1e-5: 3.0, 1e-6: 2.0}[eps] + {1: -0.2, 2: 0.5, 4: 0.0, 8: 0.3}[tpb]
        return ms * steps

    monkeypatch.setattr(autotune, "time_batch", fake_time)
    monkeypatch.setattr(autotune.native.Batch, "capacity", staticmethod(lambda device=0: 148))
    monkeypatch.setattr(autotune.native, "domain_from_deck", lambda dk, device=0: _Dom())
    decks = [_Deck(1024, 1024)] * 40 + [_Deck(64, 64)] * 10
    _Dom.closed = 0
    out = autotune.tune(decks, 1 << 30, autotune.native.PRECISION_MIXED)
    # 40 domains of 1 M cells need 40 * ceil(1M / cpc) CTAs: only cpc >= 2^20 / 3 fit
    fits = [c for c in autotune.CELLS_PER_CTA
            if autotune.ctas_needed([(d.nx, d.ny) for d in decks], c) <= 148]
    assert {t[1] for t in timed if t[0] == autotune.native.BATCH_CTA_GROUPS} == set(fits)
    assert all(c >= (1 << 20) / 3 for c in fits)
    best = out["best"]
    assert (best["packing"], best["cells_per_cta"], best["eps_inner"], best["tiles_per_block"]) == \
        ("cta_groups", 393216.0, 1e-4, 1)
    stencil = [t for t in timed if t[3] != 4]
    assert sorted(t[3] for t in stencil) == [1, 2, 8]
    assert all(t[1:3] == (393216.0, 1e-4) for t in stencil)
    assert _Dom.closed == len(decks)

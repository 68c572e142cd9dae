"""The autotuner's capacity pre-check follows the batch's CTA rule (CPU)."""
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

"""Autotuner of the batched form: picks the CG packing granularity
(cells_per_cta: how many cells of a domain one CTA of its CG carries, hence how
many CTAs each domain's solve gets and how the single-CTA domains are packed)
and, for the mixed-precision form, the inner FP32 tolerance, by timing a few
batch steps of the actual mix with each candidate.

A domain's CG CTA count depends on its own size and cells_per_cta only, so the
tuned value must be fixed before serving starts for results to stay
independent of the mix; tune once on a representative mix, then serve.
"""
from __future__ import annotations

import itertools

from . import native

CELLS_PER_CTA = (8192.0, 16384.0, 32768.0, 65536.0, 131072.0)
EPS_INNER = (1e-4, 1e-5, 1e-6)


def time_batch(decks, cells_per_cta: float, steps: int, warmup: int, budget: int,
               precision: int = native.PRECISION_FP64, eps_inner: float = 1e-5,
               device: int = 0) -> float:
    """Device milliseconds of `steps` batch steps of the decks' domains, or None
    when the mix does not fit the batch (memory budget or CG CTA capacity)."""
    import torch
    doms = [native.domain_from_deck(dk, device=device, precision=precision, eps_inner=eps_inner)
            for dk in decks]
    b = native.Batch(budget, cells_per_cta, device)
    try:
        for g in doms:
            if b.try_admit(g, 1) is None:
                return None
        for _ in range(warmup):
            b.step()
        b.sync()
        st = torch.cuda.ExternalStream(b.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            b.step()
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1)
    finally:
        for sl in list(b.members):
            b.release(sl)
        b.close()
        for g in doms:
            g.close()


def tune(decks, budget: int, precision: int = native.PRECISION_FP64, steps: int = 4,
         warmup: int = 2, cells_candidates=CELLS_PER_CTA, eps_candidates=EPS_INNER,
         device: int = 0) -> dict:
    """The fastest (cells_per_cta, eps_inner) on this mix, and every timing."""
    eps_list = eps_candidates if precision == native.PRECISION_MIXED else (1e-5,)
    results = []
    for cpc, ein in itertools.product(cells_candidates, eps_list):
        ms = time_batch(decks, cpc, steps, warmup, budget, precision, ein, device)
        if ms is None:  # the mix does not fit with this granularity
            continue
        results.append({"cells_per_cta": cpc, "eps_inner": ein, "ms_per_step": ms / steps})
    if not results:
        raise RuntimeError("no candidate packing fits the mix")
    best = min(results, key=lambda r: r["ms_per_step"])
    return {"best": best, "tried": results}

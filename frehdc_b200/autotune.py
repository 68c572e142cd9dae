"""Autotuner of the batched form: picks the packing of the batched CG -- the
tile list over all CTAs, or CTA groups with a granularity cells_per_cta (how
many cells of a domain one CTA of its CG carries, hence how many CTAs each
domain's solve gets and how the single-CTA domains are packed) -- and, for the
mixed-precision form, the inner FP32 tolerance, by timing a few batch steps of
the actual mix with each candidate; then, at the chosen solve, the number of
32 x 8 stencil tiles each block of the batched stencil kernels runs.

In either packing a domain's arithmetic depends on the domain alone (its own
tile order; or its own size and cells_per_cta), so the tuned choice must be
fixed before serving starts for results to stay independent of the mix; tune
once on a representative mix, then serve.
"""
from __future__ import annotations

import itertools
import math

from . import native

CELLS_PER_CTA = (8192.0, 16384.0, 32768.0, 65536.0, 131072.0, 196608.0, 229376.0, 262144.0,
                 294912.0, 327680.0, 393216.0, 524288.0)
EPS_INNER = (1e-4, 1e-5, 1e-6)
TILES_PER_BLOCK = (1, 2, 4, 8)
CTX, CTY = 128, 16   # CG tile of k_cg1


def ctas_needed(sizes, cells_per_cta: float, capacity: int = 148) -> int:
    """CTAs of the batched CG for domains of these (nx, ny): each domain's
    group is ceil(cells / cells_per_cta) CTAs (at least 1, at most its tile
    count), multi-CTA groups get CTAs of their own and the single-CTA domains
    share the rest (batch.cu, group_size / ctas_needed)."""
    dedicated, singles = 0, 0
    for nx, ny in sizes:
        ntiles = ((nx + CTX - 1) // CTX) * ((ny + CTY - 1) // CTY)
        g = max(1, min(int(math.ceil(nx * ny / cells_per_cta)), ntiles, capacity))
        if g > 1:
            dedicated += g
        else:
            singles += 1
    return dedicated + (1 if singles else 0)


def time_batch(doms, cells_per_cta: float, steps: int, warmup: int, budget: int,
               precision: int = native.PRECISION_FP64, eps_inner: float = 1e-5,
               device: int = 0, packing: int = native.BATCH_CTA_GROUPS,
               tiles_per_block: int = 4) -> float:
    """Device milliseconds of `steps` batch steps of the domains (set to the
    given precision; their state advances), or None when the mix does not fit
    the batch (memory budget or CG CTA capacity)."""
    import torch
    if precision != native.PRECISION_FP64:
        for g in doms:
            g.set_precision(precision, eps_inner)
    b = native.Batch(budget, cells_per_cta, device)
    b.set_cg_packing(packing)
    b.set_stencil_tiles(tiles_per_block)
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


def tune(decks, budget: int, precision: int = native.PRECISION_FP64, steps: int = 4,
         warmup: int = 2, cells_candidates=CELLS_PER_CTA, eps_candidates=EPS_INNER,
         device: int = 0) -> dict:
    """The fastest (packing, cells_per_cta, eps_inner) on this mix, then the
    fastest stencil tiles per block with it, and every timing.  The tile-list
    packing takes any mix; CTA-group granularities whose CG would need more
    co-resident CTAs than the device holds are skipped before any domain is
    built.  The domains are built once and stepped by every candidate in turn."""
    eps_list = eps_candidates if precision == native.PRECISION_MIXED else (1e-5,)
    capacity = native.Batch.capacity(device)
    sizes = [(dk.nx, dk.ny) for dk in decks]
    fits = [c for c in cells_candidates if ctas_needed(sizes, c, capacity) <= capacity]
    cands = [("tile_list", 0.0)] + [("cta_groups", c) for c in fits]
    packings = {"tile_list": native.BATCH_TILE_LIST, "cta_groups": native.BATCH_CTA_GROUPS}
    results = []
    doms = [native.domain_from_deck(dk, device=device) for dk in decks]
    try:
        for (pk, cpc), ein in itertools.product(cands, eps_list):
            ms = time_batch(doms, cpc if cpc > 0 else 1.0, steps, warmup, budget, precision, ein,
                            device, packings[pk])
            if ms is None:  # the mix does not fit with this granularity
                continue
            results.append({"packing": pk, "cells_per_cta": cpc, "eps_inner": ein,
                            "tiles_per_block": 4, "ms_per_step": ms / steps})
        if not results:
            raise RuntimeError("no candidate packing fits the mix")
        best = min(results, key=lambda r: r["ms_per_step"])
        for tpb in TILES_PER_BLOCK:
            if tpb == best["tiles_per_block"]:
                continue
            ms = time_batch(doms, best["cells_per_cta"] if best["cells_per_cta"] > 0 else 1.0,
                            steps, warmup, budget, precision, best["eps_inner"], device,
                            packings[best["packing"]], tpb)
            if ms is not None:
                results.append({**best, "tiles_per_block": tpb, "ms_per_step": ms / steps})
    finally:
        for g in doms:
            g.close()
    best = min(results, key=lambda r: r["ms_per_step"])
    return {"best": best, "tried": results}

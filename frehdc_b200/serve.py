"""Served form: a request loop over a resident batch (continuous batching).

Requests (a deck and a step count) arrive over time.  The loop admits every
arrived request whose domain fits the batch's device-memory budget and the
batched CG's CTA capacity, advances all admitted domains one step at a time
(frehd_batch_step: one launch per sub-step for the whole batch, replayed from a
CUDA graph), releases each domain as soon as it has run its steps, and admits
waiting requests as room frees up.  A request's result does not depend on the
other requests it shared the batch with (the batch engine's guarantee), so
admission order only changes latency.

Latency is arrival -> result (the domain released, its state readable), wall
clock; throughput counts cell-steps completed per second of serving.
"""
from __future__ import annotations

import dataclasses
import time
from collections import deque

import numpy as np

from . import native


@dataclasses.dataclass
class Request:
    rid: int
    deck: object            # frehdc_b200.deck.Deck
    steps: int
    arrival: float          # seconds after the start of serving
    admitted: float = -1.0
    done: float = -1.0
    slot: int = -1
    taken: int = 0
    domain: object = None
    cells: int = 0
    status: int = 0


def poisson_arrivals(n: int, rate: float, seed: int) -> np.ndarray:
    """Arrival times of n requests with exponential gaps of mean 1/rate."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


def serve(requests: list[Request], budget_bytes: int, cells_per_cta: float, device: int = 0,
          build=None, on_done=None, clock=time.perf_counter) -> dict:
    """Serve the requests; returns latency percentiles (and every request's
    latency, in completion order) and throughput.

    build(req) -> native.Domain sets up a request's domain (default: from its
    deck, fine geometry); on_done(req) is called right after a release (the
    domain's state can be downloaded there)."""
    if build is None:
        def build(req):
            return native.domain_from_deck(req.deck, device=device, geometry="fine")
    batch = native.Batch(budget_bytes, cells_per_cta, device)
    pending = deque(sorted(requests, key=lambda r: r.arrival))
    waiting: deque = deque()
    active: dict[int, Request] = {}
    finished: list[Request] = []
    cell_steps = 0
    max_active = 0
    t0 = clock()
    try:
        while pending or waiting or active:
            now = clock() - t0
            while pending and pending[0].arrival <= now:
                waiting.append(pending.popleft())
            # admit in arrival order while there is room
            while waiting:
                req = waiting[0]
                if req.domain is None:
                    req.domain = build(req)
                    req.cells = req.domain.nx * req.domain.ny
                slot = batch.try_admit(req.domain, 1)
                if slot is None:
                    if not active:
                        raise RuntimeError(f"request {req.rid} does not fit an empty batch")
                    break
                waiting.popleft()
                req.slot = slot
                req.admitted = clock() - t0
                active[slot] = req
            max_active = max(max_active, len(active))
            if not active:
                if pending:  # idle until the next arrival
                    wait = pending[0].arrival - (clock() - t0)
                    if wait > 0:
                        time.sleep(min(wait, 0.01))
                continue
            batch.step()
            done_now = []
            for slot, req in active.items():
                req.taken += 1
                cell_steps += req.cells
                if req.taken >= req.steps:
                    done_now.append(slot)
            for slot in done_now:  # release waits for the batch's queued work
                req = active.pop(slot)
                batch.release(slot)
                req.done = clock() - t0
                req.status = req.domain.stats()["status"]
                if on_done is not None:
                    on_done(req)
                req.domain.close()
                req.domain = None
                finished.append(req)
        batch.sync()
        wall = clock() - t0
    finally:
        batch.close()
    lat = np.array([r.done - r.arrival for r in finished])
    return {"requests": len(finished), "wall_s": wall, "cell_steps": cell_steps,
            "cell_steps_per_s": cell_steps / wall if wall > 0 else 0.0,
            "p50_s": float(np.percentile(lat, 50)) if lat.size else 0.0,
            "p99_s": float(np.percentile(lat, 99)) if lat.size else 0.0,
            "latencies_s": lat.tolist(),
            "max_active": max_active, "failed": sum(1 for r in finished if r.status != 0)}

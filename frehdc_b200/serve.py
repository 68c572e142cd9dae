"""Served form: requests over a resident batch (continuous batching).

Requests (a deck and a step count) arrive over time.  The stepping loop is the
library's native server (frehd_server_*, csrc/server.cu): one host thread that
admits every submitted domain that fits the batch's device-memory budget and
the batched CG's CTA capacity, advances all admitted domains one step at a time
(frehd_batch_step: one launch per sub-step for the whole batch, replayed from a
CUDA graph), and releases each domain as soon as it has run its steps, so that
waiting requests are admitted as room frees up.  Here a submitter thread
prepares each request's domain at its arrival time (deck upload and device
initialisation, on the domain's own stream, while the server steps the others)
and submits it; the calling thread collects the completions.  A request's
result does not depend on the other requests it shared the batch with (the
batch engine's guarantee), so admission order only changes latency.

Latency is arrival -> result (the domain released, its state readable), on the
server's monotonic clock; throughput counts cell-steps completed per second of
serving.
"""
from __future__ import annotations

import dataclasses
import time

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
          build=None, on_done=None) -> dict:
    """Serve the requests; returns latency percentiles (and every request's
    latency, in completion order) and throughput.

    build(req) -> native.Domain sets up a request's domain (default: from its
    deck, fine geometry); on_done(req) is called right after the request
    completes (the domain's state can be downloaded there)."""
    import threading

    if build is None:
        def build(req):
            return native.domain_from_deck(req.deck, device=device, geometry="fine")
    server = native.Server(budget_bytes, cells_per_cta, device)
    order = sorted(requests, key=lambda r: r.arrival)
    by_ticket: dict[int, Request] = {}
    lock = threading.Lock()
    errors: list = []
    t0 = server.clock()

    def submitter():
        try:
            for req in order:
                wait = t0 + req.arrival - server.clock()
                if wait > 0:
                    time.sleep(wait)
                req.domain = build(req)
                req.cells = req.domain.nx * req.domain.ny
                with lock:
                    by_ticket[server.submit(req.domain, req.steps)] = req
        except Exception as e:  # reported by the collecting thread
            errors.append(e)

    th = threading.Thread(target=submitter, daemon=True)
    th.start()
    finished: list[Request] = []
    try:
        while len(finished) < len(order):
            if errors:
                raise errors[0]
            for r in server.poll(timeout_ms=20):
                with lock:
                    req = by_ticket.pop(r["ticket"])
                req.admitted = r["t_admit"] - t0
                req.done = r["t_done"] - t0
                req.taken = r["steps"]
                req.status = r["status"]
                if req.status == 4 and req.taken == 0:
                    raise RuntimeError(f"request {req.rid} does not fit an empty batch")
                if on_done is not None:
                    on_done(req)
                req.domain.close()
                req.domain = None
                finished.append(req)
        info = server.info()
        wall = max(r.done for r in finished) if finished else 0.0
    finally:
        th.join(timeout=60)
        server.close()
    lat = np.array([r.done - r.arrival for r in finished])
    cell_steps = sum(r.cells * r.taken for r in finished)
    return {"requests": len(finished), "wall_s": wall, "cell_steps": cell_steps,
            "cell_steps_per_s": cell_steps / wall if wall > 0 else 0.0,
            "p50_s": float(np.percentile(lat, 50)) if lat.size else 0.0,
            "p99_s": float(np.percentile(lat, 99)) if lat.size else 0.0,
            "latencies_s": lat.tolist(),
            "max_active": info["max_active"], "batch_steps": info["batch_steps"],
            "failed": sum(1 for r in finished if r.status != 0)}

"""Sharding of independent domains and requests across GPUs.

One process per GPU (torchrun).  Domains of a batch mix and requests of a
served stream are independent -- the reference runs each basin as its own
program (FREHD.c:66-118) -- so they are partitioned across ranks with no
collective on the data path: every rank computes the same deterministic
assignment from the same inputs, steps only its share on its own GPU, and
the ranks meet once at the end for a host-side gather of metrics
(torch.distributed object collectives; gloo on CPU, NCCL on GPUs).

A domain's result does not depend on which rank or batch steps it (the batch
engine's guarantee for a fixed cells_per_cta), so sharding changes only
throughput and latency.
"""
from __future__ import annotations

import heapq


def balance(costs, n_ranks: int) -> list[list[int]]:
    """Static partition of items with the given costs over n_ranks
    (longest-processing-time first: items by decreasing cost, each to the least
    loaded rank, ties to the lower rank and the lower index).  Deterministic;
    the heaviest rank exceeds the lightest by at most the largest cost."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(n_ranks)]
    parts: list[list[int]] = [[] for _ in range(n_ranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(p) for p in parts]


def assign_stream(arrivals, costs, n_ranks: int) -> list[int]:
    """Online assignment of a request stream: in arrival order, each request
    goes to the rank with the least work assigned so far (ties to the lower
    rank).  Every rank evaluates the same function of the same stream, so the
    ranks agree without exchanging messages.  Returns the rank of each request."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    order = sorted(range(len(arrivals)), key=lambda i: (float(arrivals[i]), i))
    heap = [(0.0, r) for r in range(n_ranks)]
    owner = [0] * len(arrivals)
    for i in order:
        load, r = heapq.heappop(heap)
        owner[i] = r
        heapq.heappush(heap, (load + float(costs[i]), r))
    return owner


def gather(obj, world_size: int):
    """Every rank's `obj` on every rank (a host-side gather; no device data)."""
    if world_size == 1:
        return [obj]
    import torch.distributed as dist
    out = [None] * world_size
    dist.all_gather_object(out, obj)
    return out


def broadcast(obj, world_size: int, src: int = 0):
    """Rank src's `obj` on every rank."""
    if world_size == 1:
        return obj
    import torch.distributed as dist
    box = [obj]
    dist.broadcast_object_list(box, src=src)
    return box[0]


def merge_served(parts: list[dict]) -> dict:
    """Whole-job serving metrics from every rank's serve() result: cell-steps
    over the slowest rank's wall time, latency percentiles over all requests."""
    import numpy as np
    lat = np.concatenate([np.asarray(p["latencies_s"], dtype=np.float64) for p in parts])
    wall = max(p["wall_s"] for p in parts)
    cs = sum(p["cell_steps"] for p in parts)
    return {"requests": int(sum(p["requests"] for p in parts)), "wall_s": wall, "cell_steps": cs,
            "cell_steps_per_s": cs / wall if wall > 0 else 0.0,
            "p50_s": float(np.percentile(lat, 50)) if lat.size else 0.0,
            "p99_s": float(np.percentile(lat, 99)) if lat.size else 0.0,
            "max_active": max(p["max_active"] for p in parts),
            "failed": int(sum(p["failed"] for p in parts)),
            "per_rank": [{"requests": p["requests"], "cell_steps": p["cell_steps"],
                          "wall_s": p["wall_s"]} for p in parts]}

"""Sharding of independent domains and requests across ranks (one process per
GPU; here gloo ranks on the CPU, each stepping its share with the C oracle).

The partition is deterministic and balanced, every item lands on exactly one
rank, a sharded run returns for each domain the same doubles as an unsharded
run, and a rank that fails makes the others' final gather raise instead of
hang.
"""
import multiprocessing as mp
import os
import pickle
import socket

import numpy as np
import pytest

from frehdc_b200 import shard


def test_balance_partitions_every_item_once():
    rng = np.random.default_rng(0)
    costs = rng.lognormal(10, 1, size=101)
    for n in (1, 2, 3, 8):
        parts = shard.balance(costs, n)
        assert len(parts) == n
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [costs[p].sum() for p in parts]
        assert max(loads) - min(loads) <= costs.max() + 1e-6
        assert parts == shard.balance(costs, n)  # deterministic


def test_balance_more_ranks_than_items():
    parts = shard.balance([5.0, 1.0], 4)
    assert parts == [[0], [1], [], []]


def test_assign_stream_is_least_loaded_in_arrival_order():
    arrivals = [0.3, 0.1, 0.2, 0.4]
    costs = [10.0, 1.0, 1.0, 1.0]
    owner = shard.assign_stream(arrivals, costs, 2)
    # arrival order 1, 2, 0, 3: 1->r0, 2->r1, 0->r0 (tie: lower rank), 3->r1
    assert owner == [0, 0, 1, 1]
    with pytest.raises(ValueError):
        shard.assign_stream(arrivals, costs, 0)


def test_merge_served_takes_slowest_rank_and_all_latencies():
    a = {"requests": 2, "wall_s": 2.0, "cell_steps": 100, "latencies_s": [1.0, 3.0],
         "max_active": 2, "failed": 0}
    b = {"requests": 1, "wall_s": 4.0, "cell_steps": 300, "latencies_s": [2.0],
         "max_active": 1, "failed": 1}
    m = shard.merge_served([a, b])
    assert m["requests"] == 3 and m["cell_steps"] == 400 and m["wall_s"] == 4.0
    assert m["cell_steps_per_s"] == 100.0
    assert m["p50_s"] == 2.0 and m["failed"] == 1 and m["max_active"] == 2


# ------------------------------------------------------------ gloo, world_size 2
SPECS_KW = [dict(nx=16, ny=12, steps=3, seed=11), dict(nx=24, ny=16, steps=3, seed=12),
            dict(nx=16, ny=16, steps=3, seed=13, dry_frac=0.3), dict(nx=20, ny=12, steps=3, seed=14),
            dict(nx=12, ny=20, steps=3, seed=15)]
STEPS = 3


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run_domain(k: int) -> np.ndarray:
    from frehdc_b200 import deck as D
    from oracle import port
    d = D.make_deck(D.DeckSpec(**SPECS_KW[k]), with_tables=True)
    o = port.from_deck(d, precond=port.PRECOND_JACOBI, x0=port.X0_ZERO)
    for tt in range(1, STEPS + 1):
        o.step(tt)
    return o.get("surf").copy()


def _rank_main(rank: int, ws: int, port_: int, out_dir: str, fail_rank: int):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port_))
    result = {}
    try:
        dist.init_process_group("gloo", rank=rank, world_size=ws,
                                timeout=datetime.timedelta(seconds=30))
        from frehdc_b200 import deck as D
        cells = [D.DeckSpec(**kw).nx * D.DeckSpec(**kw).ny for kw in SPECS_KW]
        mine = shard.balance(cells, ws)[rank]
        if rank == fail_rank:
            raise RuntimeError("injected failure before the gather")
        local = {k: _run_domain(k) for k in mine}
        parts = shard.gather({"rank": rank, "surf": local}, ws)
        result = {"ok": True, "parts": parts}
    except Exception as e:  # recorded for the parent; the rank then exits
        result = {"ok": False, "error": f"{type(e).__name__}: {e}"}
    with open(os.path.join(out_dir, f"rank{rank}.pkl"), "wb") as f:
        pickle.dump(result, f)
    try:
        dist.destroy_process_group()
    except Exception:
        pass


def _launch(tmp_path, fail_rank: int) -> list[dict]:
    ctx = mp.get_context("spawn")
    port_ = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port_, str(tmp_path), fail_rank))
             for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    for p in procs:
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
    out = []
    for r in range(2):
        with open(os.path.join(tmp_path, f"rank{r}.pkl"), "rb") as f:
            out.append(pickle.load(f))
    return out


def test_sharded_runs_equal_unsharded(tmp_path):
    res = _launch(tmp_path, fail_rank=-1)
    assert all(r["ok"] for r in res), res
    parts = res[0]["parts"]
    # both ranks received the same gather
    for a, b in zip(parts, res[1]["parts"]):
        assert a["rank"] == b["rank"] and set(a["surf"]) == set(b["surf"])
        assert all(np.array_equal(a["surf"][k], b["surf"][k]) for k in a["surf"])
    merged = {}
    for p in parts:
        for k, v in p["surf"].items():
            assert k not in merged
            merged[k] = v
    assert sorted(merged) == list(range(len(SPECS_KW)))
    assert all(len(p["surf"]) > 0 for p in parts)  # both ranks did work
    for k, v in merged.items():
        assert np.array_equal(v, _run_domain(k)), k


def test_failed_rank_makes_the_gather_raise(tmp_path):
    res = _launch(tmp_path, fail_rank=1)
    assert not res[1]["ok"] and "injected failure" in res[1]["error"]
    assert not res[0]["ok"]  # the surviving rank's gather ended with an error

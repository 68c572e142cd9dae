"""The served form's host loop (frehdc_b200.serve.serve) on the CPU, with a
stand-in for the native server: requests are prepared and submitted in arrival
order, never before they arrive; every completion is collected, its domain
handed to on_done and then closed; latency and throughput come from the
server's clock; failures are counted; a request that cannot fit even an empty
batch, or a failing preparation, ends serving with an error."""
import itertools
import threading
import time

import pytest

from frehdc_b200 import native, serve


class FakeDomain:
    def __init__(self, nx, ny):
        self.nx, self.ny, self.closed = nx, ny, False

    def close(self):
        self.closed = True


class FakeServer:
    """Completes each request `steps` ms of its clock after submission, with the
    status the test asks for."""
    status_of: dict = {}
    instances: list = []

    def __init__(self, budget, cells_per_cta, device=0):
        self.t0 = time.perf_counter()
        self.pending = []
        self.lock = threading.Lock()
        self.tickets = itertools.count(1)
        self.submitted = []
        self.closed = False
        FakeServer.instances.append(self)

    def clock(self):
        return time.perf_counter() - self.t0

    def submit(self, dom, nsteps, t0=1):
        with self.lock:
            t = next(self.tickets)
            self.submitted.append((t, dom, self.clock()))
            self.pending.append({"ticket": t, "domain": dom, "steps": nsteps,
                                 "t_submit": self.clock(), "due": self.clock() + nsteps * 1e-3})
            return t

    def poll(self, timeout_ms=0, cap=64):
        time.sleep(min(timeout_ms, 5) / 1e3)
        now = self.clock()
        with self.lock:
            done = [r for r in self.pending if r["due"] <= now][:cap]
            self.pending = [r for r in self.pending if r not in done]
        out = []
        for r in done:
            st = FakeServer.status_of.get((r["domain"].nx, r["domain"].ny), 0)
            ran = 0 if st == 4 else r["steps"]
            out.append({"ticket": r["ticket"], "domain": r["domain"], "status": st, "steps": ran,
                        "t_submit": r["t_submit"], "t_admit": -1.0 if st == 4 else r["t_submit"],
                        "t_done": now})
        return out

    def info(self):
        return {"max_active": 3, "batch_steps": 10, "clock": self.clock()}

    def close(self):
        self.closed = True


@pytest.fixture
def fake(monkeypatch):
    FakeServer.status_of = {}
    FakeServer.instances = []
    monkeypatch.setattr(native, "Server", FakeServer)
    return FakeServer


def _requests():
    # (nx, ny, steps, arrival) in an order that is not the arrival order
    spec = [(16, 8, 5, 0.030), (8, 8, 3, 0.000), (32, 16, 7, 0.015), (8, 24, 2, 0.005)]
    return [serve.Request(k, None, steps, arr) for k, (_, _, steps, arr) in enumerate(spec)], spec


def test_serve_collects_every_request(fake):
    reqs, spec = _requests()
    built, seen = [], []

    def build(req):
        nx, ny = spec[req.rid][:2]
        built.append((req.rid, time.perf_counter()))
        return FakeDomain(nx, ny)

    def on_done(req):
        assert not req.domain.closed
        seen.append(req.rid)

    t_start = time.perf_counter()
    res = serve.serve(reqs, 1 << 30, 65536.0, build=build, on_done=on_done)
    srv = fake.instances[0]
    assert srv.closed
    # prepared and submitted in arrival order, none before its arrival
    assert [rid for rid, _ in built] == [1, 3, 2, 0]
    for rid, t in built:
        assert t - t_start >= reqs[rid].arrival - 1e-3
    assert sorted(seen) == [0, 1, 2, 3]
    assert res["requests"] == 4 and res["failed"] == 0
    assert res["cell_steps"] == sum(nx * ny * st for nx, ny, st, _ in spec)
    assert all(lat >= 0 for lat in res["latencies_s"])
    assert res["cell_steps_per_s"] == pytest.approx(res["cell_steps"] / res["wall_s"])
    assert res["max_active"] == 3 and res["batch_steps"] == 10
    assert all(r.domain is None and r.done >= r.arrival for r in reqs)


def test_serve_counts_failed_requests(fake):
    reqs, spec = _requests()
    fake.status_of = {(32, 16): 6}   # FREHD_ERR_CFL for one request
    res = serve.serve(reqs, 1 << 30, 65536.0, build=lambda r: FakeDomain(*spec[r.rid][:2]))
    assert res["requests"] == 4 and res["failed"] == 1


def test_serve_raises_for_a_request_that_never_fits(fake):
    reqs, spec = _requests()
    fake.status_of = {(8, 8): 4}     # FREHD_ERR_NOMEM, never admitted
    with pytest.raises(RuntimeError, match="does not fit"):
        serve.serve(reqs, 1 << 30, 65536.0, build=lambda r: FakeDomain(*spec[r.rid][:2]))
    assert fake.instances[0].closed


def test_serve_raises_when_preparation_fails(fake):
    reqs, spec = _requests()

    def build(req):
        if req.rid == 2:
            raise ValueError("bad deck")
        return FakeDomain(*spec[req.rid][:2])

    with pytest.raises(ValueError, match="bad deck"):
        serve.serve(reqs, 1 << 30, 65536.0, build=build)

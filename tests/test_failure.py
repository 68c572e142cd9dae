"""Failure paths of the device step, made on the host (nothing faults or hangs):

* CFL > 20 (monitorCFL's exit, nsfunctions.c:1225-1231): a wet 48 x 40 basin
  whose initial velocity (uuic.dat) is 100 m/s on an 8 x 8 block of faces; the
  flow passes CFL 20 at the second step, with either preconditioner (a flow
  that reaches CFL 20 by flooding and drying is decided by marginal wet/dry
  branches, which two converged solves need not take alike).  The device
  reports FREHD_ERR_CFL at the step where the oracle's CFL first exceeds 20,
  with the oracle's maximum; the domain then refuses to step until its state
  is set again.  In a
  served mix such a request is evicted at its failing step: it completes with
  the status, its slot goes to a waiting request at once, and the others end
  with their alone results.
* CG at maxIter (laspack's CGIter stops there silently, itersolv.c:399-418):
  with maxIter = 3 each step reports FREHD_ERR_CG_NOCONVERGE as a warning and
  goes on; the states follow the oracle's 3-iteration solves.
* A device wait that runs out: one CTA of the solve leaves before its first grid
  barrier (frehd_domain_set_wait_test), so the others' bounded wait (1 ms here)
  gives up; the step reports FREHD_ERR_TIMEOUT, and after the state is set
  again the domain steps exactly as a fresh one.
"""
import numpy as np
import pytest

from frehdc_b200 import deck as D
from frehdc_b200 import native
from oracle import port
from tests.helpers import deck_for, mismatches

pytestmark = pytest.mark.gpu

FIELDS = ["surf", "uuXP", "vvYP", "S", "depth", "cellV", "ind"]
# an initial 100 m/s jet (CFL 10 on 10 m cells at dt = 1 s) passes CFL 20 at step 2
CFL_SPEC = D.DeckSpec(nx=48, ny=40, steps=30, seed=3, u0_block=(20, 28, 16, 24, 100.0))
STATUS_NOCONV, STATUS_CFL, STATUS_TIMEOUT = 5, 6, 7


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if native.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")


@pytest.fixture(scope="module")
def cfl_case():
    """The CFL deck and the first step at which the oracle's max CFL exceeds 20."""
    d = D.make_deck(CFL_SPEC)
    o = port.from_deck(d, precond=port.PRECOND_JACOBI, x0=port.X0_ZERO)
    for tt in range(1, CFL_SPEC.steps + 1):
        c = o.step(tt)
        if c > 20:
            return d, tt, c
    pytest.fail("the CFL deck never exceeds CFL 20 in the oracle")


def test_cfl_exceedance_reported_at_the_oracles_step(cfl_case):
    d, k, cmax = cfl_case
    g = native.domain_from_deck(d)
    rc = g.run(1, CFL_SPEC.steps)
    st = g.stats()
    assert rc == STATUS_CFL
    assert st["step"] == k and st["status"] == STATUS_CFL
    assert abs(max(st["max_cflx"], st["max_cfly"]) - cmax) <= 1e-9 * cmax
    # the step before stays within the parity bound of the oracle
    h = native.domain_from_deck(d)
    assert h.run(1, k - 1) == 0
    o = port.from_deck(d, precond=port.PRECOND_JACOBI, x0=port.X0_ZERO)
    for tt in range(1, k):
        assert o.step(tt) <= 20
    N = d.nx * d.ny
    got = h.download(["surf"])["surf"][:N]
    ref = o.get("surf")[:N]
    assert np.max(np.abs(got - ref)) <= 1e-9 * np.max(np.abs(ref))


def test_cfl_stopped_domain_refuses_until_state_is_set(cfl_case):
    d, k, _ = cfl_case
    g = native.domain_from_deck(d)
    assert g.run(1, CFL_SPEC.steps) == STATUS_CFL
    after = g.download(FIELDS)
    assert g.run(k + 1, 3) == STATUS_CFL  # refused: nothing ran
    assert mismatches(g.download(FIELDS), after, FIELDS) == []
    # a new state clears the status: the domain steps from it like a fresh one
    g.init(d.bottom, d.bottomXP, d.bottomYP, d.surf0, d.u0, None, d.S0)
    assert g.run(1, k - 1) == 0
    fresh = native.domain_from_deck(d)
    assert fresh.run(1, k - 1) == 0
    assert mismatches(g.download(FIELDS), fresh.download(FIELDS), FIELDS) == []


def test_cg_at_maxiter_is_a_warning_and_follows_the_oracle(scratch):
    d, _ = deck_for("dry40x36", str(scratch))
    cfg = D.config_dict(d)
    cfg["maxIter"] = 3
    g = native.Domain(cfg, 0)
    g.set_fine_bottoms(d.zf, d.r)
    g.set_tide(D.tide_series(d))
    g.init(d.bottom, d.bottomXP, d.bottomYP, d.surf0, None, None, d.S0)
    o = port.Oracle(cfg, D.build_tables(d), D.tide_series(d), precond=port.PRECOND_JACOBI,
                    x0=port.X0_ZERO)
    o.init(d.bottom, d.bottomXP, d.bottomYP, d.surf0, None, None, d.S0)
    for tt in (1, 2, 3):
        assert g.step(tt) == STATUS_NOCONV
        st = g.stats()
        assert st["step"] == tt and st["cg_iters"] == 3 and st["cg_noconverge"] == 1
        assert st["cg_rel_residual"] >= cfg["eps"]
        o.step(tt)
        assert o.last_iters == 3
    N = d.nx * d.ny
    for f in ("surf", "S"):
        got, ref = g.download([f])[f][:N], o.get(f)[:N]
        assert np.max(np.abs(got - ref)) <= 1e-9 * np.max(np.abs(ref)), f
    # a run reports the warning once, after running every step
    assert g.run(4, 3) == STATUS_NOCONV and g.stats()["step"] == 6


def test_converged_steps_report_no_warning(scratch):
    d, _ = deck_for("dry40x36", str(scratch))
    g = native.domain_from_deck(d)
    assert g.run(1, 3) == 0 and g.stats()["cg_noconverge"] == 0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_barrier_wait_runs_out_then_domain_recovers(precision, scratch):
    d, _ = deck_for("wet48x40", str(scratch))  # 48 x 40 cells: three CTAs in the solve
    prec = native.PRECISION_MIXED if precision == "mixed" else native.PRECISION_FP64
    g = native.domain_from_deck(d, precision=prec)
    assert g.run(1, 2) == 0
    g.set_wait_test(1_000_000, skip_barrier_rank=0)
    with pytest.raises(native.FrehdError) as e:
        g.run(3, 2)
    assert e.value.status == STATUS_TIMEOUT
    assert g.stats()["status"] == STATUS_TIMEOUT
    # the context is still usable: a new state clears the status and the test
    # settings, and the domain steps exactly as a fresh one
    g.init(d.bottom, d.bottomXP, d.bottomYP, d.surf0, None, None, d.S0)
    assert g.run(1, 4) == 0
    fresh = native.domain_from_deck(d, precision=prec)
    assert fresh.run(1, 4) == 0
    assert mismatches(g.download(FIELDS), fresh.download(FIELDS), FIELDS) == []


def test_lone_cta_skip_reports_timeout(scratch):
    """A solve of one CTA has no partner whose wait could run out: the CTA that
    skips reports the timeout itself."""
    d = D.make_deck(D.DeckSpec(nx=24, ny=12, steps=10, seed=4))  # one 128 x 16 tile
    g = native.domain_from_deck(d)
    g.set_wait_test(1_000_000, skip_barrier_rank=0)
    with pytest.raises(native.FrehdError) as e:
        g.step(1)
    assert e.value.status == STATUS_TIMEOUT


def test_served_mix_evicts_the_failing_request(cfl_case, scratch):
    """Room for two domains: the CFL request and a long one run first, a third
    waits.  The CFL request completes with FREHD_ERR_CFL at its failing step
    and the third is admitted then, long before the long request ends; the two
    others end with their alone results."""
    d_cfl, k, _ = cfl_case
    d_long, _ = deck_for("wet48x40", str(scratch))
    d_wait, _ = deck_for("dry40x36", str(scratch))
    long_steps, wait_steps = k + 150, 20
    need = max(native.footprint(D.config_dict(x), x.r) for x in (d_cfl, d_long, d_wait))
    srv = native.Server(int(2.5 * need), 1e9)
    g_cfl, g_long, g_wait = (native.domain_from_deck(x) for x in (d_cfl, d_long, d_wait))
    t_cfl = srv.submit(g_cfl, CFL_SPEC.steps)
    t_long = srv.submit(g_long, long_steps)
    t_wait = srv.submit(g_wait, wait_steps)
    got = {}
    while len(got) < 3:
        for r in srv.poll(timeout_ms=200):
            got[r["ticket"]] = r
    srv.close()
    rc, rl, rw = got[t_cfl], got[t_long], got[t_wait]
    assert rc["status"] == STATUS_CFL and rc["steps"] == k
    assert rl["status"] == 0 and rl["steps"] == long_steps
    assert rw["status"] == 0 and rw["steps"] == wait_steps
    assert rw["t_admit"] >= rc["t_done"] - 1e-3  # waited for the evicted slot ...
    assert rw["t_admit"] < rl["t_done"]           # ... not for the long request
    for g, x, n in ((g_long, d_long, long_steps), (g_wait, d_wait, wait_steps)):
        b = native.Batch(8 << 30, 1e9)
        alone = native.domain_from_deck(x)
        slot = b.admit(alone, 1)
        for _ in range(n):
            b.step()
        b.release(slot)
        b.close()
        assert mismatches(g.download(FIELDS), alone.download(FIELDS), FIELDS) == []


def test_admitted_domain_cannot_be_destroyed(scratch):
    d, _ = deck_for("wet48x40", str(scratch))
    g = native.domain_from_deck(d)
    b = native.Batch(8 << 30, 1e9)
    slot = b.admit(g, 1)
    b.step()
    assert native.lib().frehd_domain_destroy(g.h) == 8  # FREHD_ERR_STATE: release first
    b.release(slot)
    b.close()
    assert g.run(2, 1) == 0
    g.close()

"""The batched form (frehd_batch_*): many resident domains, one launch per
sub-step over all of them.

A domain's arithmetic in a batch is the single-domain step's: the stencil
kernels run the same tile code.  Its solve depends on the packing:
* CTA groups: its CG runs on ceil(cells/cells_per_cta) CTAs; with
  cells_per_cta = 1 (as many CTAs as the single-domain solve uses) a batch
  reproduces single-domain runs bit for bit;
* the tile list (default): the same sweeps over the domain's tiles, with the
  partial sums added in the domain's own tile order; its results agree with
  the single-domain runs to the solver's rounding.
In either packing a domain's result is the same alone and in a mix, bit for bit.
"""
import numpy as np
import pytest

from frehdc_b200 import native
from tests.helpers import SPECS, deck_for, mismatches

pytestmark = pytest.mark.gpu
FIELDS = ["surf", "uuXP", "vvYP", "S", "depth", "cellV", "CDXP", "CDYP", "ind"]
BUDGET = 8 << 30


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if native.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")


def _run_batch(names, steps, scratch, cells_per_cta, graph=True, packing=None,
               precision=native.PRECISION_FP64, tiles_per_block=None):
    b = native.Batch(BUDGET, cells_per_cta)
    b.set_graph(graph)
    if packing is not None:
        b.set_cg_packing(packing)
    if tiles_per_block is not None:
        b.set_stencil_tiles(tiles_per_block)
    doms = {}
    for n in names:
        d, _ = deck_for(n, str(scratch))
        g = native.domain_from_deck(d, geometry="fine", precision=precision, eps_inner=1e-5)
        doms[n] = (g, b.admit(g, 1))
    for _ in range(steps):
        b.step()
    info = b.info()
    out = {}
    for n, (g, slot) in doms.items():
        b.release(slot)
        out[n] = (g.download(FIELDS), g.stats())
    b.close()
    return out, info


def test_batch_matches_single_domain_bitwise(scratch):
    names = list(SPECS)
    got, info = _run_batch(names, 12, scratch, cells_per_cta=1, packing=native.BATCH_CTA_GROUPS)
    assert info["domains"] == len(names)
    for n in names:
        d, _ = deck_for(n, str(scratch))
        g = native.domain_from_deck(d, geometry="fine")
        assert g.run(1, 12) == 0
        ref = g.download(FIELDS)
        assert mismatches(got[n][0], ref, FIELDS) == [], n
        st = g.stats()
        assert got[n][1]["step"] == st["step"] == 12
        assert got[n][1]["volume"] == st["volume"]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tile_list_matches_single_domain(precision, scratch):
    """The tile-list solve against each domain stepped alone: the same solver,
    partial sums added in another order."""
    names = list(SPECS)
    prec = native.PRECISION_MIXED if precision == "mixed" else native.PRECISION_FP64
    got, info = _run_batch(names, 12, scratch, cells_per_cta=1, packing=native.BATCH_TILE_LIST,
                           precision=prec)
    assert info["cg_ctas"] == info["cg_capacity"] > 0
    for n in names:
        d, _ = deck_for(n, str(scratch))
        g = native.domain_from_deck(d, geometry="fine", precision=prec, eps_inner=1e-5)
        assert g.run(1, 12) == 0
        ref = g.download(FIELDS)
        # the parity tests' whole-run bounds: 1e-9, face velocities 3e-9
        assert mismatches(got[n][0], ref, ["ind"]) == [], n
        assert mismatches(got[n][0], ref, ["uuXP", "vvYP"], exact=False, rtol=3e-9) == [], n
        assert mismatches(got[n][0], ref, [f for f in FIELDS if f not in ("ind", "uuXP", "vvYP")],
                          exact=False, rtol=1e-9) == [], n
        st = g.stats()
        assert got[n][1]["step"] == st["step"] == 12
        assert abs(got[n][1]["volume"] - st["volume"]) <= 1e-12 * abs(st["volume"])
        if precision == "fp64":
            assert abs(got[n][1]["cg_iters"] - st["cg_iters"]) <= 2


@pytest.mark.parametrize("packing", ["tile_list", "cta_groups"])
@pytest.mark.parametrize("graph", [True, False])
def test_same_alone_and_in_mix(graph, packing, scratch):
    names = list(SPECS)
    pk = native.BATCH_TILE_LIST if packing == "tile_list" else native.BATCH_CTA_GROUPS
    mix, info = _run_batch(names, 10, scratch, cells_per_cta=1e9, graph=graph, packing=pk)
    assert info["graph"] == (1 if graph else 0)
    for n in names:
        alone, _ = _run_batch([n], 10, scratch, cells_per_cta=1e9, graph=graph, packing=pk)
        assert mismatches(mix[n][0], alone[n][0], FIELDS) == [], n


@pytest.mark.parametrize("tiles_per_block", [1, 3, 8])
def test_stencil_tiles_per_block_same_doubles(tiles_per_block, scratch):
    """The stencil blocks' tile count changes the launch shape, not the
    arithmetic: the same doubles as the default four tiles per block."""
    names = list(SPECS)
    ref, _ = _run_batch(names, 6, scratch, cells_per_cta=1e9)
    got, info = _run_batch(names, 6, scratch, cells_per_cta=1e9, tiles_per_block=tiles_per_block)
    for n in names:
        assert mismatches(got[n][0], ref[n][0], FIELDS) == [], n


def test_stencil_tiles_per_block_checked():
    b = native.Batch(BUDGET, 1e9)
    for bad in (0, 9, -1):
        with pytest.raises(native.FrehdError):
            b.set_stencil_tiles(bad)
    b.close()


def test_mixed_precision_same_alone_and_in_mix(scratch):
    names = list(SPECS)
    mix, _ = _run_batch(names, 10, scratch, cells_per_cta=1, precision=native.PRECISION_MIXED)
    for n in ("wet48x40", "dry40x36", "tvd44x36"):
        alone, _ = _run_batch([n], 10, scratch, cells_per_cta=1, precision=native.PRECISION_MIXED)
        assert mismatches(mix[n][0], alone[n][0], FIELDS) == [], n


def test_admission_by_budget(scratch):
    d, _ = deck_for("wet48x40", str(scratch))
    need = native.footprint(native.domain_from_deck(d).cfg, d.r)
    g1 = native.domain_from_deck(d, geometry="fine")
    g2 = native.domain_from_deck(d, geometry="fine")
    b = native.Batch(int(1.5 * need), 1e9)
    assert b.try_admit(g1) is not None
    assert b.try_admit(g2) is None  # over the budget: refused, still usable alone
    assert g2.run(1, 2) == 0
    b.close()


def test_served_results_equal_alone(scratch):
    """Requests served with staggered arrivals (continuous batching) give the
    same state as each request's domain stepped alone in a batch."""
    from frehdc_b200 import serve
    names = list(SPECS)
    steps = {"wet48x40": 7, "dry40x36": 11, "dry37x29": 5, "tvd44x36": 9, "tvdwet44x36": 4,
             "inflow36x30": 6, "wind40x32": 8}
    results = {}

    def done(req):
        results[req.rid] = req.domain.download(FIELDS)

    reqs = []
    for k, n in enumerate(names):
        d, _ = deck_for(n, str(scratch))
        reqs.append(serve.Request(k, d, steps[n], arrival=0.002 * k))
    res = serve.serve(reqs, BUDGET, 1e9, on_done=done)
    assert res["requests"] == len(names) and res["failed"] == 0
    for k, n in enumerate(names):
        alone, _ = _run_batch([n], steps[n], scratch, cells_per_cta=1e9)
        assert mismatches(results[k], alone[n][0], FIELDS) == [], n


def test_server_waits_for_room_and_refuses_what_never_fits(scratch):
    """The native server admits a request only when the budget has room (with
    room for one domain at a time they run one after another, each with its
    single-domain result) and completes a request larger than the whole budget
    with FREHD_ERR_NOMEM without running it."""
    names = ["wet48x40", "dry40x36", "dry37x29"]
    decks = {n: deck_for(n, str(scratch))[0] for n in names}
    need = max(native.footprint(native.domain_from_deck(d).cfg, d.r) for d in decks.values())
    srv = native.Server(int(1.2 * need), 1e9)
    doms = {n: native.domain_from_deck(d) for n, d in decks.items()}
    tickets = {srv.submit(g, 6): n for n, g in doms.items()}
    big_deck = deck_for("tvd44x36", str(scratch))[0]
    big = native.domain_from_deck(big_deck)
    small_srv = native.Server(native.footprint(big.cfg, big_deck.r) // 2, 1e9)
    t_big = small_srv.submit(big, 3)
    got = []
    while len(got) < len(names):
        got += srv.poll(timeout_ms=200)
    assert srv.info()["max_active"] == 1
    for r in got:
        n = tickets[r["ticket"]]
        assert r["status"] == 0 and r["steps"] == 6 and r["t_admit"] >= r["t_submit"]
        alone, _ = _run_batch([n], 6, scratch, cells_per_cta=1e9)
        assert mismatches(r["domain"].download(FIELDS), alone[n][0], FIELDS) == [], n
    # admitted one after another: each waited for the previous one's release
    order = sorted(got, key=lambda r: r["t_admit"])
    for a, b in zip(order, order[1:]):
        assert b["t_admit"] >= a["t_done"] - 1e-3
    refused = []
    while not refused:
        refused = small_srv.poll(timeout_ms=200)
    assert refused[0]["ticket"] == t_big and refused[0]["status"] == 4
    assert refused[0]["steps"] == 0 and refused[0]["t_admit"] < 0
    assert big.run(1, 2) == 0  # handed back untouched, usable alone
    srv.close()
    small_srv.close()

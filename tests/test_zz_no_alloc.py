"""frehd_cg_solve_noalloc (the solve for callers that cannot allocate) against
the domain's own solve (frehd_domain_phase SOLVE), through the C ABI.

The domain assembles each step's system; the test rewrites it into the
no-allocation entry point's row-major convention, solves it there from
caller-owned device buffers, and compares x with the domain's solution.  Both
run the same Jacobi-PCG with the same tile partition and stopping rule, so x
agrees to the solve tests' 1e-10.  Two calls in a row per deck: the second
finds the first call's contents in the shared scratch.  The same bound holds
against an independent numpy Jacobi-PCG of the system, from a warm start, for a
solve only queued on the caller's stream, and at the 512 x 512 maximum.  This
file is collected last so that it also runs after every other GPU test in one
process.
"""
import numpy as np
import pytest

from frehdc_b200 import native
from tests.helpers import deck_for, max_rel

pytestmark = pytest.mark.gpu

SOLVE_TOL = 1e-10
MAX_CELLS = 512 * 512


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if native.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")


def _noalloc_system(sysr: dict, nx: int, ny: int):
    """The domain's system (reference terms) in the entry point's convention:
    row-major, Gx/Gy per east/north face, decoupled rows with a negative Ct."""
    ct = sysr["GnCt"].reshape(ny, nx)
    xp, xm = sysr["GnXP"].reshape(ny, nx), sysr["GnXM"].reshape(ny, nx)
    yp, ym = sysr["GnYP"].reshape(ny, nx), sysr["GnYM"].reshape(ny, nx)
    iso = (xp == 0) & (xm == 0) & (yp == 0) & (ym == 0)
    gx = xp.copy()
    gx[:, :-1] = np.where(gx[:, :-1] != 0, gx[:, :-1], xm[:, 1:])
    gy = yp.copy()
    gy[:-1, :] = np.where(gy[:-1, :] != 0, gy[:-1, :], ym[1:, :])
    Ct = np.where(iso, -ct, ct)
    b = sysr["z"].reshape(nx, ny).T  # transposed order -> row-major
    return [np.ascontiguousarray(a, dtype=np.float64).ravel() for a in (Ct, gx, gy, b)]


@pytest.mark.parametrize("name", ["dry40x36", "wet48x40"])
def test_noalloc_matches_domain_solve(name, scratch):
    import torch

    d, _ = deck_for(name, str(scratch))
    # the no-allocation solve takes decoupled rows' couplings in b (its documented
    # convention), so the domain solves the same, eliminated form
    g = native.domain_from_deck(d, geometry="fine", decoupled=native.DECOUPLED_ELIMINATED)
    nx, ny = g.nx, g.ny
    eps, max_iter = g.cfg["eps"], g.cfg["maxIter"]
    dev = torch.device("cuda", 0)
    x = torch.full((nx * ny,), np.nan, dtype=torch.float64, device=dev)
    for tt in (1, 2):
        g.phase(native.PHASE_EXPLICIT, tt)
        g.phase(native.PHASE_SOLVE, tt)
        want = g.solution().reshape(nx, ny).T.ravel()  # transposed -> row-major
        bufs = [torch.from_numpy(a).to(dev) for a in _noalloc_system(g.system(), nx, ny)]
        torch.cuda.synchronize()
        its, rel = native.cg_solve_noalloc(nx, ny, *[t.data_ptr() for t in bufs], x.data_ptr(),
                                           eps, max_iter, x0_from_x=False)
        got = x.cpu().numpy()
        assert np.isfinite(got).all(), tt
        assert 0 < its < max_iter and rel < eps, (tt, its, rel)
        assert max_rel(got, want) <= SOLVE_TOL, (tt, max_rel(got, want))
        g.phase(native.PHASE_UPDATE, tt)


def _numpy_jacobi_pcg(Ct, Gx, Gy, b, nx, ny, eps, max_iter):
    """The entry point's system solved by a plain numpy Jacobi-PCG from x = 0
    (CGIter's ordering, itersolv.c:355-456; stop at ||r|| < eps*||b||, checked
    before each iteration): decoupled rows (Ct < 0) hold b/|Ct| and enter their
    neighbours' rows at that value."""
    import scipy.sparse as sp
    n = nx * ny
    d = np.abs(Ct)
    dec = Ct < 0
    idx = np.arange(n).reshape(ny, nx)
    rows, cols, vals = [], [], []
    gx, gy = Gx.reshape(ny, nx), Gy.reshape(ny, nx)
    for (a, c, g) in ((idx[:, :-1], idx[:, 1:], gx[:, :-1]), (idx[:-1, :], idx[1:, :], gy[:-1, :])):
        a, c, g = a.ravel(), c.ravel(), g.ravel()
        rows += [a, c]
        cols += [c, a]
        vals += [-g, -g]
    rows, cols, vals = np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)
    keep = ~dec[rows]  # a decoupled row has no couplings
    off = sp.csr_matrix((vals[keep], (rows[keep], cols[keep])), shape=(n, n))
    xdec = np.where(dec, b / d, 0.0)
    bm = b - off @ xdec                                   # decoupled neighbours into b
    offc = off @ sp.diags((~dec).astype(np.float64))      # couplings to unknown rows only
    A = sp.diags(d) + offc
    x = np.zeros(n)
    r = bm - A @ x
    bnorm = np.linalg.norm(b)
    rho, rho_old, p, it = float(r @ (r / d)), 1.0, np.zeros(n), 0
    while not np.linalg.norm(r) < eps * bnorm and it < max_iter:
        it += 1
        beta = 0.0 if it == 1 else rho / rho_old
        p = r / d + beta * p
        q = A @ p
        alpha = rho / float(p @ q)
        x = x + alpha * p
        r = r - alpha * q
        rho_old, rho = rho, float(r @ (r / d))
    return x, it


@pytest.mark.parametrize("name", ["dry40x36", "wet48x40"])
def test_noalloc_matches_an_independent_jacobi_pcg(name, scratch):
    """The entry point against a numpy Jacobi-PCG of the same system (not the
    library's own solve)."""
    import torch

    d, _ = deck_for(name, str(scratch))
    g = native.domain_from_deck(d, geometry="fine", decoupled=native.DECOUPLED_ELIMINATED)
    nx, ny = g.nx, g.ny
    eps, max_iter = g.cfg["eps"], g.cfg["maxIter"]
    g.phase(native.PHASE_EXPLICIT, 1)
    host = _noalloc_system(g.system(), nx, ny)
    want, _ = _numpy_jacobi_pcg(*host, nx, ny, eps, max_iter)
    dev = torch.device("cuda", 0)
    bufs = [torch.from_numpy(a).to(dev) for a in host]
    x = torch.full((nx * ny,), np.nan, dtype=torch.float64, device=dev)
    for _ in range(2):  # the second call finds the first one's scratch contents
        torch.cuda.synchronize()
        its, rel = native.cg_solve_noalloc(nx, ny, *[t.data_ptr() for t in bufs], x.data_ptr(),
                                           eps, max_iter, x0_from_x=False)
        assert 0 < its < max_iter and rel < eps
        assert max_rel(x.cpu().numpy(), want) <= SOLVE_TOL


def test_noalloc_warm_start_and_queued_on_a_stream(scratch):
    """x0_from_x starts from the x passed in (the converged solution: at most a
    few iterations, the same answer), and with wait=False the call only queues
    the solve on the caller's stream."""
    import torch

    d, _ = deck_for("dry40x36", str(scratch))
    g = native.domain_from_deck(d, geometry="fine", decoupled=native.DECOUPLED_ELIMINATED)
    nx, ny = g.nx, g.ny
    eps, max_iter = g.cfg["eps"], g.cfg["maxIter"]
    g.phase(native.PHASE_EXPLICIT, 1)
    g.phase(native.PHASE_SOLVE, 1)
    want = g.solution().reshape(nx, ny).T.ravel()
    dev = torch.device("cuda", 0)
    bufs = [torch.from_numpy(a).to(dev) for a in _noalloc_system(g.system(), nx, ny)]
    ptrs = [t.data_ptr() for t in bufs]
    x = torch.from_numpy(want.copy()).to(dev)
    torch.cuda.synchronize()
    its, rel = native.cg_solve_noalloc(nx, ny, *ptrs, x.data_ptr(), eps, max_iter, x0_from_x=True)
    assert its <= 2 and rel < eps
    assert max_rel(x.cpu().numpy(), want) <= SOLVE_TOL
    st = torch.cuda.Stream(device=dev)
    y = torch.full((nx * ny,), np.nan, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    assert native.cg_solve_noalloc(nx, ny, *ptrs, y.data_ptr(), eps, max_iter, x0_from_x=False,
                                   stream=st.cuda_stream, wait=False) is None
    st.synchronize()
    assert max_rel(y.cpu().numpy(), want) <= SOLVE_TOL


def test_noalloc_at_the_maximum_size():
    """512 x 512 cells, the largest size the static scratch holds (its last
    vector ends at the array's end), twice in a row."""
    import torch

    from frehdc_b200 import deck as D
    d = D.make_deck(D.DeckSpec(nx=512, ny=512, dx=10.0, steps=5, seed=31, dry_frac=0.25))
    g = native.domain_from_deck(d, geometry="fine", decoupled=native.DECOUPLED_ELIMINATED)
    nx, ny = g.nx, g.ny
    assert nx * ny == MAX_CELLS
    eps, max_iter = g.cfg["eps"], g.cfg["maxIter"]
    dev = torch.device("cuda", 0)
    x = torch.full((nx * ny,), np.nan, dtype=torch.float64, device=dev)
    for tt in (1, 2):
        g.phase(native.PHASE_EXPLICIT, tt)
        g.phase(native.PHASE_SOLVE, tt)
        want = g.solution().reshape(nx, ny).T.ravel()
        bufs = [torch.from_numpy(a).to(dev) for a in _noalloc_system(g.system(), nx, ny)]
        torch.cuda.synchronize()
        its, rel = native.cg_solve_noalloc(nx, ny, *[t.data_ptr() for t in bufs], x.data_ptr(),
                                           eps, max_iter, x0_from_x=False)
        assert 0 < its < max_iter and rel < eps, (tt, its, rel)
        assert max_rel(x.cpu().numpy(), want) <= SOLVE_TOL, tt
        g.phase(native.PHASE_UPDATE, tt)


def test_noalloc_rejects_oversize():
    with pytest.raises(native.FrehdError) as e:
        native.cg_solve_noalloc(513, 512, 1, 1, 1, 1, 1, 1e-12, 10)
    assert e.value.status == 1 and str(MAX_CELLS) in str(e.value)

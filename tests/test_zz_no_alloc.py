"""frehd_cg_solve_noalloc (the solve for callers that cannot allocate) against
the domain's own solve (frehd_domain_phase SOLVE), through the C ABI.

The domain assembles each step's system; the test rewrites it into the
no-allocation entry point's row-major convention, solves it there from
caller-owned device buffers, and compares x with the domain's solution.  Both
run the same Jacobi-PCG with the same tile partition and stopping rule, so x
agrees to the solve tests' 1e-10.  Two calls in a row per deck: the second
finds the first call's contents in the shared scratch.  This file is collected
last so that it also runs after every other GPU test in one process.
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


def test_noalloc_rejects_oversize():
    with pytest.raises(native.FrehdError) as e:
        native.cg_solve_noalloc(513, 512, 1, 1, 1, 1, 1, 1e-12, 10)
    assert e.value.status == 1 and str(MAX_CELLS) in str(e.value)

"""Block-check face areas (checkBlock = 1 of the reference's pre-processor).

CPU: frehd_build_tables_ex with FREHD_GEOM_BLOCK_CHECK against the step-by-step
restatement of ComputeFaceAreaWithBlockCheck.m (oracle/blockcheck.py), bit for
bit, on rough decks with r = 2, 4, 8 and on a hand-made block with two equal
largest clusters; only the face areas change.  GPU: the device's on-the-fly
evaluation from fine bottoms gives the same initial geometry as the tables,
every phase of a step matches the C oracle driven by those tables, and a whole
run matches the oracle to the plain form's tolerances.
"""
import numpy as np
import pytest

from frehdc_b200 import deck as D
from frehdc_b200 import native
from oracle import blockcheck as BC
from tests.helpers import max_rel, mismatches

ROUGH = [dict(nx=24, ny=20, seed=3, dry_frac=0.35, roughness=0.4),
         dict(nx=16, ny=12, seed=7, dry_frac=0.5, roughness=0.8),
         dict(nx=12, ny=10, r=2, seed=5, dry_frac=0.4, roughness=0.6),
         dict(nx=8, ny=6, r=8, seed=9, dry_frac=0.4, roughness=0.6)]


def _deck(kw, block=True):
    return D.make_deck(D.DeckSpec(steps=5, block_check=block, **kw), with_tables=False)


@pytest.mark.parametrize("kw", ROUGH, ids=lambda k: f"r{k.get('r', 4)}_{k['nx']}x{k['ny']}")
def test_tables_match_restatement(kw):
    d = _deck(kw)
    t = D.build_tables(d)
    o = BC.face_tables(d.zf, d.nx, d.ny, d.r, d.spec.dx / d.r, d.surfmin, d.dsurf, d.Ne)
    for q, name in enumerate(["Np", "Nm", "Op", "Om"]):
        assert np.array_equal(t[6 + q], o[q]), name
    # V, Z and the half volumes never use the clusters
    plain = D.build_tables(_deck(kw, block=False))
    assert np.array_equal(t[:6], plain[:6])


def test_block_check_changes_face_areas():
    d = _deck(ROUGH[0])
    t, plain = D.build_tables(d), D.build_tables(_deck(ROUGH[0], block=False))
    changed = int((t[6:] != plain[6:]).sum())
    assert changed > 100
    assert np.all(t[6:] <= plain[6:])   # masking only removes water


def test_equal_clusters_and_boundaries():
    """Two 2 x 2 blocks: block 0 holds two separate 2-pixel puddles (a tie), the
    first one in MATLAB's column-major scan must win; block 1 is wet at its
    east (domain-boundary) edge only through a one-pixel cluster."""
    r, nx, ny = 4, 2, 1
    zf = np.full((ny * r, nx * r), 1.0)
    # block 0 (fi 0..3): puddle A at (fi 0..1, fj 1), puddle B at (fi 3, fj 2..3)
    zf[1, 0:2] = -1.0
    zf[2:4, 3] = -1.0
    # block 1 (fi 4..7): a 3-pixel cluster at fi 4 (west edge) and a lone pixel at fi 7
    zf[0:3, 4] = -1.0
    zf[3, 7] = -1.0
    t = native.build_tables(zf, nx, ny, r, 0.5, 0.5, 0.0, 0.1, 2, block_check=True)
    o = BC.face_tables(zf, nx, ny, r, 0.5, 0.0, 0.1, 2)
    for q in range(4):
        assert np.array_equal(t[6 + q], o[q])
    # puddle A (first in the x-fastest scan) wins: block 0's west edge is wet
    assert t[7, 0, 0] > 0          # Nm of block 0 (boundary face, unmasked sum)
    # block 0's east edge pixels belong to puddle B only: the shared face is dry
    assert t[6, 0, 0] == 0 and t[7, 0, 1] == 0
    # block 1's lone east pixel is not its largest cluster: boundary face blocked
    assert t[6, 0, 1] == 0


def test_rejects_bad_options():
    zf = np.zeros((36, 36))
    with pytest.raises(native.FrehdError) as e:
        native.build_tables(zf, 4, 4, 9, 1.0, 1.0, 0.0, 0.1, 2, block_check=True)
    assert e.value.status == 2
    out = np.empty((10, 2, 16))
    rc = native.lib().frehd_build_tables_ex(native.as_dp(zf), 36, 4, 4, 9, 1.0, 1.0, 0.0, 0.1, 2,
                                            4, native.as_dp(out))
    assert rc == 1


# ---------------------------------------------------------------- GPU
PUDDLES = dict(nx=40, ny=32, seed=3, dry_frac=0.35, roughness=0.4)
UPLOAD = ["surf", "uuXP", "vvYP", "S", "depth", "CDXP", "CDYP", "CFLx", "CFLy", "V", "Z", "Nx",
          "Oy", "Vx", "Vy", "Zx", "Zy", "ind", "bottomZ", "bottomXP", "bottomYP"]
EXACT = ["surf", "uuXP", "vvYP", "S", "depth", "V", "Z", "Nx", "Oy", "Vx", "Vy", "Zx", "Zy", "ind",
         "surfOld", "cellV", "Sm", "Fuu", "Fvv", "CFLx", "CFLy", "uuYP", "vvXP"]
POW = ["CDXP", "CDYP"]


def _gpu_deck(steps):
    if native.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")
    return D.make_deck(D.DeckSpec(steps=steps, block_check=True, **PUDDLES), with_tables=True)


@pytest.mark.gpu
def test_device_geometry_equals_tables():
    d = _gpu_deck(5)
    gf = native.domain_from_deck(d, geometry="fine")
    gt = native.domain_from_deck(d, geometry="tables")
    a, b = gf.download(UPLOAD), gt.download(UPLOAD)
    assert mismatches(a, b, UPLOAD) == []
    plain = native.domain_from_deck(D.make_deck(D.DeckSpec(steps=5, **PUDDLES), with_tables=False))
    c = plain.download(["Nx", "Oy"])
    assert not (np.array_equal(a["Nx"], c["Nx"]) and np.array_equal(a["Oy"], c["Oy"]))


@pytest.mark.gpu
def test_phases_bitwise_with_block_check():
    from oracle import port
    d = _gpu_deck(12)
    o = port.from_deck(d, precond=port.PRECOND_JACOBI, x0=port.X0_ZERO)
    g = native.domain_from_deck(d, geometry="fine")
    for tt in range(1, 13):
        g.upload({n: o.get(n) for n in UPLOAD})
        o.explicit(tt)
        g.phase(native.PHASE_EXPLICIT, tt)
        sysg = {**g.system(), **g.download(["EnXP", "EnYP"])}
        names = ["GnCt", "GnXP", "GnXM", "GnYP", "GnYM", "z", "EnXP", "EnYP"]
        assert mismatches(sysg, {n: o.get(n) for n in names}, names) == [], tt
        o.solve()
        x = o.get("x")
        o.update(tt, x)
        g.phase(native.PHASE_UPDATE, tt, x_ext=x)
        got = g.download(EXACT + POW)
        ref = {n: o.get(n) for n in EXACT + POW}
        assert mismatches(got, ref, EXACT) == [], tt
        assert mismatches(got, ref, POW, exact=False, rtol=1e-15) == [], tt


@pytest.mark.gpu
def test_full_run_with_block_check():
    from oracle import port
    steps = 30
    d = _gpu_deck(steps)
    o = port.from_deck(d, precond=port.PRECOND_JACOBI, x0=port.X0_ZERO)
    for tt in range(1, steps + 1):
        o.step(tt)
    g = native.domain_from_deck(d, geometry="fine")
    assert g.run(1, steps) == 0
    got = g.download(["surf", "uuXP", "vvYP", "S"])
    for n, tol in [("surf", 1e-9), ("S", 1e-9), ("uuXP", 3e-9), ("vvYP", 3e-9)]:
        assert max_rel(got[n], o.get(n)) <= tol, n

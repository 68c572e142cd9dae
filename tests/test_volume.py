"""Water-volume bookkeeping of the step.

Every step, the cell volumes after the flux update (cellV, volumeByFluxSub,
subgrid.c:1227-1263) must equal the volumes before it plus dt times the net
inflow through the outer faces (the tidal row), plus the inflow cells' volume,
plus the water added where a negative volume is clipped: interior face fluxes leave one cell and enter the
next with the same value, so they cancel.  Checked to 1e-13 relative, per step,
for the C oracle (CPU) and the device step (GPU).  The device's total volume
against the reference program's is checked by tests/test_golden.py.
"""
import pytest

from tests.helpers import SPECS, deck_for, inflow_source, ledger_residual

LEDGER_TOL = 1e-13


@pytest.mark.parametrize("name", list(SPECS))
def test_oracle_volume_ledger(name, scratch):
    from oracle import port
    d, _ = deck_for(name, str(scratch))
    o = port.from_deck(d, precond=port.PRECOND_SSOR, x0=port.X0_ZERO)
    for tt in range(1, d.spec.steps + 1):
        V_old = o.get("V")
        o.step(tt)
        r = ledger_residual(V_old, o.get("cellV"), o.get("Fuu"), o.get("Fvv"), d.spec.nx,
                            d.spec.ny, d.spec.dt, inflow_source(d, tt))
        assert r <= LEDGER_TOL, (tt, r)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(SPECS))
def test_device_volume_ledger(name, scratch):
    from frehdc_b200 import native
    if native.device_count() < 1:
        pytest.fail("no CUDA device visible: the GPU tests need a B200")
    d, _ = deck_for(name, str(scratch))
    g = native.domain_from_deck(d, geometry="fine")
    for tt in range(1, d.spec.steps + 1):
        V_old = g.download(["V"])["V"]
        assert g.step(tt) == 0
        st = g.download(["cellV", "Fuu", "Fvv"])
        r = ledger_residual(V_old, st["cellV"], st["Fuu"], st["Fvv"], d.spec.nx, d.spec.ny,
                            d.spec.dt, inflow_source(d, tt))
        assert r <= LEDGER_TOL, (tt, r)

"""Failure detection without faulting the GPU: every failure is made on the
host (a NaN planted in an initial field, an iteration budget too small to
converge) or by a wait that runs out (one CTA of the single-launch solve
leaves before a grid barrier, so the others' bounded waits expire).  Each
case must come back as a status code, and the device must stay usable."""
import numpy as np
import pytest

import ifc

pytestmark = pytest.mark.gpu


def test_nan_initial_field_reports_diverged(gpu_ok):
    cfg = ifc.cavity2d(32)
    s = ifc.Solver(cfg)
    u = np.zeros(32 * 32, dtype=np.float32)
    u[100] = np.nan
    s.set("u", u)
    with pytest.raises(ifc.IfcError) as e:
        s.solve()
    assert e.value.status == ifc.DIVERGED


def test_iteration_budget_exhausted_reports_not_converged(gpu_ok):
    s = ifc.Solver(ifc.cavity2d(32, numOuterIter=5))
    st = s.solve()
    assert st["status"] == ifc.NOT_CONVERGED and not st["converged"]
    assert st["outer_iterations"] == 5


def test_grid_barrier_timeout_is_reported_and_device_stays_usable(gpu_ok, monkeypatch):
    cfg = ifc.channel2d(64, 16)
    monkeypatch.setenv("IFC_TEST_STALL_BARRIER", "1")
    s = ifc.Solver(cfg)
    with pytest.raises(ifc.IfcError) as e:
        s.iterate(3)
    assert e.value.status == ifc.TIMEOUT
    s.close()
    monkeypatch.delenv("IFC_TEST_STALL_BARRIER")
    t = ifc.Solver(cfg)
    st = t.iterate(3)
    assert st["status"] == ifc.OK and st["outer_iterations"] == 3
    assert np.isfinite(t.get("u")).all()


def test_energy_barrier_timeout_is_reported_and_handle_stays_usable(gpu_ok, monkeypatch):
    """The cooperative 2D energy launch (k_coef_solve2d) with CTA 0 leaving
    before its first grid barrier: the other CTAs' bounded waits run out,
    solve_energy returns TIMEOUT, and the same handle then solves normally."""
    monkeypatch.delenv("IFC_PERSIST_OFF", raising=False)
    cfg = ifc.cavity2d(32)
    s = ifc.Solver(cfg)
    s.iterate(50)
    monkeypatch.setenv("IFC_TEST_STALL_BARRIER", "1")
    with pytest.raises(ifc.IfcError) as e:
        s.solve_energy(max_sweeps=40, tol=0.0)
    assert e.value.status == ifc.TIMEOUT
    monkeypatch.delenv("IFC_TEST_STALL_BARRIER")
    r = s.solve_energy(max_sweeps=40, tol=0.0)
    assert r["status"] == ifc.OK and r["sweeps"] == 40
    assert np.isfinite(s.get("T")).all()
    st = s.iterate(3)
    assert st["status"] == ifc.OK


def test_3d_cooperative_timeout_is_reported_at_sync_and_handle_stays_usable(gpu_ok, monkeypatch):
    """The cooperative 3D p' solve (k_csolve3d) enqueued without a host wait,
    with CTA 0 leaving before its first grid barrier: the other CTAs' bounded
    waits run out, ifc_sync reports TIMEOUT, and the same handle then runs
    the stage and whole outer iterations normally."""
    s = ifc.Solver(ifc.cavity3d(16))
    s.iterate(5)
    s.stage("mom_solve")
    s.stage("rhie_chow")
    monkeypatch.setenv("IFC_TEST_STALL_BARRIER", "1")
    s.stage("pcorr_solve", wait=False)
    with pytest.raises(ifc.IfcError) as e:
        s.sync()
    assert e.value.status == ifc.TIMEOUT
    monkeypatch.delenv("IFC_TEST_STALL_BARRIER")
    s.stage("pcorr_solve")
    st = s.iterate(3)
    assert st["status"] == ifc.OK and st["outer_iterations"] == 8
    assert np.isfinite(s.get("u")).all()

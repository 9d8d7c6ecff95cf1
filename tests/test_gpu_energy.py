"""Energy equation on the GPU (ifc_solve_energy) against its restatement in
the oracle: bit for bit after a fixed number of sweeps (both round every
operation as written), on a converged cavity and channel flow and a 3D
cavity; and a converged solve that obeys the maximum principle."""
import numpy as np
import pytest

import ifc
import oracle as O
from helpers import assert_bitwise

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["cooperative", "passes"])
def energy_form(request, monkeypatch):
    """Both 2D device forms of the energy sweeps: one cooperative launch per
    cycle, or one launch per pass of 5 sweeps (IFC_PERSIST_OFF=1)."""
    if request.param == "passes":
        monkeypatch.setenv("IFC_PERSIST_OFF", "1")
    else:
        monkeypatch.delenv("IFC_PERSIST_OFF", raising=False)
    return request.param


@pytest.mark.parametrize("case", ["cavity24", "channel48x16", "cavity3d8", "cavity24_fp64", "channel200x70"])
def test_energy_sweeps_match_oracle(gpu_ok, energy_form, case):
    prec = "d" if case.endswith("fp64") else "f"
    cfg = {"cavity24": ifc.cavity2d(24), "channel48x16": ifc.channel2d(48, 16), "cavity3d8": ifc.cavity3d(8),
           "cavity24_fp64": ifc.cavity2d(24), "channel200x70": ifc.channel2d(200, 70)}[case]
    cfg = dict(cfg, precision=prec, numOuterIter=400)
    s = ifc.Solver(cfg)
    s.solve()
    t0 = s.get("T").copy()
    r = s.solve_energy(max_sweeps=37, tol=0.0)
    assert r["sweeps"] == 37
    wf = s.get("wf") if cfg["dim"] == 3 else None
    coef, src = O.energy_assemble(cfg, s.get("uf"), s.get("vf"), wf, prec)
    t, _ = O.energy_sweeps(cfg, coef, src, t0, 37, prec)
    assert_bitwise(s.get("T"), t, "T")


def test_energy_converges_within_wall_temperatures(gpu_ok):
    cfg = ifc.cavity2d(32, re=100.0)
    s = ifc.Solver(cfg)
    s.solve()
    r = s.solve_energy(max_sweeps=50000, tol=1e-6)
    assert r["status"] == ifc.OK and r["converged"], r
    t = s.get("T")
    # maximum principle: no source, so T stays within the Dirichlet values
    assert t.min() >= 293.0 - 1e-3 and t.max() <= 373.0 + 1e-3
    # heat enters at the hot south wall: the bottom row is warmer than the top row
    tt = t.reshape(32, 32)
    assert tt[0].mean() > tt[-1].mean()


@pytest.mark.parametrize("scheme", ["quick", "van_leer"])
@pytest.mark.parametrize("case", ["channel48x16", "cavity3d8", "cavity24_fp64"])
def test_energy_dc_cycles_match_oracle(gpu_ok, energy_form, case, scheme):
    """Higher-order convection of T: every cycle of 25 sweeps starts from the
    source plus the deferred correction of the current T.  With tol 0 the
    cycles are fixed (25, 25, 10) and the device matches the numpy restatement
    bit for bit."""
    prec = "d" if case.endswith("fp64") else "f"
    cfg = {"channel48x16": ifc.channel2d(48, 16), "cavity3d8": ifc.cavity3d(8),
           "cavity24_fp64": ifc.cavity2d(24)}[case]
    cfg = dict(cfg, precision=prec, numOuterIter=400, convection_scheme=scheme)
    s = ifc.Solver(cfg)
    s.solve()
    t0 = s.get("T").copy()
    r = s.solve_energy(max_sweeps=60, tol=0.0)
    assert r["sweeps"] == 60
    wf = s.get("wf") if cfg["dim"] == 3 else None
    coef, src = O.energy_assemble(cfg, s.get("uf"), s.get("vf"), wf, prec)
    t = O.energy_dc_sweeps(cfg, coef, src, s.get("uf"), s.get("vf"), wf, t0, 60, prec)
    assert_bitwise(s.get("T"), t, "T")


def test_energy_dc_converges(gpu_ok):
    """With QUICK the cycles run until a fresh correction moves T by less than
    the tolerance in one sweep; the result is the fixed point: one more cycle
    (restated on the host) changes it by at most that much."""
    cfg = dict(ifc.cavity2d(32, re=100.0), convection_scheme="quick", precision="d")
    s = ifc.Solver(cfg)
    s.solve()
    r = s.solve_energy(max_sweeps=50000, tol=1e-9)
    assert r["status"] == ifc.OK and r["converged"], r
    t = s.get("T")
    coef, src = O.energy_assemble(cfg, s.get("uf"), s.get("vf"), None, "d")
    t2 = O.energy_dc_sweeps(cfg, coef, src, s.get("uf"), s.get("vf"), None, t, 25, "d")
    assert np.abs(t2 - t).max() <= 1e-5 * (np.abs(t).max() - np.abs(t).min())
    assert t.min() >= 293.0 - 0.5 and t.max() <= 373.0 + 0.5

"""Higher-order convection by deferred correction, on the CPU oracle (no GPU).

The reference has first-order upwind convection only; the deferred-correction
source restated in the oracle (ifc_oracle_impl.h, dc_source) is checked here
against closed-form answers:
- on a linear profile every scheme's face value is the linear one, so only the
  cells next to a face that keeps the upwind value carry a correction, of
  known size -F h / 2 and +F h / 2;
- across a step the TVD limiters (minmod, van Leer) add nothing, QUICK does;
- the corrections of interior faces cancel in the domain sum (conservation);
- on a lid-driven cavity the higher-order schemes land closer to a finer
  grid's solution than upwind does.
Tolerances are written in each test.
"""
import ctypes as C

import numpy as np
import pytest

import ifc
import oracle as O
from helpers import to_oracle_cfg

SCHEMES = ["central", "sou", "quick", "minmod", "van_leer"]


def _dc(cfg, fields, prec="d"):
    """Deferred-correction source of u and v for the given fields (the
    difference of the momentum sources after and before dc_source)."""
    o = O.Oracle(to_oracle_cfg(cfg), prec)
    for k, v in fields.items():
        o.field(k)[:] = v
    o.mom_link_coef()
    o.mom_src()
    o.bc_mom()
    before = {k: o.field(k).astype(np.float64).copy() for k in ("src_u", "src_v")}
    o.dc_source()
    return {k: o.field(k).astype(np.float64) - before[k] for k in before}, o


def _channel(nx, ny, scheme):
    return ifc.channel2d(nx, ny, density=2.0, dynamicViscosity=0.01, xmin=0.0, xmax=float(nx), ymin=0.0,
                         ymax=float(ny), convection_scheme=scheme)


@pytest.mark.parametrize("scheme", SCHEMES)
def test_linear_profile_known_answer(scheme):
    nx, ny = 12, 5
    cfg = _channel(nx, ny, scheme)
    h = 0.25
    x = np.arange(nx, dtype=np.float64)
    u = np.tile(h * x, ny)                       # linear in x, uniform in y
    uf = np.full((ny, nx + 1), 1.5)             # uniform flow in +x on every x-face
    vf = np.zeros((ny + 1, nx))
    dc, o = _dc(cfg, {"u": u, "v": np.zeros(nx * ny), "uf": uf.ravel(), "vf": vf.ravel()})
    F = 2.0 * 1.5 * 1.0                         # rho * u_f * A (dy = dz = 1)
    want = np.zeros((ny, nx))
    want[:, 1] = -F * 0.5 * h                   # its west face keeps the upwind value
    want[:, nx - 1] = F * 0.5 * h               # its east face is the boundary
    # tolerance: a few FP64 ulps of the source magnitude
    np.testing.assert_allclose(dc["src_u"].reshape(ny, nx), want, rtol=0, atol=1e-13)
    assert np.all(dc["src_v"] == 0.0)


@pytest.mark.parametrize("scheme", SCHEMES)
def test_reversed_flow_mirrors(scheme):
    """The same linear profile under flow in -x: the upwind side flips, so the
    face next to the east boundary keeps the upwind value and the first
    correction sits in cell 0 (-q) and cell nx-2 (+q), q = F (0.5 (-h))."""
    nx, ny = 10, 4
    cfg = _channel(nx, ny, scheme)
    h = 0.5
    u = np.tile(h * np.arange(nx, dtype=np.float64), ny)
    uf = np.full((ny, nx + 1), -0.75)
    dc, _ = _dc(cfg, {"u": u, "v": np.zeros(nx * ny), "uf": uf.ravel(), "vf": np.zeros((ny + 1) * nx)})
    q = (2.0 * -0.75) * (0.5 * -h)
    want = np.zeros((ny, nx))
    want[:, 0] = -q
    want[:, nx - 2] = q
    np.testing.assert_allclose(dc["src_u"].reshape(ny, nx), want, rtol=0, atol=1e-13)


def test_step_tvd_limiters_add_nothing():
    nx, ny = 16, 3
    u = np.tile(np.where(np.arange(nx) < 7, 0.0, 1.0), ny)
    flds = {"u": u, "v": np.zeros(nx * ny), "uf": np.full((ny, nx + 1), 1.0).ravel(),
            "vf": np.zeros((ny + 1) * nx)}
    for scheme in ("minmod", "van_leer"):
        dc, _ = _dc(_channel(nx, ny, scheme), flds)
        assert np.all(dc["src_u"] == 0.0), scheme
    dc, _ = _dc(_channel(nx, ny, "quick"), flds)
    assert np.abs(dc["src_u"]).max() > 0.1


@pytest.mark.parametrize("scheme", SCHEMES)
def test_corrections_are_conservative(scheme):
    """Every interior face adds +Q to one cell and -Q to the other, so the
    domain sum vanishes (tolerance: FP64 rounding of the sum)."""
    cfg = dict(ifc.cavity2d(14, ny=11), convection_scheme=scheme)
    rng = np.random.default_rng(4)
    flds = {"u": rng.uniform(-1, 1, 154), "v": rng.uniform(-1, 1, 154),
            "uf": rng.uniform(-1, 1, 15 * 11), "vf": rng.uniform(-1, 1, 14 * 12)}
    dc, _ = _dc(cfg, flds)
    for k in dc:
        assert abs(dc[k].sum()) <= 1e-12 * np.abs(dc[k]).sum(), k
        assert np.abs(dc[k]).max() > 0


def test_upwind_adds_nothing():
    cfg = dict(ifc.cavity2d(9), convection_scheme="upwind")
    rng = np.random.default_rng(1)
    flds = {"u": rng.uniform(-1, 1, 81), "v": rng.uniform(-1, 1, 81),
            "uf": rng.uniform(-1, 1, 90), "vf": rng.uniform(-1, 1, 90)}
    dc, _ = _dc(cfg, flds, "f")
    assert all(np.all(v == 0.0) for v in dc.values())


def _restrict(a, n):
    """2x2 average of an (2n x 2n) cell field onto the n x n grid."""
    return a.reshape(n, 2, n, 2).mean(axis=(1, 3))


def test_higher_order_schemes_converge_faster_on_the_cavity():
    """Lid-driven cavity, Re 100: the 24^2 solution of each higher-order
    scheme is closer (relative L2 of u, after 2x2 restriction of the 48^2
    QUICK solution) than the 24^2 upwind solution, by at least 1.5x."""
    re, n = 100.0, 24

    def solve(nn, scheme):
        cfg = dict(ifc.cavity2d(nn, re=re), convection_scheme=scheme)
        o = O.Oracle(to_oracle_cfg(dict(cfg, sweep_mode=O.GS_LEX)), "d")
        its, nm = o.solve()
        assert nm["converged"], (nn, scheme)
        return o.field("u").reshape(nn, nn).copy()

    fine = _restrict(solve(2 * n, "quick"), n)
    err = {s: np.linalg.norm(solve(n, s) - fine) / np.linalg.norm(fine) for s in ["upwind", "quick", "van_leer"]}
    assert err["quick"] * 1.5 < err["upwind"], err
    assert err["van_leer"] * 1.5 < err["upwind"], err


def test_scheme_range_is_checked():
    """Validation happens before any device work, so this runs without a GPU."""
    lib = ifc.load()
    cfg = dict(ifc.cavity2d(16), convection_scheme="quick")
    s, _ = ifc.make_struct(cfg)
    assert lib.ifc_config_check(C.byref(s)) == ifc.OK
    for bad in (-1, 6):
        s.convection_scheme = bad
        assert lib.ifc_config_check(C.byref(s)) == ifc.BAD_CONFIG


@pytest.mark.parametrize("prec", ["f", "d"])
@pytest.mark.parametrize("scheme", SCHEMES)
def test_energy_restatement_equals_momentum_restatement(scheme, prec):
    """The numpy correction used for the temperature (oracle.energy_dc) and the
    C oracle's momentum correction are the same formula: on the same field and
    faces they agree bit for bit."""
    cfg = dict(ifc.cavity2d(13, ny=10), convection_scheme=scheme)
    rng = np.random.default_rng(8)
    T = np.float32 if prec == "f" else np.float64
    flds = {"u": rng.uniform(-1, 1, 130).astype(T), "v": np.zeros(130, T),
            "uf": rng.uniform(-1, 1, 14 * 10).astype(T), "vf": rng.uniform(-1, 1, 13 * 11).astype(T)}
    o = O.Oracle(to_oracle_cfg(cfg), prec)
    for k, v in flds.items():
        o.field(k)[:] = v
    o.field("src_u")[:] = 0
    o.field("src_v")[:] = 0
    o.dc_source()
    ref = o.field("src_u").copy()            # 0 + dc, exact
    got = O.energy_dc(cfg, flds["uf"], flds["vf"], None, flds["u"], prec)
    assert np.array_equal(got.astype(T), ref.astype(T))


def test_energy_quick_beats_upwind_on_advection_diffusion():
    """Steady 1D advection-diffusion between Dirichlet walls (uniform flow U,
    Peclet number 5): T = T0 + (T1 - T0) (exp(Pe x) - 1)/(exp(Pe) - 1).  Max
    cell error, FP64, at 24 and 48 cells: upwind converges at first order (error
    ratio below 2.2), QUICK by deferred correction at second order (ratio above
    3) and is at least 4x closer at 24 cells."""
    Pe, ny, U, rho, L = 5.0, 3, 1.0, 1.0, 1.0
    gam = rho * U * L / Pe
    err = {}
    for nx in (24, 48):
        cfg = dict(ifc.channel2d(nx, ny), xmin=0.0, xmax=L, ymin=0.0, ymax=ny * L / nx, density=rho,
                   thermalConductivity=gam, specificHeatCapacity=1.0,
                   TempBC_type=[0, 0, 1, 1, 1, 1], TempBC_val=[1.0, 0.0, 0.0, 0.0, 0.0, 0.0])
        uf = np.full((ny, nx + 1), U)
        vf = np.zeros((ny + 1, nx))
        x = (np.arange(nx) + 0.5) / nx
        exact = (np.exp(Pe * x) - 1.0) / (np.exp(Pe) - 1.0)
        for scheme in ("upwind", "quick"):
            c = dict(cfg, convection_scheme=scheme)
            coef, src = O.energy_assemble(c, uf.ravel(), vf.ravel(), None, "d")
            t0 = np.zeros(nx * ny)
            if scheme == "upwind":
                t, _ = O.energy_sweeps(c, coef, src, t0, 8000, "d")
            else:
                t = O.energy_dc_sweeps(c, coef, src, uf.ravel(), vf.ravel(), None, t0, 8000, "d")
            err[scheme, nx] = np.abs(t.reshape(ny, nx)[1] - exact).max()
    assert err["upwind", 24] / err["upwind", 48] < 2.2, err
    assert err["quick", 24] / err["quick", 48] > 3.0, err
    assert err["quick", 24] * 4.0 < err["upwind", 24], err

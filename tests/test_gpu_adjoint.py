"""Discrete adjoint on the GPU (ifc_adjoint / ifc_adjoint_apply through the
C ABI) against the oracle's reverse pass and against central finite
differences of FP64 solves.

Tolerances: one reverse pass agrees with the oracle's to 1e-10 relative (the
device gathers where the oracle scatters, so the FP64 sums are ordered
differently); the adjoint gradient agrees with the oracle's to 1e-8 and with
central finite differences (relative step 1e-3) to 1e-4 relative, the
differentiation form's bound.  The torch.autograd.Function below exists only
in this test harness: it wraps the C ABI so that torch's gradcheck can drive
the adjoint.
"""
import numpy as np
import pytest
import torch

import ifc
import oracle as O
from helpers import to_oracle_cfg

pytestmark = pytest.mark.gpu

KEYS = ("u", "v", "p", "uf", "vf")


def _channel(nx, ny, seed=0, **kw):
    rng = np.random.default_rng(seed)
    theta = 0.001 + rng.normal(0, 1e-4, ny)
    opts = dict(precision="d", tol_u=0, tol_v=0, tol_p=0, tol_mass=0)
    opts.update(kw)
    return ifc.channel2d(nx, ny, inlet_profile=theta, **opts), theta


@pytest.fixture(params=["single_launch", "graph"])
def adjoint_form(request, monkeypatch):
    """Both device forms of the adjoint: the cooperative single-launch solve
    and the graph of per-step kernels (chosen when a handle first calls the
    adjoint)."""
    if request.param == "graph":
        monkeypatch.setenv("IFC_ADJOINT_GRAPH", "1")
    else:
        monkeypatch.delenv("IFC_ADJOINT_GRAPH", raising=False)
    return request.param


def _state(s):
    return {k: s.get(k).astype(np.float64) for k in KEYS}


def _oracle_at(cfg, state):
    oc = to_oracle_cfg(cfg)
    if cfg.get("precision", "f") not in ("d", 1, "fp64", "double") and cfg.get("inlet_profile") is not None:
        # an FP32 handle holds its inlet profile in FP32
        oc["inlet_profile"] = np.asarray(cfg["inlet_profile"], dtype=np.float32).astype(np.float64)
    o = O.AdjointOracle(oc)
    for k in KEYS:
        o.field(k)[:] = state[k]
    return o


def _random_seed(nx, ny, rng):
    lam = {k: rng.standard_normal(n) for k, n in
           {"u": nx * ny, "v": nx * ny, "p": nx * ny, "uf": (nx + 1) * ny, "vf": nx * (ny + 1)}.items()}
    lam["uf"].reshape(ny, nx + 1)[:, [0, -1]] = 0.0
    lam["vf"].reshape(ny + 1, nx)[[0, -1], :] = 0.0
    return lam


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("case", ["channel24x10", "cavity16", "channel20x8_fp32"])
def test_reverse_pass_matches_oracle(gpu_ok, adjoint_form, case):
    if case == "channel24x10":
        cfg, _ = _channel(24, 10)
    elif case == "channel20x8_fp32":
        cfg, _ = _channel(20, 8, precision="f")
    else:
        cfg = dict(ifc.cavity2d(16), precision="d", tol_u=0, tol_v=0, tol_p=0, tol_mass=0)
    nx, ny = cfg["nx"], cfg["ny"]
    s = ifc.Solver(cfg)
    s.iterate(2000)
    st = _state(s)
    o = _oracle_at(cfg, st)
    rng = np.random.default_rng(5)
    for _ in range(2):
        lam = _random_seed(nx, ny, rng)
        dev, dth, dmu = s.adjoint_apply(lam)
        ref, rth, rmu = o.apply_transpose(lam)
        for k in KEYS:
            assert _rel(dev[k], ref[k]) < 1e-10, (k, _rel(dev[k], ref[k]))
        if cfg["velBC_type"][ifc.WEST] == ifc.INLET:
            assert _rel(dth, rth) < 1e-10
        assert abs(dmu - rmu) <= 1e-10 * abs(rmu)


def test_gradient_matches_oracle(gpu_ok, adjoint_form):
    cfg, _ = _channel(24, 10)
    s = ifc.Solver(cfg)
    s.iterate(20000)
    dth, res = s.adjoint(tol=1e-12)
    assert res["status"] == ifc.OK and res["converged"], res
    o = _oracle_at(cfg, _state(s))
    rth, rmu, its = o.adjoint_gradient(tol=1e-12)
    assert _rel(dth, rth) < 1e-8
    assert abs(res["dJ_dmu"] - rmu) <= 1e-8 * abs(rmu)
    assert abs(res["iterations"] - its) <= 2, (res["iterations"], its)
    assert abs(res["objective"] - o.objective()) <= 1e-12 * abs(o.objective())


def _solve_J(cfg, theta, mu, start, n_iter):
    c = dict(cfg, inlet_profile=np.asarray(theta, dtype=np.float64), dynamicViscosity=float(mu))
    s = ifc.Solver(c)
    if start is not None:
        for k in KEYS:
            s.set(k, start[k])
    s.iterate(n_iter)
    p = s.get("p").reshape(cfg["ny"], cfg["nx"])
    return float(p[:, 0].mean() - p[:, -1].mean()), s


class PressureDrop(torch.autograd.Function):
    """J(theta, mu) through the C ABI: forward solves, backward returns the
    adjoint gradient.  Test-harness only."""

    cfg = None
    n_iter = 0
    start = None

    @staticmethod
    def forward(ctx, theta, mu):
        J, s = _solve_J(PressureDrop.cfg, theta.detach().cpu().numpy(), mu.item(), PressureDrop.start,
                        PressureDrop.n_iter)
        dth, res = s.adjoint(tol=1e-12)
        assert res["converged"]
        ctx.save_for_backward(torch.from_numpy(dth), torch.tensor(res["dJ_dmu"], dtype=torch.float64))
        return torch.tensor(J, dtype=torch.float64)

    @staticmethod
    def backward(ctx, g):
        dth, dmu = ctx.saved_tensors
        return g * dth, g * dmu


def test_gradient_matches_central_differences(gpu_ok):
    cfg, theta = _channel(32, 8, seed=11)
    mu = cfg["dynamicViscosity"]
    J0, s = _solve_J(cfg, theta, mu, None, 40000)
    base = _state(s)
    dth, res = s.adjoint(tol=1e-12)
    assert res["converged"]
    fd = np.empty_like(theta)
    for j in range(theta.size):
        h = 1e-3 * theta[j]
        tp, tm = theta.copy(), theta.copy()
        tp[j] += h
        tm[j] -= h
        fd[j] = (_solve_J(cfg, tp, mu, base, 20000)[0] - _solve_J(cfg, tm, mu, base, 20000)[0]) / (2 * h)
    assert _rel(dth, fd) <= 1e-4, (dth, fd)
    h = 1e-3 * mu
    fdmu = (_solve_J(cfg, theta, mu + h, base, 20000)[0] - _solve_J(cfg, theta, mu - h, base, 20000)[0]) / (2 * h)
    assert abs(res["dJ_dmu"] - fdmu) <= 1e-4 * abs(fdmu)


def test_autograd_function_gradcheck(gpu_ok):
    cfg, theta = _channel(16, 6, seed=2)
    mu = cfg["dynamicViscosity"]
    _, s = _solve_J(cfg, theta, mu, None, 40000)
    PressureDrop.cfg, PressureDrop.n_iter, PressureDrop.start = cfg, 20000, _state(s)
    th = torch.tensor(theta, dtype=torch.float64, requires_grad=True)
    m = torch.tensor(mu, dtype=torch.float64, requires_grad=True)
    # Absolute steps of 1e-6 are relative steps of about 1e-3 for theta and mu.
    assert torch.autograd.gradcheck(PressureDrop.apply, (th, m), eps=1e-6, atol=1e-6, rtol=1e-4)


def test_adjoint_is_deterministic_and_rejects_3d(gpu_ok):
    cfg, _ = _channel(24, 10)
    s = ifc.Solver(cfg)
    s.iterate(3000)
    a, ra = s.adjoint(tol=1e-9)
    b, rb = s.adjoint(tol=1e-9)
    assert np.array_equal(a, b) and ra["dJ_dmu"] == rb["dJ_dmu"] and ra["iterations"] == rb["iterations"]
    s3 = ifc.Solver(ifc.cavity3d(8))
    with pytest.raises(ifc.IfcError):
        s3.adjoint()


def test_set_inlet_profile_matches_a_new_handle(gpu_ok):
    cfg, theta = _channel(24, 10, precision="f", tol_u=1e-5, tol_v=1e-5, tol_p=1e-5)
    s = ifc.Solver(cfg)
    s.solve()
    theta2 = theta * 1.1
    s.set_inlet_profile(theta2)
    s.set_uniform()
    s.solve()
    t = ifc.Solver(dict(cfg, inlet_profile=theta2))
    t.solve()
    for k in ("u", "v", "p"):
        assert np.array_equal(s.get(k), t.get(k))
    a, _ = s.adjoint(tol=1e-9)
    b, _ = t.adjoint(tol=1e-9)
    assert np.array_equal(a, b)
    with pytest.raises(ifc.IfcError):
        ifc.Solver(ifc.channel2d(24, 10)).set_inlet_profile(theta)

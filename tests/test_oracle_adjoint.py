"""The oracle's discrete adjoint on its own (no GPU): the reverse pass is the
transpose of one linearised SIMPLE outer iteration, and the adjoint gradient
of J = mean p(first column) - mean p(last column) matches central finite
differences in FP64."""
import numpy as np
import pytest

import ifc
import oracle as O
from helpers import to_oracle_cfg


def _channel(nx=12, ny=6, seed=0, **kw):
    rng = np.random.default_rng(seed)
    theta = 0.001 + rng.normal(0, 1e-4, ny)
    cfg = ifc.channel2d(nx, ny, inlet_profile=theta, tol_u=0, tol_v=0, tol_p=0, tol_mass=0, **kw)
    oc = to_oracle_cfg(cfg)
    oc["check_every"] = 1
    return oc, theta


def _zero_boundary_faces(x, nx, ny):
    x["uf"].reshape(ny, nx + 1)[:, [0, -1]] = 0.0
    x["vf"].reshape(ny + 1, nx)[[0, -1], :] = 0.0


def _state(o, sz):
    return {k: o.field(k).copy() for k in sz}


def _transpose_gap(oc, nx, ny, n_primal):
    """<lambda, G_x dx> (central difference of one outer iteration) against
    <G_x^T lambda, dx> at the converged state."""
    rng = np.random.default_rng(7)
    o = O.AdjointOracle(oc)
    o.solve(n_primal)
    sz = o.state_sizes()
    x0 = _state(o, sz)
    lam = {k: rng.standard_normal(n) for k, n in sz.items()}
    dx = {k: rng.standard_normal(n) for k, n in sz.items()}
    _zero_boundary_faces(lam, nx, ny)
    _zero_boundary_faces(dx, nx, ny)
    out, _, _ = o.apply_transpose(lam)
    scal = {k: np.abs(x0[k]).max() + 1e-12 for k in sz}

    def G(xs):
        o2 = O.AdjointOracle(oc)
        o2.set_iteration_count(5)
        for k in sz:
            o2.field(k)[:] = xs[k]
        o2.outer_iteration()
        return _state(o2, sz)

    eps = 1e-7
    gp = G({k: x0[k] + eps * scal[k] * dx[k] for k in sz})
    gm = G({k: x0[k] - eps * scal[k] * dx[k] for k in sz})
    lhs = sum((lam[k] * (gp[k] - gm[k]) / (2 * eps)).sum() for k in sz)
    rhs = sum((out[k] * dx[k] * scal[k]).sum() for k in sz)
    return abs(lhs - rhs) / abs(rhs)


def test_reverse_pass_is_the_transpose_channel():
    oc, _ = _channel()
    assert _transpose_gap(oc, 12, 6, 30000) < 1e-7


def test_reverse_pass_is_the_transpose_cavity():
    cfg = ifc.cavity2d(8, re=100.0, tol_u=0, tol_v=0, tol_p=0, tol_mass=0)
    oc = to_oracle_cfg(cfg)
    oc["check_every"] = 1
    assert oc["pin_pressure"] == 1
    assert _transpose_gap(oc, 8, 8, 20000) < 1e-7


def _fd_objective(oc, x0, sz, n_primal):
    o2 = O.AdjointOracle(oc)
    for k in sz:
        o2.field(k)[:] = x0[k]
    o2.set_iteration_count(5)
    o2.solve(n_primal)
    return o2.objective()


def test_adjoint_gradient_matches_central_differences():
    oc, theta = _channel()
    o = O.AdjointOracle(oc)
    o.solve(30000)
    sz = o.state_sizes()
    x0 = _state(o, sz)
    lth, lmu, its = o.adjoint_gradient()
    assert its < 100000
    fd = np.empty_like(theta)
    for j in range(theta.size):
        h = 1e-3 * theta[j]
        Js = []
        for sgn in (1, -1):
            th = theta.copy()
            th[j] += sgn * h
            Js.append(_fd_objective(dict(oc, inlet_profile=th), x0, sz, 30000))
        fd[j] = (Js[0] - Js[1]) / (2 * h)
    assert np.abs(lth - fd).max() <= 1e-4 * np.abs(fd).max()
    mu = oc["dynamicViscosity"]
    h = 1e-3 * mu
    Jp = _fd_objective(dict(oc, dynamicViscosity=mu + h), x0, sz, 30000)
    Jm = _fd_objective(dict(oc, dynamicViscosity=mu - h), x0, sz, 30000)
    fdmu = (Jp - Jm) / (2 * h)
    assert abs(lmu - fdmu) <= 1e-4 * abs(fdmu)


def test_reverse_pass_is_linear_in_the_seed():
    oc, _ = _channel(10, 5, seed=3)
    o = O.AdjointOracle(oc)
    o.solve(2000)
    sz = o.state_sizes()
    rng = np.random.default_rng(1)
    a = {k: rng.standard_normal(n) for k, n in sz.items()}
    b = {k: rng.standard_normal(n) for k, n in sz.items()}
    _zero_boundary_faces(a, 10, 5)
    _zero_boundary_faces(b, 10, 5)
    oa, ta, ma = o.apply_transpose(a)
    ob, tb, mb = o.apply_transpose(b)
    oab, tab, mab = o.apply_transpose({k: 2.0 * a[k] - 3.0 * b[k] for k in sz})
    for k in sz:
        assert np.allclose(oab[k], 2.0 * oa[k] - 3.0 * ob[k], rtol=1e-12, atol=1e-12 * np.abs(oab[k]).max())
    assert np.allclose(tab, 2.0 * ta - 3.0 * tb, rtol=1e-12, atol=1e-15)
    assert abs(mab - (2.0 * ma - 3.0 * mb)) <= 1e-10 * (abs(mab) + 1e-30)


def test_adjoint_rejects_3d():
    cfg = to_oracle_cfg(ifc.cavity3d(4))
    o = O.AdjointOracle(cfg)
    with pytest.raises(AssertionError):
        o.apply_transpose({k: np.zeros(n) for k, n in o.state_sizes().items()})

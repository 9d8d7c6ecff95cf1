"""The CPU oracle on its own (no GPU): properties of the restated method that
hold at any size, and agreement between its orderings and precisions."""
import numpy as np
import pytest

import ifc
import oracle as O
from cases import small_cases
from helpers import rel_l2, seeded_state, to_oracle_cfg


@pytest.mark.parametrize("name", list(small_cases()))
def test_coefficient_identities(name):
    cfg = to_oracle_cfg(small_cases()[name])
    o = O.Oracle(cfg, "d")
    for k, v in seeded_state(cfg, 5, np.float64).items():
        o.field(k)[:] = v
    o.mom_link_coef()
    N, nc = o.N, 2 * cfg["dim"] + 1
    a = o.field("mcoef").reshape(nc, N)
    # before the fold-in aC = -sum(a_nb) exactly as computed
    assert np.allclose(a[0], -a[1:].sum(0), rtol=1e-13, atol=1e-13)
    assert (a[1:] < 0).all()
    o.mom_src(); o.bc_mom()
    o.pcorr_link_coef()
    pcoef = o.field("pcoef").reshape(nc, N)
    # p' links are symmetric: aE(C) == aW(E)
    nx = cfg["nx"]
    pe = pcoef[1].reshape(-1, nx)[:, :-1]
    pw = pcoef[2].reshape(-1, nx)[:, 1:]
    assert np.array_equal(pe, pw)
    assert np.allclose(pcoef[0], -pcoef[1:].sum(0), rtol=1e-12, atol=1e-300)


def test_mass_imbalance_sums_to_boundary_flux():
    cfg = to_oracle_cfg(ifc.channel2d(24, 10))
    o = O.Oracle(cfg, "d")
    for k, v in seeded_state(cfg, 2, np.float64).items():
        o.field(k)[:] = v
    o.bc_face_vel()
    o.pcorr_src()
    b = o.field("src_p")
    nx, ny = 24, 10
    uf = o.field("uf").reshape(ny, nx + 1)
    vf = o.field("vf").reshape(ny + 1, nx)
    dy = 0.025 / ny
    dx = 0.125 / nx
    flux = 998.2 * (dy * (uf[:, 0].sum() - uf[:, -1].sum()) + dx * (vf[0].sum() - vf[-1].sum()))
    assert abs(b.sum() - flux) < 1e-9 * (np.abs(b).sum() + 1e-30)


@pytest.mark.parametrize("mode", [O.GS_REDBLACK, O.GS_LEX, O.JACOBI])
def test_sweeps_reduce_residual(mode):
    cfg = to_oracle_cfg(ifc.cavity2d(16))
    o = O.Oracle(cfg, "d")
    for k, v in seeded_state(cfg, 4, np.float64).items():
        o.field(k)[:] = v
    o.mom_link_coef(); o.mom_src(); o.bc_mom()
    sq = [o.sweep(O.EQ_U, mode) for _ in range(300)]
    assert sq[-1] < sq[0] * 1e-3


def test_converged_cavity_orderings_and_precisions_agree():
    """64x64 lid-driven cavity (Re=100) to residual 1e-5: red-black vs
    lexicographic Gauss-Seidel and float vs double reach the same fixed point
    within relative L2 1e-4 (p compared after removing its mean)."""
    base = ifc.cavity2d(64)
    res = {}
    for mode in (O.GS_REDBLACK, O.GS_LEX):
        for prec in ("f", "d"):
            o = O.Oracle(to_oracle_cfg(dict(base, sweep_mode=mode)), prec)
            n, nm = o.solve()
            assert nm["converged"], (mode, prec, n)
            p = o.field("p").astype(np.float64)
            res[(mode, prec)] = (o.field("u").copy(), o.field("v").copy(), p - p.mean())
    ref = res[(O.GS_LEX, "d")]
    for key, val in res.items():
        for a, b in zip(val, ref):
            assert rel_l2(a, b) < 1e-4, key
    u = res[(O.GS_REDBLACK, "f")][0].reshape(64, 64)
    # Re=100 cavity, first-order upwind on 64^2: min u on the vertical centre line
    assert -0.25 < u[:, 31:33].min() < -0.19


def test_residual_rule_restatement():
    """The residual rule of the oracle: the FP64 momentum residual it reports is
    the residual of the assembled equations at the iteration's starting field
    (recomputed here with numpy from the coefficient planes), and a 24^2
    cavity stopped by it agrees with the per-field rule's answer to 1e-4."""
    cfg = dict(ifc.cavity2d(24), criterion=O.CRIT_RESIDUAL)
    o = O.Oracle(to_oracle_cfg(cfg), "d")
    o.solve(30)
    u0, v0 = o.field("u").copy(), o.field("v").copy()
    nm = o.outer_iteration()
    # the coefficients of that iteration are still in the planes
    N = 24 * 24
    a = o.field("mcoef").reshape(5, N)
    for x, b, res in ((u0, o.field("src_u"), nm["res_u"]), (v0, o.field("src_v"), nm["res_v"])):
        X = x.reshape(24, 24)
        E = np.zeros_like(X); E[:, :-1] = X[:, 1:]
        W = np.zeros_like(X); W[:, 1:] = X[:, :-1]
        Nn = np.zeros_like(X); Nn[:-1, :] = X[1:, :]
        S = np.zeros_like(X); S[1:, :] = X[:-1, :]
        r = b - a[0] * x - a[1] * E.ravel() - a[2] * W.ravel() - a[3] * Nn.ravel() - a[4] * S.ravel()
        assert abs(np.sqrt(np.mean(r ** 2)) - res) <= 1e-12 * max(res, 1e-300) + 1e-300
    o2 = O.Oracle(to_oracle_cfg(cfg), "d")
    n, nm2 = o2.solve()
    assert nm2["converged"]
    o3 = O.Oracle(to_oracle_cfg(dict(cfg, criterion=O.CRIT_PER_FIELD)), "d")
    o3.solve()
    for k in ("u", "v"):
        assert rel_l2(o2.field(k), o3.field(k)) < 1e-4, k


def test_openmp_build_matches_the_serial_oracle(tmp_path):
    """The OpenMP build of the oracle (the all-cores CPU baseline of bench.py)
    computes every cell as the serial build does: after outer iterations with
    every inner sweep run (no early exit), the fields are the same bits."""
    import os
    import subprocess
    import sys

    import ifc
    from helpers import to_oracle_cfg

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    subprocess.run(["make", "-s", "-C", os.path.join(root, "oracle"), "oracle_omp"], check=True)
    cfg = dict(ifc.channel2d(48, 20, nIter_u=3, nIter_v=3, nIter_p=6), tol_u=0.0, tol_v=0.0, tol_p=0.0)
    out = tmp_path / "omp.npz"
    code = ("import sys, numpy as np; sys.path[:0] = %r; import ifc, oracle as O; from helpers import to_oracle_cfg; "
            "o = O.Oracle(to_oracle_cfg(%r), 'f'); [o.outer_iteration() for _ in range(5)]; "
            "np.savez(%r, **{k: o.field(k) for k in ('u', 'v', 'p', 'uf', 'vf')}); print(O.LIB_PATH)"
            % ([os.path.join(root, "oracle"), os.path.join(root, "tests"),
                os.path.join(root, "incompflow-cuda_b200", "python")], cfg, str(out)))
    env = dict(os.environ, IFC_ORACLE_LIB=os.path.join(root, "oracle", "_build", "libifc_oracle_omp.so"),
               OMP_NUM_THREADS="4")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "_omp.so" in r.stdout, r.stdout + r.stderr
    o = O.Oracle(to_oracle_cfg(cfg), "f")
    for _ in range(5):
        o.outer_iteration()
    got = np.load(out)
    for k in ("u", "v", "p", "uf", "vf"):
        np.testing.assert_array_equal(got[k], o.field(k), err_msg=k)

"""The CPU oracle against the reference itself (no GPU needed here).

Fixtures in tests/golden/ were produced by tests/golden/make_golden.py from
the reference's own CUDA build (its sources compiled by oracle/build_ref.py
and run on a B200):

* ref_kernels_<case>.npz -- seeded inputs and the outputs of the reference's
  kernels, launched one by one with the reference's launch shapes;
* ref_solve_<case>.npz -- the reference's converged u, v, p (Solver::solve()
  for 3000 outer iterations, far past convergence), read from its VTK output
  with 6 significant digits.

Step tolerances: the reference was compiled with nvcc's default FMA
contraction while the oracle rounds every operation as written, so values may
differ by a few units in the last place; each comparison allows 8 float ulps
of the value's magnitude (plus 8 ulps of the array's scale for values that
cancel to near zero).  Converged fields: relative L2 1e-5 at the same number of
outer iterations (pressure of the closed cavity compared after removing its
mean, since the reference never fixes its level).
"""
import os

import numpy as np
import pytest

import oracle as O
from helpers import rel_l2, to_oracle_cfg

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


def kernel_cases():
    import build_ref

    return build_ref.kernel_cases()


def fixture(name):
    path = os.path.join(GOLD, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not generated yet")
    return np.load(path)


def close(got, ref, what):
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    eps = np.finfo(np.float32).eps
    tol = 8 * eps * (np.abs(ref) + np.abs(ref).max())
    bad = np.abs(got - ref) > tol
    assert not bad.any(), f"{what}: {bad.sum()} of {ref.size} differ; worst {np.abs(got - ref).max():.3e}"


def fresh(cfg, g):
    o = O.Oracle(to_oracle_cfg(cfg), "f")
    for k in ("u", "v", "p", "pc", "uf", "vf"):
        o.field(k)[:] = g[f"in_{k}"]
    o.field("mcoef")[:] = g["in_coef"]
    return o


@pytest.mark.parametrize("name", ["mixed20x13", "cavity17x19"])
def test_oracle_steps_match_reference_kernels(name):
    g = fixture(f"ref_kernels_{name}.npz")
    cfg = kernel_cases()[name]

    o = fresh(cfg, g)
    o.init_face_vel()
    o.bc_face_vel()
    close(o.field("uf"), g["out_faces_uf"], "face init + BCs uf")
    close(o.field("vf"), g["out_faces_vf"], "face init + BCs vf")

    o = fresh(cfg, g)
    o.mom_link_coef()
    close(o.field("mcoef"), g["out_mom_coef_raw"], "momentum link coefficients")
    o.mom_src()
    o.bc_mom()
    close(o.field("mcoef"), g["out_mom_coef"], "coefficients after the fold-in")
    close(o.field("mcoef"), g["out_mom_vcoef"], "v coefficients (identical set)")
    close(o.field("src_u"), g["out_mom_src_u"], "u source")
    close(o.field("src_v"), g["out_mom_src_v"], "v source")
    o.sweep(O.EQ_U, O.JACOBI)
    close(o.field("u"), g["out_jacobi_u"], "one Jacobi sweep")

    o = fresh(cfg, g)
    o.rhie_chow()
    n_in = cfg["nx"] * cfg["ny"]
    uf, vf = o.field("uf"), o.field("vf")
    nx, ny = cfg["nx"], cfg["ny"]
    # the reference's Rhie-Chow kernels write interior faces only
    ref_uf = g["out_rc_uf"].reshape(ny, nx + 1)
    close(uf.reshape(ny, nx + 1)[:, 1:-1], ref_uf[:, 1:-1], "Rhie-Chow uf")
    close(vf.reshape(ny + 1, nx)[1:-1], g["out_rc_vf"].reshape(ny + 1, nx)[1:-1], "Rhie-Chow vf")

    o = fresh(cfg, g)
    o.pcorr_link_coef()
    close(o.field("pcoef"), g["out_pcorr_coef"], "p' link coefficients")
    o.pcorr_src()
    close(o.field("src_p"), g["out_pcorr_src"], "p' source")

    o = fresh(cfg, g)
    o.update_field()
    for k in ("p", "u", "v", "uf", "vf"):
        close(o.field(k), g[f"out_upd_{k}"], f"correction {k}")
    assert n_in == g["out_upd_p"].size


@pytest.mark.parametrize("mode", [O.GS_LEX, O.GS_REDBLACK])
@pytest.mark.parametrize("name,closed", [("cavity64", True), ("channel128x32", False)])
def test_oracle_converged_matches_reference_solve(name, closed, mode):
    """Same number of outer iterations as the reference run (3000, far past
    convergence); agreement is limited by the 6 significant digits of the
    reference's VTK output (~1e-6), so the bound is 1e-5."""
    import build_ref

    g = fixture(f"ref_solve_{name}.npz")
    cfg, n_outer = build_ref.cases()[name][:2]
    o = O.Oracle(to_oracle_cfg(dict(cfg, sweep_mode=mode, tol_u=0, tol_v=0, tol_p=0, tol_mass=0)), "f")
    n, _ = o.solve(n_outer)
    assert n == n_outer
    for k in ("u", "v"):
        assert rel_l2(o.field(k), g[k]) < 1e-5, (k, rel_l2(o.field(k), g[k]))
    p, pr = o.field("p").astype(np.float64), g["p"]
    if closed:
        p, pr = p - p.mean(), pr - pr.mean()
    assert rel_l2(p, pr) < 1e-5, rel_l2(p, pr)


def test_oracle_3d_matches_fp64_golden():
    """The 3D pin: the reference's own 3D build cannot run, so the 16^3
    cavity solved by the FP64 oracle (red-black, per-field rule) is committed
    as a fixture; the oracle must reproduce it (it is deterministic)."""
    import ifc

    g = fixture("oracle_cavity3d16.npz")
    o = O.Oracle(to_oracle_cfg(ifc.cavity3d(16)), "d")
    n, nm = o.solve()
    assert n == int(g["iterations"]) and nm["converged"] == int(g["converged"])
    for k in ("u", "v", "w", "p"):
        assert rel_l2(o.field(k), g[k]) < 1e-12, k

"""Higher-order convection (deferred correction) on the GPU against the oracle.

Every device path that assembles momentum adds the same correction, computed
in the same order, so the values must agree bit for bit (tolerance: exact):
- the materialised assembly (IFC_STAGE_MOM_ASSEMBLE, k_mom_assemble);
- the fused sweeps (IFC_STAGE_MOM_SOLVE: k_mom_pass2d in 2D, k_mom_half3d in 3D);
- whole outer iterations (the single-launch k_simple2d in 2D, the graph in 3D);
- Jacobi sweeps on materialised coefficients.
Converged solves agree with the oracle's like the upwind ones (relative L2
1e-6 against the same red-black ordering, 1e-4 against FP64 lexicographic).
"""
import numpy as np
import pytest

import ifc
import oracle as O
from cases import small_cases
from helpers import assert_bitwise, load_both, rel_l2, seeded_state, to_oracle_cfg

pytestmark = pytest.mark.gpu

SCHEMES = ["central", "sou", "quick", "minmod", "van_leer"]
CASES = small_cases()
UNPINNED = ["channel20x9", "mixed12x11", "channel7x5x6"]


def _keys(cfg):
    d3 = cfg["dim"] == 3
    return ["u", "v"] + (["w"] if d3 else []), ["uf", "vf"] + (["wf"] if d3 else [])


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("name", list(CASES))
def test_dc_assembly_and_fused_sweeps_bitwise(gpu_ok, name, scheme):
    cfg = dict(CASES[name], convection_scheme=scheme)
    o = O.Oracle(to_oracle_cfg(cfg), "f")
    s = ifc.Solver(cfg)
    load_both(o, s, seeded_state(cfg, 5, np.float32))
    vel, faces = _keys(cfg)
    s.stage("face_bc")
    o.init_face_vel()
    o.bc_face_vel()
    s.stage("mom_assemble")
    o.mom_link_coef()
    o.mom_src()
    o.bc_mom()
    o.dc_source()
    for k in ["src_u", "src_v"] + (["src_w"] if cfg["dim"] == 3 else []):
        assert_bitwise(s.get(k), o.field(k), f"{name} {scheme} {k}")
    s.stage("mom_solve")
    for eq in range(cfg["dim"]):
        o.linear_solve(eq)
    for k in vel:
        assert_bitwise(s.get(k), o.field(k), f"{name} {scheme} mom_solve {k}")


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("prec", ["f", "d"])
@pytest.mark.parametrize("name", UNPINNED)
def test_dc_outer_iterations_bitwise(gpu_ok, name, prec, scheme):
    cfg = dict(CASES[name], precision=prec, convection_scheme=scheme)
    o = O.Oracle(to_oracle_cfg(cfg), prec)
    s = ifc.Solver(cfg)
    load_both(o, s, seeded_state(cfg, 3, s.dtype))
    vel, faces = _keys(cfg)
    for it in range(3):
        s.iterate(1)
        o.outer_iteration()
        o.bc_face_vel()  # the device writes the next iteration's boundary faces
        for k in vel + ["p"] + faces:
            assert_bitwise(s.get(k), o.field(k), f"{name} {scheme} it{it} {k}")


@pytest.mark.parametrize("scheme", ["quick", "van_leer"])
def test_dc_jacobi_iterations_bitwise(gpu_ok, scheme):
    cfg = dict(CASES["channel20x9"], linear_solver=ifc.JACOBI, convection_scheme=scheme)
    o = O.Oracle(to_oracle_cfg(cfg), "f")
    s = ifc.Solver(cfg)
    load_both(o, s, seeded_state(cfg, 9, np.float32))
    for it in range(3):
        s.iterate(1)
        o.outer_iteration()
        o.bc_face_vel()
        for k in ("u", "v", "p", "uf", "vf"):
            assert_bitwise(s.get(k), o.field(k), f"jacobi {scheme} it{it} {k}")


@pytest.mark.parametrize("scheme", ["quick", "minmod"])
def test_dc_converged_cavity(gpu_ok, scheme):
    cfg = dict(ifc.cavity2d(64, re=400.0), convection_scheme=scheme)
    s = ifc.Solver(cfg)
    st = s.solve()
    assert st["status"] == ifc.OK and st["converged"], st
    o = O.Oracle(to_oracle_cfg(cfg), "f")
    n, nm = o.solve()
    assert nm["converged"]
    assert abs(st["outer_iterations"] - n) <= 2, (st["outer_iterations"], n)
    for k in ("u", "v"):
        assert rel_l2(s.get(k), o.field(k)) < 1e-6, k
    o64 = O.Oracle(to_oracle_cfg(dict(cfg, sweep_mode=O.GS_LEX)), "d")
    o64.solve()
    for k in ("u", "v"):
        assert rel_l2(s.get(k), o64.field(k)) < 1e-4, k
    # the higher-order scheme moves the centreline minimum of u well beyond upwind's
    up = ifc.Solver(ifc.cavity2d(64, re=400.0))
    up.solve()
    umin = lambda x: x.reshape(64, 64)[:, 32].min()
    assert umin(s.get("u")) < umin(up.get("u")) - 0.02


def test_dc_rejected_by_adjoint(gpu_ok):
    cfg = dict(ifc.channel2d(24, 10), convection_scheme="quick")
    s = ifc.Solver(cfg)
    s.iterate(10)
    with pytest.raises(ifc.IfcError) as e:
        s.adjoint()
    assert e.value.status == ifc.UNSUPPORTED


@pytest.mark.parametrize("scheme", ["quick", "van_leer"])
def test_dc_batch_matches_oracle(gpu_ok, scheme):
    """The batched solve applies the correction in its whole-row kernel (every
    case with a higher-order scheme runs there): each case of a mixed batch
    equals its oracle solve, which checks the inner early exit after every
    sweep as that kernel does (tolerance: exact)."""
    cfgs = [dict(ifc.cavity2d(24, ny=20, re=200.0), convection_scheme=scheme),
            dict(ifc.channel2d(40, 12), convection_scheme=scheme),
            ifc.cavity2d(16)]
    res, fields, _ = ifc.batch_solve(cfgs)
    for c, r, f in zip(cfgs, res, fields):
        assert r["converged"], r
        if "convection_scheme" in c:
            assert r["sweeps_per_pass"] == 1  # the whole-row kernel
        o = O.Oracle(to_oracle_cfg(dict(c, check_every=r["sweeps_per_pass"])), "f")
        n, nm = o.solve()
        assert nm["converged"] and n == r["outer_iterations"], (n, r["outer_iterations"])
        for k in ("u", "v"):
            assert_bitwise(f[k], o.field(k), f"batch {scheme} {c['nx']}x{c['ny']} {k}")

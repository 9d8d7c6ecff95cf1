"""Parity of every device step with the CPU oracle, one application each.

The device library is compiled without FMA contraction and with IEEE division,
and the oracle restates the reference's arithmetic in the same order, so the
values must agree bit for bit (tolerance: exact).  Each case starts from seeded
random fields and runs the SIMPLE steps in the order of the reference's
Solver::solve (src/Solver.cu:160-198), comparing after every step.
"""
import numpy as np
import pytest

import ifc
import oracle as O
from cases import small_cases
from helpers import assert_bitwise, load_both, seeded_state, to_oracle_cfg

pytestmark = pytest.mark.gpu
CASES = small_cases()


@pytest.mark.parametrize("prec", ["f", "d"])
@pytest.mark.parametrize("name", list(CASES))
def test_steps_bitwise(gpu_ok, name, prec):
    cfg = dict(CASES[name], precision=prec)
    o = O.Oracle(to_oracle_cfg(cfg), prec)
    s = ifc.Solver(cfg)
    dt = s.dtype
    load_both(o, s, seeded_state(cfg, 7, dt))
    d3 = cfg["dim"] == 3
    vel = ["u", "v"] + (["w"] if d3 else [])
    faces = ["uf", "vf"] + (["wf"] if d3 else [])

    # a2 + a3: first-iteration face init, then face boundary conditions.
    s.stage("face_bc")
    o.init_face_vel()
    o.bc_face_vel()
    for k in faces:
        assert_bitwise(s.get(k), o.field(k), f"{name} face_bc {k}")

    # a4 + a5 + a6: coefficients, sources, boundary fold-in.
    s.stage("mom_assemble")
    o.mom_link_coef()
    o.mom_src()
    o.bc_mom()
    assert_bitwise(s.get("mcoef"), o.field("mcoef"), f"{name} mom coef")
    for k in ["src_u", "src_v"] + (["src_w"] if d3 else []):
        assert_bitwise(s.get(k), o.field(k), f"{name} {k}")

    # a7: momentum sweeps with the inner early-exit rule.
    s.stage("mom_solve")
    for eq in range(cfg["dim"]):
        o.linear_solve(eq)
    for k in vel:
        assert_bitwise(s.get(k), o.field(k), f"{name} mom_solve {k}")
    assert_bitwise(s.get("ac"), o.field("mcoef")[: o.N], f"{name} aC")

    # a9 + a3 + a11: Rhie-Chow faces, face BCs, p' source.
    s.stage("rhie_chow")
    o.rhie_chow()
    o.bc_face_vel()
    o.pcorr_src()
    for k in faces + ["src_p"]:
        assert_bitwise(s.get(k), o.field(k), f"{name} rhie_chow {k}")

    # a10: p' link coefficients.
    s.stage("pcorr_coef")
    o.pcorr_link_coef()
    assert_bitwise(s.get("pcoef"), o.field("pcoef"), f"{name} pcoef")

    # a12: p' = 0 and the p' sweeps (+ FP64 mean removal in closed domains).
    s.stage("pcorr_solve")
    o.field("pc")[:] = 0
    o.linear_solve(O.EQ_P)
    if to_oracle_cfg(cfg)["pin_pressure"]:
        o.pin_pcorr()
    pc_dev = s.get("pc")
    if to_oracle_cfg(cfg)["pin_pressure"]:
        # the mean is an FP64 sum whose order differs between CPU and GPU
        np.testing.assert_allclose(pc_dev, o.field("pc"), rtol=0, atol=4 * np.finfo(dt).eps * np.abs(pc_dev).max())
        o.field("pc")[:] = pc_dev
        s.set("pc", pc_dev)
    else:
        assert_bitwise(pc_dev, o.field("pc"), f"{name} pc")

    # a13: corrections.
    # (the device also writes the next iteration's boundary faces)
    s.stage("update")
    o.update_field()
    o.bc_face_vel()
    for k in ["p"] + vel + faces:
        assert_bitwise(s.get(k), o.field(k), f"{name} update {k}")


@pytest.mark.parametrize("name", list(CASES))
def test_single_sweeps_and_norms(gpu_ok, name):
    """One red-black sweep at a time on materialised coefficients, with the
    FP64 sum of squared changes of each sweep."""
    cfg = CASES[name]
    o = O.Oracle(to_oracle_cfg(cfg), "f")
    s = ifc.Solver(cfg)
    load_both(o, s, seeded_state(cfg, 11, np.float32))
    s.stage("face_bc"); o.init_face_vel(); o.bc_face_vel()
    s.stage("mom_assemble"); o.mom_link_coef(); o.mom_src(); o.bc_mom()
    sq_dev = s.sweep(0, 3)
    sq_ref = [o.sweep(O.EQ_U, O.GS_REDBLACK) for _ in range(3)]
    assert_bitwise(s.get("u"), o.field("u"), f"{name} u after 3 sweeps")
    np.testing.assert_allclose(sq_dev, sq_ref, rtol=1e-12)


@pytest.mark.parametrize("prec", ["f", "d"])
@pytest.mark.parametrize("name", list(CASES))
def test_outer_iterations(gpu_ok, name, prec):
    """Whole outer iterations through the CUDA graph (ifc_iterate)."""
    cfg = dict(CASES[name], precision=prec)
    oc = to_oracle_cfg(cfg)
    o = O.Oracle(oc, prec)
    s = ifc.Solver(cfg)
    load_both(o, s, seeded_state(cfg, 3, s.dtype))
    for it in range(3):
        st = s.iterate(1)
        nm = o.outer_iteration()
        o.bc_face_vel()  # the device writes the next iteration's boundary faces
        assert st["outer_iterations"] == it + 1
        keys = ["u", "v", "p"] + (["w"] if cfg["dim"] == 3 else [])
        if oc["pin_pressure"]:
            for k in keys:
                np.testing.assert_allclose(s.get(k), o.field(k), rtol=1e-5, atol=1e-6 * (1 + np.abs(o.field(k)).max()))
                o.field(k)[:] = s.get(k)
            for k in ("uf", "vf", "wf", "pc"):
                o.field(k)[:] = s.get(k)
        else:
            for k in keys + ["uf", "vf"]:
                assert_bitwise(s.get(k), o.field(k), f"{name} it{it} {k}")
        for a, b in (("norm_u", "u"), ("norm_v", "v"), ("norm_p", "p"), ("norm_mass", "mass")):
            np.testing.assert_allclose(st[a], nm[b], rtol=1e-6, atol=1e-300)


def _coop_cases():
    c = dict(CASES)
    c["channel96x40"] = dict(ifc.channel2d(96, 40), nIter_u=3, nIter_v=3, nIter_p=7)
    c["cavity12x10x14"] = dict(ifc.cavity3d(12, nx=12, ny=10, nz=14), nIter_u=3, nIter_v=3, nIter_w=3, nIter_p=7)
    return c


COOP = _coop_cases()


@pytest.mark.parametrize("prec", ["f", "d"])
@pytest.mark.parametrize("name", list(COOP))
def test_sweeps_without_norms_bitwise(gpu_ok, name, prec):
    """ifc_sweep without per-sweep norms runs the n sweeps as one cooperative
    launch on the stored planes (k_coef_solve2d in 2D, k_csolve3d in 3D):
    the fields must equal the oracle's n red-black sweeps bit for bit, for
    every momentum component and p', from a seeded state."""
    cfg = dict(COOP[name], precision=prec)
    o = O.Oracle(to_oracle_cfg(cfg), prec)
    s = ifc.Solver(cfg)
    load_both(o, s, seeded_state(cfg, 13, s.dtype))
    d3 = cfg["dim"] == 3
    s.stage("face_bc"); o.init_face_vel(); o.bc_face_vel()
    s.stage("mom_assemble"); o.mom_link_coef(); o.mom_src(); o.bc_mom()
    for eq, k in enumerate(["u", "v"] + (["w"] if d3 else [])):
        assert s.sweep(eq, 4, norms=False) is None
        for _ in range(4):
            o.sweep(eq, O.GS_REDBLACK)
        assert_bitwise(s.get(k), o.field(k), f"{name} {k} after 4 sweeps")
    s.stage("rhie_chow"); o.rhie_chow(); o.bc_face_vel(); o.pcorr_src()
    s.stage("pcorr_coef"); o.pcorr_link_coef()
    s.sweep(O.EQ_P, 6, norms=False)
    for _ in range(6):
        o.sweep(O.EQ_P, O.GS_REDBLACK)
    assert_bitwise(s.get("pc"), o.field("pc"), f"{name} pc after 6 sweeps")


@pytest.mark.parametrize("name", ["channel20x9", "channel7x5x6"])
def test_async_stages_equal_sync_stages(gpu_ok, name):
    """ifc_run_stage_async enqueues the same launches as ifc_run_stage; after
    ifc_sync the fields are the same bits, for two whole outer iterations."""
    cfg = dict(CASES[name], tol_u=0.0, tol_v=0.0, tol_w=0.0, tol_p=0.0, tol_mass=0.0, pin_pressure=0)
    a, b = ifc.Solver(cfg), ifc.Solver(cfg)
    state = seeded_state(cfg, 21, a.dtype)
    for s in (a, b):
        for k, v in state.items():
            s.set(k, v)
    steps = ["face_bc"] + ["mom_solve", "rhie_chow", "pcorr_solve", "update"] * 2
    for st in steps:
        a.stage(st)
        b.stage(st, wait=False)
    b.sync()
    names = ["u", "v", "p", "uf", "vf"] + (["w", "wf"] if cfg["dim"] == 3 else [])
    for k in names:
        assert_bitwise(b.get(k), a.get(k), f"{name} async {k}")

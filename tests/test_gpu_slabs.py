"""Slab decomposition on the device: one grid cut into 2-4 overlapping slabs,
each an ifc.Solver handle on the same GPU with halo rows refreshed by device
copies after every step (ifc_slabs.LocalHalo), against the undecomposed
solve on the whole grid after the same outer iterations.  Tolerance: exact
(bit for bit) on u, v, w, p and the face velocities; the whole grid's mass
imbalance formed from the owned rows agrees with the undecomposed handle's
to FP64 summation order (1e-9 relative).

Both granularities run: whole stages between exchanges (the fused 2D sweeps,
the cooperative 3D p' solve) and chunks of k sweeps on materialised
coefficients."""
import numpy as np
import pytest

import ifc
import ifc_slabs as S
import oracle as O
from helpers import assert_bitwise, to_oracle_cfg

pytestmark = pytest.mark.gpu


def _undecomposed(cfg, iterations):
    c = dict(cfg, tol_u=0.0, tol_v=0.0, tol_w=0.0, tol_p=0.0, tol_mass=0.0, pin_pressure=0)
    s = ifc.Solver(c)
    st = s.iterate(iterations)
    assert st["outer_iterations"] == iterations, st
    return s, st


def _names(dim):
    return ["u", "v", "p", "uf", "vf"] + (["w", "wf"] if dim == 3 else [])


CASES = {
    # 10/10/20 sweeps: halo 44 rows, two slabs of 48 owned rows
    "channel128x96_stages_2": (lambda: ifc.channel2d(128, 96), 2, None, 12),
    "channel128x64_chunk2_4": (lambda: ifc.channel2d(128, 64), 4, 2, 12),
    "cavity64x80_chunk5_3": (lambda: ifc.cavity2d(64, ny=80), 3, 5, 8),
    # 5/5/5/50 sweeps: chunks of 4 (halo 12), or whole stages (halo 104)
    "cavity16x16x48_chunk4_3": (lambda: ifc.cavity3d(16, nx=16, ny=16, nz=48), 3, 4, 5),
    "cavity12x12x240_stages_2": (lambda: ifc.cavity3d(12, nx=12, ny=12, nz=240), 2, None, 3),
    # Jacobi sweeps, whole stages between exchanges
    "channel128x96_jacobi_stages_2": (lambda: ifc.channel2d(128, 96, linear_solver=ifc.JACOBI), 2, None, 8),
    # higher-order convection, an inlet on a cut face and a west inlet profile
    "mixed_quick96x72_chunk2_3": (lambda: _mixed_quick(), 3, 2, 6),
}


def _mixed_quick():
    c = ifc.channel2d(96, 72, nIter_u=4, nIter_v=4, nIter_p=8, convection_scheme="quick")
    c["velBC_type"] = [ifc.OUTLET, ifc.INLET, ifc.INLET, ifc.WALL, ifc.WALL, ifc.WALL]
    c["velBC_val"] = [[0, 0, 0], [0.002, 0.0005, 0], [0.0003, -0.001, 0], [0, 0, 0], [0, 0, 0], [0, 0, 0]]
    c["inlet_profile"] = np.linspace(0.0005, 0.0015, 72)
    return c


@pytest.mark.parametrize("prec", ["f", "d"])
@pytest.mark.parametrize("name", list(CASES))
def test_slabs_match_undecomposed_bitwise(gpu_ok, name, prec):
    make, parts, k, its = CASES[name]
    cfg = dict(make(), precision=prec)
    whole, st_whole = _undecomposed(cfg, its)
    ref = {n: whole.get(n) for n in _names(cfg["dim"])}
    whole.close()
    with S.SlabSolver(cfg, parts=parts, sweeps_per_exchange=k) as ss:
        assert ss.plan.parts == parts
        st = ss.iterate(its)
        for n in ref:
            assert_bitwise(ss.gather(n), ref[n], f"{name} {prec} {n}")
    assert st["outer_iterations"] == its and st["exchanges"] > 0
    np.testing.assert_allclose(st["norm_mass"], st_whole["norm_mass"], rtol=1e-9, atol=0)


def test_slabs_match_oracle_3d(gpu_ok):
    """The same decomposition against the CPU oracle on the whole grid."""
    cfg = ifc.cavity3d(8, nx=8, ny=6, nz=30, nIter_u=2, nIter_v=2, nIter_w=2, nIter_p=6)
    with S.SlabSolver(cfg, parts=3, sweeps_per_exchange=2) as ss:
        ss.iterate(4)
        got = {n: ss.gather(n) for n in _names(3)}
    c = dict(cfg, tol_u=0.0, tol_v=0.0, tol_w=0.0, tol_p=0.0, tol_mass=0.0, pin_pressure=0)
    o = O.Oracle(to_oracle_cfg(c), "f")
    for _ in range(4):
        o.outer_iteration()
    o.bc_face_vel()
    for n in got:
        assert_bitwise(got[n], o.field(n), f"3d slabs vs oracle {n}")


def test_3d_handles_of_different_sizes_coexist(gpu_ok):
    """The cooperative 3D p' kernel's shared-memory limit is one setting
    shared by every handle: a smaller handle created later must not break
    the larger one's launches (as the slabs of one grid are)."""
    a = ifc.Solver(ifc.cavity3d(16, nx=16, ny=16, nz=40))
    b = ifc.Solver(ifc.cavity3d(8))
    for s in (a, b, a):
        st = s.iterate(2)
        assert st["status"] == ifc.OK, st
    a.close()
    b.close()


@pytest.mark.parametrize("name", ["channel128x96_stages_2", "cavity16x16x48_chunk4_3"])
def test_slab_vtk_equals_the_whole_handle_file(gpu_ok, tmp_path, name):
    """The VTK file written from the slabs' gathered fields is byte for byte
    the file the undecomposed handle writes after the same iterations."""
    make, parts, k, its = CASES[name]
    cfg = make()
    whole, _ = _undecomposed(cfg, its)
    a = tmp_path / "whole.vtk"
    whole.write_vtk(str(a))
    whole.close()
    with S.SlabSolver(cfg, parts=parts, sweeps_per_exchange=k) as ss:
        ss.iterate(its)
        b = tmp_path / "slabs.vtk"
        ss.write_vtk(str(b))
    assert a.read_bytes() == b.read_bytes()

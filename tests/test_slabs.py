"""Slab decomposition (ifc_slabs) on the CPU: the plan, the halo rule, and
whole decomposed solves with oracle slabs against the undecomposed oracle, bit
for bit, in one process (LocalHalo) and over two gloo ranks (DistHalo, the
exchange the NCCL form runs).

The oracle slabs run the oracle functions that each device step matches bit
for bit, so these tests check the orchestration, the halo rule and the
exchange on the CPU; tests/test_gpu_slabs.py runs the same decomposition on
device slabs."""
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import ifc
import ifc_slabs as S
from slab_oracle import OracleSlab, assert_equal_fields, state_names, undecomposed


def _oracle_factory(prec):
    return lambda c: OracleSlab(c, prec)


def _compare(ss, cfg, iterations, prec, what):
    ref = undecomposed(cfg, iterations, prec)
    names = state_names(cfg["dim"])
    assert_equal_fields({n: ss.gather(n) for n in names}, {n: ref.field(n) for n in names}, what)
    return ref


@pytest.mark.parametrize("cells,parts,halo", [(40, 2, 14), (96, 4, 8), (97, 3, 6), (60, 5, 12), (64, 1, 0)])
def test_plan_properties(cells, parts, halo):
    p = S.plan_slabs(cells, parts, halo)
    assert p.parts == parts
    assert p.own[0][0] == 0 and p.own[-1][1] == cells
    for s in range(parts):
        o0, o1 = p.own[s]
        g0, g1 = p.span[s]
        assert o1 - o0 >= halo and o0 % 2 == 0 and g0 % 2 == 0  # global red-black colours
        assert g0 == max(0, o0 - halo) and g1 == min(cells, o1 + halo)
        if s:
            assert p.own[s - 1][1] == o0
    sizes = [o1 - o0 for o0, o1 in p.own]
    assert max(sizes) - min(sizes) <= 3


def test_plan_rejects_thin_slabs():
    with pytest.raises(ValueError, match="thinner than the halo"):
        S.plan_slabs(40, 4, 14)
    with pytest.raises(ValueError):
        S.plan_slabs(40, 2, 5)  # odd halo would flip the colours of the upper slab


def test_halo_depth():
    c = ifc.channel2d(64, 64)  # 10/10/20 sweeps
    assert S.halo_depth(c) == 44
    assert S.halo_depth(c, 4) == 12
    assert S.halo_depth(c, 100) == 44
    c3 = ifc.cavity3d(8)  # 5/5/5/50
    assert S.halo_depth(c3) == 104 and S.halo_depth(c3, 1) == 6


def test_field_rows_layout():
    # 2D: rows along y; uf has nx+1 faces per row, vf ny+1 face rows
    assert S.field_rows("u", 2, 10, 7, 1) == (10, 7, 1)
    assert S.field_rows("uf", 2, 10, 7, 1) == (11, 7, 1)
    assert S.field_rows("vf", 2, 10, 7, 1) == (10, 8, 1)
    assert S.field_rows("mcoef", 2, 10, 7, 1) == (10, 7, 5)
    # 3D: planes along z
    assert S.field_rows("p", 3, 10, 7, 5) == (70, 5, 1)
    assert S.field_rows("uf", 3, 10, 7, 5) == (77, 5, 1)
    assert S.field_rows("vf", 3, 10, 7, 5) == (80, 5, 1)
    assert S.field_rows("wf", 3, 10, 7, 5) == (70, 6, 1)
    assert S.field_rows("pcoef", 3, 10, 7, 5) == (70, 5, 7)


def test_slab_config():
    cfg = ifc.channel2d(32, 40, inlet_profile=np.arange(40.0))
    p = S.plan_slabs(40, 2, 8)
    c = S.slab_config(cfg, p, 1)
    assert c["ny"] == p.span[1][1] - p.span[1][0] and c["slab_axis_cells"] == 40
    assert c["ymin"] == cfg["ymin"] and c["ymax"] == cfg["ymax"]
    assert c["tol_p"] == 0 and c["pin_pressure"] == 0
    np.testing.assert_array_equal(c["inlet_profile"], np.arange(p.span[1][0], p.span[1][1], dtype=float))


def _mixed_quick():
    c = ifc.channel2d(20, 44, nIter_u=2, nIter_v=2, nIter_p=3, convection_scheme="quick")
    c["velBC_type"] = [ifc.OUTLET, ifc.INLET, ifc.INLET, ifc.WALL, ifc.WALL, ifc.WALL]
    c["velBC_val"] = [[0, 0, 0], [0.002, 0.0005, 0], [0.0003, -0.001, 0], [0, 0, 0], [0, 0, 0], [0, 0, 0]]
    c["inlet_profile"] = np.linspace(0.0005, 0.0015, 44)
    return c


CASES = {
    "channel24x40_stages_2": (lambda: ifc.channel2d(24, 40, nIter_u=3, nIter_v=3, nIter_p=5), 2, None, 4),
    "channel24x40_chunk1_3": (lambda: ifc.channel2d(24, 40, nIter_u=3, nIter_v=3, nIter_p=5), 3, 1, 4),
    "channel24x40_chunk2_2": (lambda: ifc.channel2d(24, 40, nIter_u=3, nIter_v=3, nIter_p=5), 2, 2, 4),
    "cavity17x48_chunk2_3": (lambda: ifc.cavity2d(17, ny=48, nIter_u=3, nIter_v=3, nIter_p=6), 3, 2, 4),
    "mixed_quick_chunk1_3": (_mixed_quick, 3, 1, 5),
    "cavity6x5x30_chunk1_3": (lambda: ifc.cavity3d(6, nx=6, ny=5, nz=30, nIter_u=2, nIter_v=2, nIter_w=2,
                                                   nIter_p=4), 3, 1, 3),
    "cavity6x5x30_stages_2": (lambda: ifc.cavity3d(6, nx=6, ny=5, nz=30, nIter_u=2, nIter_v=2, nIter_w=2,
                                                   nIter_p=4), 2, None, 3),
    "channel24x60_jacobi_chunk2_3": (lambda: ifc.channel2d(24, 60, nIter_u=3, nIter_v=3, nIter_p=5,
                                                           linear_solver=ifc.JACOBI), 3, 2, 4),
    "channel24x60_jacobi_stages_2": (lambda: ifc.channel2d(24, 60, nIter_u=3, nIter_v=3, nIter_p=5,
                                                           linear_solver=ifc.JACOBI), 2, None, 4),
}


@pytest.mark.parametrize("prec", ["f", "d"])
@pytest.mark.parametrize("name", list(CASES))
def test_oracle_slabs_bitwise(name, prec):
    make, parts, k, its = CASES[name]
    cfg = make()
    ss = S.SlabSolver(cfg, parts=parts, sweeps_per_exchange=k, make_slab=_oracle_factory(prec))
    st = ss.iterate(its)
    assert st["outer_iterations"] == its and st["exchanges"] > 0 and st["halo_bytes"] > 0
    ref = _compare(ss, cfg, its, prec, name)
    # the whole grid's mass imbalance from the owned rows of every slab
    mass = np.sqrt(np.sum(ref.field("src_p").astype(np.float64) ** 2) / ref.field("src_p").size)
    assert abs(st["norm_mass"] - mass) <= 1e-12 * mass


def test_thin_halo_breaks_parity(monkeypatch):
    """A halo below the reach of a step's sweeps shows in the owned rows: the
    exact comparison above would catch a halo rule that is too shallow."""
    cfg = ifc.channel2d(24, 40, nIter_u=3, nIter_v=3, nIter_p=5)
    monkeypatch.setattr(S, "halo_depth", lambda c, k=None: 6)
    ss = S.SlabSolver(cfg, parts=2, make_slab=_oracle_factory("f"))
    ss.iterate(4)
    with pytest.raises(AssertionError, match="differ"):
        _compare(ss, cfg, 4, "f", "thin halo")


def test_load_and_gather_round_trip():
    cfg = ifc.channel2d(16, 40, nIter_u=1, nIter_v=1, nIter_p=1)
    ss = S.SlabSolver(cfg, parts=3, sweeps_per_exchange=1, make_slab=_oracle_factory("d"))
    rng = np.random.default_rng(5)
    for name, n in (("u", 16 * 40), ("uf", 17 * 40), ("vf", 16 * 41)):
        a = rng.uniform(-1, 1, n)
        ss.load(name, a)
        np.testing.assert_array_equal(ss.gather(name), a)


def _gloo_worker(rank, world, port, q, name, prec):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        make, _, k, its = CASES[name]
        cfg = make()
        ss = S.SlabSolver(cfg, sweeps_per_exchange=k, group=dist.group.WORLD, make_slab=_oracle_factory(prec))
        st = ss.iterate(its)
        got = {n: ss.gather(n) for n in state_names(cfg["dim"])}
        if rank == 0:
            q.put((st, got, ss.plan))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,world", [("channel24x40_stages_2", 2), ("cavity6x5x30_chunk1_3", 2),
                                        ("cavity6x5x30_chunk1_3", 3)])
def test_gloo_ranks_bitwise(name, world):
    """One slab per gloo rank; with three ranks the middle one swaps halos
    with both neighbours in one grouped exchange."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + (os.getpid() + len(name) + 7 * world) % 1000
    procs = [ctx.Process(target=_gloo_worker, args=(r, world, port, q, name, "f")) for r in range(world)]
    for p in procs:
        p.start()
    st, got, plan = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert plan.parts == world and st["exchanges"] > 0
    make, _, _, its = CASES[name]
    cfg = make()
    ref = undecomposed(cfg, its, "f")
    assert_equal_fields(got, {n: ref.field(n) for n in state_names(cfg["dim"])}, f"gloo {name}")


def test_solve_stops_on_the_whole_grid_mass_imbalance():
    """solve() runs blocks of outer iterations until the mass imbalance over
    the whole grid (formed from the slabs' owned rows) falls below tol_mass
    times its largest value at the checks; the fields are still bit for bit
    those of the undecomposed oracle after the same number of iterations."""
    cfg = ifc.cavity2d(16, ny=48, nIter_u=3, nIter_v=3, nIter_p=8)
    ss = S.SlabSolver(cfg, parts=2, make_slab=_oracle_factory("d"))
    st = ss.solve(tol_mass=0.15, max_outer=400, check_every=25)
    assert st["converged"] and st["rel_mass"] < 0.15, st
    assert st["outer_iterations"] % 25 == 0 and st["outer_iterations"] < 400
    _compare(ss, cfg, st["outer_iterations"], "d", "solve")
    st2 = ss.solve(tol_mass=0.0, max_outer=st["outer_iterations"] + 5, check_every=25)
    assert st2["outer_iterations"] == st["outer_iterations"] + 5 and not st2["converged"]


@pytest.mark.parametrize("binary", [False, True])
def test_write_vtk_equals_the_whole_grid_file(tmp_path, binary):
    """The VTK file from the slabs' gathered fields is byte for byte the one
    the writer makes from the undecomposed oracle's fields."""
    make, parts, k, its = CASES["cavity6x5x30_chunk1_3"]
    cfg = make()
    ss = S.SlabSolver(cfg, parts=parts, sweeps_per_exchange=k, make_slab=_oracle_factory("f"))
    ss.iterate(its)
    a = tmp_path / "slabs.vtk"
    ss.write_vtk(str(a), binary=binary)
    ref = undecomposed(cfg, its, "f")
    b = tmp_path / "whole.vtk"
    T = np.full(ref.field("u").size, 273.0, dtype=np.float32)
    ifc.write_vtk_host(cfg, ref.field("u"), ref.field("v"), ref.field("w"), ref.field("p"), T, str(b), binary)
    assert a.read_bytes() == b.read_bytes()

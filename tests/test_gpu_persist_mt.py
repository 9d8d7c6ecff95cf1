"""The single-launch 2D solve with several tiles per CTA (grids with more
tiles than co-resident CTAs, such as the reference's own 1024 x 256 case).
IFC_PERSIST_MAX_CTAS caps the CTAs so that small grids take the multi-tile
form.  Whole outer iterations must match the oracle bit for bit (tolerance:
exact), like the one-tile form; a converged solve must agree with the
one-tile solve (relative L2 1e-6, outer iterations within 2: the per-sweep
FP64 sums are grouped by CTA, so only their rounding can differ)."""
import numpy as np
import pytest

import ifc
import oracle as O
from helpers import assert_bitwise, load_both, rel_l2, seeded_state, to_oracle_cfg

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["channel100x40_f", "channel100x40_d", "channel100x40_quick", "channel70x50_f"])
def test_multi_tile_iterations_bitwise(gpu_ok, monkeypatch, case):
    monkeypatch.setenv("IFC_PERSIST_MAX_CTAS", "5")
    nx, ny = (70, 50) if "70x50" in case else (100, 40)
    cfg = dict(ifc.channel2d(nx, ny), precision="d" if case.endswith("_d") else "f")
    if case.endswith("quick"):
        cfg["convection_scheme"] = "quick"
    o = O.Oracle(to_oracle_cfg(cfg), "d" if cfg["precision"] == "d" else "f")
    s = ifc.Solver(cfg)
    load_both(o, s, seeded_state(cfg, 4, s.dtype))
    for it in range(3):
        st = s.iterate(1)
        assert st["kernel_launches"] == 3, st  # face BCs, begin, the one cooperative launch
        o.outer_iteration()
        o.bc_face_vel()
        for k in ("u", "v", "p", "uf", "vf"):
            assert_bitwise(s.get(k), o.field(k), f"{case} it{it} {k}")


def test_multi_tile_converged_cavity_matches_one_tile(gpu_ok, monkeypatch):
    cfg = ifc.cavity2d(64)
    one = ifc.Solver(cfg)
    st1 = one.solve()
    monkeypatch.setenv("IFC_PERSIST_MAX_CTAS", "3")
    mt = ifc.Solver(cfg)
    st2 = mt.solve()
    assert st1["converged"] and st2["converged"]
    assert abs(st1["outer_iterations"] - st2["outer_iterations"]) <= 2
    for k in ("u", "v"):
        assert rel_l2(mt.get(k), one.get(k)) < 1e-6, k

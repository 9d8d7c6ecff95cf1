"""The C ABI library loads and exports every symbol include/*.h declares; the
default config equals the reference's include/config.h; bad configs are
rejected without touching a GPU."""
import ctypes as C
import glob
import os
import re

import pytest

import ifc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(ifc_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_exports_every_declared_symbol():
    lib = ifc.load()
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.ifc_abi_version() == 1


def test_default_config_is_reference_config_h():
    c = ifc.IfcConfig()
    assert ifc.load().ifc_config_default(C.byref(c)) == ifc.OK
    # include/config.h:6-81
    assert (c.dim, c.nx, c.ny, c.nz) == (2, 1024, 256, 1)
    assert (c.xmin, c.xmax, c.ymin, c.ymax, c.zmin, c.zmax) == (-2, 2, -0.5, 0.5, 0.0, 1.0)
    assert (c.density, c.dynamic_viscosity) == (50, 1)
    assert list(c.vel_bc_type) == [2, 1, 0, 0, 0, 0]
    assert [list(v) for v in c.vel_bc_val] == [[0, 0, 0], [1, 0, 0]] + [[0, 0, 0]] * 4
    assert list(c.temp_bc_type) == [1, 1, 0, 0, 1, 1]
    assert list(c.temp_bc_val) == [0, 0, 293, 373, 0, 0]
    assert (c.num_outer_iter, c.n_iter_u, c.n_iter_v, c.n_iter_w, c.n_iter_p) == (20000, 10, 10, 10, 20)
    assert (c.relax_u, c.relax_v, c.relax_w, c.relax_p) == (0.75, 0.75, 0.75, 0.25)
    assert (c.tol_u, c.tol_v, c.tol_w, c.tol_p, c.tol_mass) == (1e-5, 1e-5, 1e-5, 1e-3, 1e-9)


@pytest.mark.parametrize("change", [
    dict(dim=4), dict(nx=2), dict(ny=0), dict(dim=3, nz=2), dict(xmax=-3.0),
    dict(velBC_type=[3, 0, 0, 0, 0, 0]), dict(nIter_p=-1), dict(numOuterIter=-5),
    dict(linear_solver=7), dict(criterion=9), dict(sweeps_per_pass=99),
])
def test_bad_configs_rejected(change):
    cfg = ifc.cavity2d(16)
    cfg.update(change)
    s, _ = ifc.make_struct(cfg)
    assert ifc.load().ifc_config_check(C.byref(s)) == ifc.BAD_CONFIG


def test_presets_valid():
    for cfg in (ifc.cavity2d(64), ifc.channel2d(), ifc.cavity3d(128), ifc.default_config()):
        s, _ = ifc.make_struct(cfg)
        assert ifc.load().ifc_config_check(C.byref(s)) == ifc.OK


def test_null_arguments():
    lib = ifc.load()
    assert lib.ifc_create(None, None) == ifc.BAD_ARGUMENT
    assert lib.ifc_destroy(None) == ifc.OK
    assert lib.ifc_solve(None, None) == ifc.BAD_ARGUMENT
    assert lib.ifc_status_string(ifc.DIVERGED) == b"diverged"


def test_bounds_checked_build_exports_the_same_symbols():
    """lib/libifc_bc.so (make lib_bc) is the same C ABI with index checks in
    its kernels; ifc_build_flags tells the two builds apart."""
    path = os.path.join(ROOT, "incompflow-cuda_b200", "lib", "libifc_bc.so")
    if not os.path.exists(path):
        import subprocess

        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "incompflow-cuda_b200"), "lib_bc"], check=True)
    bc = C.CDLL(path)
    missing = [n for n in declared_functions() if not hasattr(bc, n)]
    assert not missing, missing
    assert bc.ifc_build_flags() == 1
    assert ifc.load().ifc_build_flags() == 0

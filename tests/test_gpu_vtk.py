"""The handle-level VTK writers (ifc_write_vtk, ifc_write_vtk_binary): they
copy the handle's fields from the device and write the same files as the
host-array writers, whose layout tests/test_vtk.py checks (tolerance: exact)."""
import numpy as np
import pytest

import ifc
from test_vtk import read_legacy_binary_vtk

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["f", "d"])
def test_handle_vtk_files_match_host_writer(gpu_ok, tmp_path, prec):
    cfg = dict(ifc.channel2d(40, 12), precision=prec)
    s = ifc.Solver(cfg)
    s.iterate(30)
    s.solve_energy(max_sweeps=100, tol=0.0)
    f = {k: s.get(k) for k in ("u", "v", "w", "p", "T")}
    dev_b, host_b = str(tmp_path / "dev.bin.vtk"), str(tmp_path / "host.bin.vtk")
    s.write_vtk(dev_b, binary=True)
    ifc.write_vtk_host(cfg, f["u"], f["v"], f["w"], f["p"], f["T"], host_b, binary=True)
    assert open(dev_b, "rb").read() == open(host_b, "rb").read()
    r = read_legacy_binary_vtk(dev_b)
    assert np.array_equal(r["pressure"], f["p"]) and np.array_equal(r["temperature"], f["T"])
    dev_a, host_a = str(tmp_path / "dev.vtk"), str(tmp_path / "host.vtk")
    s.write_vtk(dev_a)
    ifc.write_vtk_host(cfg, f["u"], f["v"], f["w"], f["p"], f["T"], host_a)
    assert open(dev_a).read() == open(host_a).read()

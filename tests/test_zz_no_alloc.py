"""ifc_rb_sweeps_noalloc: red-black sweeps without any device allocation.

Callers that cannot allocate (a program that has reserved the whole GPU for
its own memory pool, or a time-critical loop that cannot afford cudaFree)
give the entry point buffers they already own; its scratch comes from a fixed
array inside the library.  These tests call it through the C ABI and check
that two calls in a row give exactly what the handle-based entry point
(ifc_sweep) gives on the same coefficients, sources and field -- the same
kernel, so the fields must agree bit for bit and the per-sweep FP64 norms to
1e-12 (their block partition may differ).  The file is collected last so that
a failure here does not hide the other tests' results.
"""
import ctypes as C

import numpy as np
import pytest

import ifc
from helpers import seeded_state

pytestmark = pytest.mark.gpu

CASES = [("cavity20x13", ifc.cavity2d(20, ny=13), "f"),
         ("channel24x9_fp64", ifc.channel2d(24, 9), "d"),
         ("cavity5x6x7", ifc.cavity3d(5, nx=5, ny=6, nz=7), "f")]


def noalloc():
    fn = ifc.load().ifc_rb_sweeps_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_int] * 5 + [C.c_void_p] * 3 + [C.c_double, C.c_int, C.POINTER(C.c_double), C.c_void_p]
    return fn


@pytest.mark.parametrize("name,cfg,prec", CASES)
def test_noalloc_matches_handle_sweeps(gpu_ok, name, cfg, prec):
    import torch

    cfg = dict(cfg, precision=prec)
    s = ifc.Solver(cfg)
    for k, v in seeded_state(cfg, 21, s.dtype).items():
        s.set(k, v)
    s.stage("face_bc")
    s.stage("mom_assemble")
    coef, src, u0 = s.get("mcoef"), s.get("src_u"), s.get("u")
    dims = (cfg["dim"], s.nx, s.ny, s.nz, 1 if prec == "d" else 0)
    tdt = torch.float64 if prec == "d" else torch.float32
    d_coef = torch.from_numpy(coef).to("cuda", tdt)
    d_src = torch.from_numpy(src).to("cuda", tdt)
    d_phi = torch.from_numpy(u0).to("cuda", tdt)
    torch.cuda.synchronize()
    fn = noalloc()
    for call, n in enumerate((3, 2)):
        ref_sq = s.sweep(0, n)          # the handle-based entry point
        ref_u = s.get("u")
        sq = (C.c_double * n)()
        rc = fn(*dims, d_coef.data_ptr(), d_src.data_ptr(), d_phi.data_ptr(), cfg["relax_u"], n, sq, None)
        assert rc == ifc.OK, (call, rc)
        got = d_phi.cpu().numpy()
        assert np.array_equal(got, ref_u), (name, call, float(np.abs(got - ref_u).max()))
        np.testing.assert_allclose(np.array(sq[:n]), ref_sq, rtol=1e-12)
    s.close()


def test_noalloc_rejects_oversize_grid(gpu_ok, capfd):
    rc = noalloc()(3, 1024, 1024, 1024, 0, None, None, None, 0.7, 1, None, None)
    assert rc == ifc.BAD_ARGUMENT
    assert "exceed the maximum" in capfd.readouterr().err


def test_noalloc_grid_stride_path_on_caller_stream(gpu_ok):
    """A 1024 x 600 FP32 grid: 307,200 cells of each colour need more than the
    1024 blocks of 256 threads the entry point launches, so its kernel walks
    the grid in strides.  The call goes on a caller-created stream, twice in
    a row, and must equal the handle's sweeps bit for bit."""
    import torch

    cfg = ifc.cavity2d(1024, ny=600)
    s = ifc.Solver(cfg)
    for k, v in seeded_state(cfg, 5, s.dtype).items():
        s.set(k, v)
    s.stage("face_bc")
    s.stage("mom_assemble")
    d_coef = torch.from_numpy(s.get("mcoef")).cuda()
    d_src = torch.from_numpy(s.get("src_u")).cuda()
    d_phi = torch.from_numpy(s.get("u")).cuda()
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    fn = noalloc()
    for call, n in enumerate((2, 1)):
        ref_sq = s.sweep(0, n)
        ref_u = s.get("u")
        sq = (C.c_double * n)()
        rc = fn(2, s.nx, s.ny, 1, 0, d_coef.data_ptr(), d_src.data_ptr(), d_phi.data_ptr(), cfg["relax_u"], n, sq,
                stream.cuda_stream)
        assert rc == ifc.OK, (call, rc)
        stream.synchronize()
        got = d_phi.cpu().numpy()
        assert np.array_equal(got, ref_u), (call, int((got != ref_u).sum()))
        np.testing.assert_allclose(np.array(sq[:n]), ref_sq, rtol=1e-12)
    s.close()

"""VTK writer on host arrays, checked against the byte layout that the
reference's Solver::writeVTK produces (src/Solver.cu:301-367): std::ostream
default formatting (%g, 6 significant digits), a space after every value,
"float" type labels, no newline after the pressure block."""
import numpy as np
import pytest

import ifc


def expected_vtk(cfg, u, v, w, p, t, dtype):
    nx, ny = cfg["nx"], cfg["ny"]
    nz = cfg["nz"] if cfg["dim"] == 3 else 1
    T = dtype

    def coords(lo, hi, n):
        lo_t, d = T(lo), (T(hi) - T(lo)) / T(n)
        return "".join("%g " % float(lo_t + T(i) * d) for i in range(n + 1))

    n = nx * ny * nz
    s = ["# vtk DataFile Version 3.0\n", "flash 3d grid and solution\n", "ASCII\n",
         "DATASET RECTILINEAR_GRID\n", f"DIMENSIONS {nx + 1} {ny + 1} {nz + 1}\n",
         f"X_COORDINATES {nx + 1} float\n", coords(cfg["xmin"], cfg["xmax"], nx), "\n",
         f"Y_COORDINATES {ny + 1} float\n", coords(cfg["ymin"], cfg["ymax"], ny), "\n",
         f"Z_COORDINATES {nz + 1} float\n", coords(cfg["zmin"], cfg["zmax"], nz), "\n",
         f"CELL_DATA {n}\n", "FIELD FieldData 3\n", f"temperature 1 {n} float\n",
         "".join("%g " % float(x) for x in t), "\n", f"velocity 3 {n} float\n",
         "".join("%g %g %g " % (float(a), float(b), float(c)) for a, b, c in zip(u, v, w)), "\n",
         f"pressure 1 {n} float\n", "".join("%g " % float(x) for x in p)]
    return "".join(s)


@pytest.mark.parametrize("case", ["vtk_mixed20x13", "vtk_box5x4x3"])
def test_vtk_bytes_equal_the_reference_writers(tmp_path, case):
    """Files written by the reference's own Solver::writeVTK (src/Solver.cu:
    301-367) from seeded FP32 fields (tests/golden/ref_<case>.npz, made by
    tests/golden/make_golden.py --vtk-only through oracle/ref_vtk.cpp): the
    library's writer, given the same fields, reproduces every byte."""
    import os

    import build_ref

    cfg = build_ref.vtk_cases()[case]
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", f"ref_{case}.npz"))
    path = str(tmp_path / "out.vtk")
    ifc.write_vtk_host(cfg, g["u"], g["v"], g["w"], g["p"], g["T"], path)
    mine, ref = open(path, "rb").read(), g["vtk"].tobytes()
    assert len(mine) == len(ref)
    assert mine == ref


@pytest.mark.parametrize("prec", ["f", "d"])
@pytest.mark.parametrize("cfg", [ifc.channel2d(12, 5), ifc.cavity3d(4, nx=4, ny=3, nz=5)])
def test_vtk_bytes(tmp_path, cfg, prec):
    cfg = dict(cfg, precision=prec)
    dt = np.float32 if prec == "f" else np.float64
    n = cfg["nx"] * cfg["ny"] * (cfg["nz"] if cfg["dim"] == 3 else 1)
    rng = np.random.default_rng(1)
    u, v, w, p = (rng.standard_normal(n).astype(dt) * 10.0 ** rng.integers(-6, 6, n) for _ in range(4))
    u[0] = -0.0
    t = np.full(n, 273.0, dt)
    path = str(tmp_path / "out.vtk")
    ifc.write_vtk_host(cfg, u, v, w, p, t, path)
    got = open(path).read()
    assert got == expected_vtk(cfg, u, v, w, p, t, dt)


def test_vtk_bad_path():
    cfg = ifc.cavity2d(4)
    z = np.zeros(16, np.float32)
    with pytest.raises(ifc.IfcError):
        ifc.write_vtk_host(cfg, z, z, z, z, z, "/nonexistent-dir/x.vtk")


@pytest.mark.parametrize("prec", ["f", "d"])
def test_value_formatting_matches_printf_g(prec, tmp_path):
    """The writer's own %g formatter against Python's correctly rounded '%g'
    on random bit patterns over the whole exponent range, powers of ten and
    their neighbours, and values at or near rounding ties."""
    rng = np.random.default_rng(3)
    dt = np.float32 if prec == "f" else np.float64
    ut = np.uint32 if prec == "f" else np.uint64
    bits = rng.integers(0, np.iinfo(ut).max, 150_000, dtype=np.uint64).astype(ut)
    vals = [bits.view(dt)]
    special = []
    for k in range(-40, 39):
        for base in (1.0, 9.999995, 9.9999949, 9.9999951, 5.0, 1.000005, 1.234565):
            v = dt(base * 10.0 ** k)
            special += [v, np.nextafter(v, dt(np.inf)), np.nextafter(v, dt(-np.inf))]
    special += [dt(x) for x in (0.0, -0.0, 1234565.0, 999999.5, 99999.95, 1e-4, 1e-5, 9.5e-5, 123456.5, 2.5, 1e6)]
    vals.append(np.array(special, dt))
    vals.append((rng.standard_normal(50_000) * 10.0 ** rng.integers(-8, 9, 50_000)).astype(dt))
    v = np.concatenate(vals)
    v = v[np.isfinite(v)]
    nx = 1000
    ny = -(-v.size // nx)
    u = np.zeros(nx * ny, dt)
    u[: v.size] = v
    z = np.zeros_like(u)
    cfg = ifc.cavity2d(3, nx=nx, ny=ny, precision=prec)
    path = str(tmp_path / "fmt.vtk")
    ifc.write_vtk_host(cfg, u, z, z, z, z, path)
    txt = open(path).read()
    got = txt.split("velocity 3")[1].split("\n", 1)[1].split("\npressure")[0].split(" ")[:-1][0::3]
    ref = ["%g" % float(x) for x in u]
    bad = [i for i in range(u.size) if got[i] != ref[i]]
    assert not bad, [(float(u[i]), got[i], ref[i]) for i in bad[:5]]


def read_legacy_binary_vtk(path):
    """Reads the legacy VTK BINARY layout written by ifc_write_vtk_binary_host:
    text header lines, then for each block a label line "<name> <count...>
    <type>" followed by big-endian values and a newline."""
    data = open(path, "rb").read()
    pos = 0

    def line():
        nonlocal pos
        end = data.index(b"\n", pos)
        s = data[pos:end].decode()
        pos = end + 1
        return s

    def block(count, ty):
        nonlocal pos
        dt = np.dtype(">f4" if ty == "float" else ">f8")
        a = np.frombuffer(data, dtype=dt, count=count, offset=pos).astype(dt.newbyteorder("="))
        pos += count * dt.itemsize
        assert data[pos:pos + 1] == b"\n"
        pos += 1
        return a

    hdr = [line() for _ in range(5)]
    out = {"header": hdr}
    for _ in range(3):
        name, n, ty = line().split()
        out[name] = block(int(n), ty)
    out["cell_data"] = line()
    out["field"] = line()
    for _ in range(3):
        name, comps, n, ty = line().split()
        out[name] = block(int(comps) * int(n), ty)
        out[name + "_type"] = ty
    assert pos == len(data)
    return out


@pytest.mark.parametrize("prec", ["f", "d"])
@pytest.mark.parametrize("cfg", [ifc.channel2d(12, 5), ifc.cavity3d(4, nx=4, ny=3, nz=5)])
def test_vtk_binary_round_trip(tmp_path, cfg, prec):
    """Every value comes back exactly, in the handle's precision; header and
    coordinates match the ASCII file's (coordinates to its 6 digits)."""
    cfg = dict(cfg, precision=prec)
    dt = np.float32 if prec == "f" else np.float64
    nx, ny = cfg["nx"], cfg["ny"]
    nz = cfg["nz"] if cfg["dim"] == 3 else 1
    n = nx * ny * nz
    rng = np.random.default_rng(2)
    u, v, w, p, t = ((rng.standard_normal(n) * 10.0 ** rng.integers(-6, 6, n)).astype(dt) for _ in range(5))
    path = str(tmp_path / "out_bin.vtk")
    ifc.write_vtk_host(cfg, u, v, w, p, t, path, binary=True)
    r = read_legacy_binary_vtk(path)
    assert r["header"] == ["# vtk DataFile Version 3.0", "flash 3d grid and solution", "BINARY",
                           "DATASET RECTILINEAR_GRID", f"DIMENSIONS {nx + 1} {ny + 1} {nz + 1}"]
    assert r["cell_data"] == f"CELL_DATA {n}" and r["field"] == "FIELD FieldData 3"
    assert r["temperature_type"] == ("float" if prec == "f" else "double")
    assert np.array_equal(r["temperature"], t)
    assert np.array_equal(r["pressure"], p)
    assert np.array_equal(r["velocity"], np.stack([u, v, w], axis=1).ravel())
    for name, lo, hi, m in (("X_COORDINATES", "xmin", "xmax", nx), ("Y_COORDINATES", "ymin", "ymax", ny),
                            ("Z_COORDINATES", "zmin", "zmax", nz)):
        lo_t, d = dt(cfg[lo]), (dt(cfg[hi]) - dt(cfg[lo])) / dt(m)
        assert np.array_equal(r[name], np.array([lo_t + dt(i) * d for i in range(m + 1)], dtype=dt)), name
    # the ASCII file of the same fields: the same values to 6 significant digits
    apath = str(tmp_path / "out.vtk")
    ifc.write_vtk_host(cfg, u, v, w, p, t, apath)
    lines = open(apath).read().split("\n")
    ascii_p = np.array(lines[-1].split(), dtype=np.float64)
    np.testing.assert_allclose(ascii_p, p.astype(np.float64), rtol=5e-6, atol=0)

"""The drop-in Solver class (incompflow-cuda_b200/host/Solver.h) and its CLI.

A reference user keeps their main.cpp, types.h and config.h and replaces the
reference's include/Solver.h + src/Solver.cu with this package.  The CPU test
compiles the reference's own main.cpp against the drop-in header (skipped
where the reference sources are not on the machine); the GPU test builds the
CLI for a small lid-driven cavity, runs it and compares its VTK output with
the CPU oracle under the reference's own stopping rule.
"""
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

import ifc
import oracle as O
from helpers import rel_l2, to_oracle_cfg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "incompflow-cuda_b200")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
from build_ref import DEFAULT_REF_ROOT  # noqa: E402

REF_MAIN = os.path.join(DEFAULT_REF_ROOT, "main.cpp")


def write_case(d, cfg, scalar="float"):
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "types.h"), "w") as f:
        f.write(f"#ifndef TYPES_H\n#define TYPES_H\nusing scalar = {scalar};\n#endif\n")
    r = lambda x: repr(float(x))
    vt = ", ".join(str(t) for t in cfg["velBC_type"])
    vv = ", ".join("{" + ", ".join(r(x) for x in row) + "}" for row in cfg["velBC_val"])
    nz = cfg.get("nz", 1) if cfg["dim"] == 3 else 1
    with open(os.path.join(d, "config.h"), "w") as f:
        f.write(f"""#ifndef CONFIG_H
#define CONFIG_H
#include "types.h"
constexpr int dim = {cfg['dim']};
constexpr int nx = {cfg['nx']}, ny = {cfg['ny']}, nz = {nz};
constexpr scalar xmin = {r(cfg['xmin'])}, xmax = {r(cfg['xmax'])}, ymin = {r(cfg['ymin'])}, ymax = {r(cfg['ymax'])};
constexpr scalar zmin = {r(cfg['zmin'])}, zmax = {r(cfg['zmax'])};
constexpr scalar thermalConductivity = 1, specificHeatCapacity = 1;
constexpr scalar density = {r(cfg['density'])}, dynamicViscosity = {r(cfg['dynamicViscosity'])};
constexpr scalar thermalDiffusivity = thermalConductivity / specificHeatCapacity / density;
struct velBCs {{ static constexpr int type[6] = {{{vt}}}; static constexpr scalar val[6][3] = {{{vv}}}; }};
struct TempBCs {{ static constexpr int type[6] = {{1, 1, 0, 0, 1, 1}}; static constexpr scalar val[6] = {{0, 0, 293, 373, 0, 0}}; }};
constexpr int numOuterIter = {cfg['numOuterIter']};
constexpr int nIter_u = {cfg['nIter_u']}, nIter_v = {cfg['nIter_v']}, nIter_w = {cfg['nIter_w']}, nIter_p = {cfg['nIter_p']};
constexpr scalar relax_u = {r(cfg['relax_u'])}, relax_v = {r(cfg['relax_v'])}, relax_w = {r(cfg['relax_w'])}, relax_p = {r(cfg['relax_p'])};
constexpr scalar tol_u = {r(cfg['tol_u'])}, tol_v = {r(cfg['tol_v'])}, tol_w = {r(cfg['tol_w'])}, tol_p = {r(cfg['tol_p'])}, tol_mass = {r(cfg['tol_mass'])};
#endif
""")


def build_cli(case_dir, main_cpp, out):
    lib = os.path.join(PKG, "lib")
    cmd = ["g++", "-std=c++20", "-O2", f"-I{case_dir}", f"-I{PKG}/host", f"-I{ROOT}/include", main_cpp,
           f"-L{lib}", "-lifc", f"-Wl,-rpath,{lib}", "-o", out]
    subprocess.run(cmd, check=True)


@pytest.mark.skipif(not os.path.exists(REF_MAIN), reason="reference sources not on this machine")
def test_reference_main_builds_against_dropin(tmp_path):
    write_case(str(tmp_path / "case"), ifc.cavity2d(16))
    build_cli(str(tmp_path / "case"), REF_MAIN, str(tmp_path / "app"))
    assert os.path.exists(tmp_path / "app")


def test_dropin_builds_double(tmp_path):
    write_case(str(tmp_path / "case"), ifc.channel2d(32, 8), scalar="double")
    build_cli(str(tmp_path / "case"), os.path.join(PKG, "host", "main.cpp"), str(tmp_path / "app"))


def read_vtk(path, n):
    toks = open(path).read().split()
    i = toks.index("temperature")
    t = np.array(toks[i + 4:i + 4 + n], dtype=np.float64)
    i = toks.index("velocity")
    vel = np.array(toks[i + 4:i + 4 + 3 * n], dtype=np.float64).reshape(n, 3)
    i = toks.index("pressure")
    p = np.array(toks[i + 4:i + 4 + n], dtype=np.float64)
    return vel[:, 0], vel[:, 1], vel[:, 2], p, t


@pytest.mark.gpu
def test_cli_cavity_matches_oracle(gpu_ok, tmp_path):
    cfg = ifc.cavity2d(32, tol_u=1e-4, tol_v=1e-4, tol_p=1e-4, tol_mass=1e-9)
    write_case(str(tmp_path / "case"), cfg)
    app = str(tmp_path / "app")
    build_cli(str(tmp_path / "case"), os.path.join(PKG, "host", "main.cpp"), app)
    out = subprocess.run([app], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert out.stdout.startswith("iter: 1\n") and "Elapsed time:" in out.stdout
    u, v, w, p, t = read_vtk(str(tmp_path / "output" / "test1.vtk"), 32 * 32)
    o = O.Oracle(to_oracle_cfg(dict(cfg, criterion=O.CRIT_REFERENCE)), "f")
    n, nm = o.solve()
    assert nm["converged"]
    assert rel_l2(u, o.field("u")) < 1e-5 and rel_l2(v, o.field("v")) < 1e-5
    pr = o.field("p").astype(np.float64)
    assert rel_l2(p - p.mean(), pr - pr.mean()) < 1e-5
    assert np.all(t == 0.0) and np.all(w == 0.0)

#!/usr/bin/env python
"""Compile the reference solver from its own sources, where they lie, once per
case (TEST/BASELINE INFRASTRUCTURE ONLY).

The reference is configured at compile time by include/config.h.  For every
case this script writes a config.h that defines the same names
(include/config.h:6-81) into oracle/_ref/cfg_<case>/ and compiles the
reference's src/Solver.cu together with a small driver of ours
(ref_bench.cpp, ref_kernels.cu) using its public API.  The generated
directory comes first on the include path; the reference's own config.h is
then skipped by its include guard.  Nothing is copied from the reference and
its build system is not used.  Outputs go to oracle/_ref/ only.

Only 2D cases are built: the reference's 3D path launches 2048-thread blocks
(src/Solver.cu:381,882,933) and indexes out of bounds in the top-face
kernels (include/kernels.cuh:294,299,695), so it is not run.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
sys.path.insert(0, os.path.join(HERE, "..", "incompflow-cuda_b200", "python"))

# Where the reference's sources lie on the machine that builds the checker;
# IFC_REFERENCE_ROOT overrides it.
DEFAULT_REF_ROOT = os.environ.get("IFC_REFERENCE_ROOT", "/root/reference")

NVCC = ["nvcc", "-std=c++20", "-O2", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-O2"]


def config_h(c: dict, num_outer: int, tol: float, tol_p: float, tol_mass: float) -> str:
    f = lambda x: repr(float(x))
    vt = ", ".join(str(int(t)) for t in c["velBC_type"])
    vv = ", ".join("{" + ", ".join(f(x) for x in row) + "}" for row in c["velBC_val"])
    return f"""// generated by oracle/build_ref.py -- same names as the reference's include/config.h
#ifndef CONFIG_H
#define CONFIG_H
#include "types.h"
constexpr int dim = {c['dim']};
constexpr int nx = {c['nx']};
constexpr int ny = {c['ny']};
constexpr int nz = {c.get('nz', 1) if c['dim'] == 3 else 1};
constexpr scalar xmin = {f(c['xmin'])};
constexpr scalar xmax = {f(c['xmax'])};
constexpr scalar ymin = {f(c['ymin'])};
constexpr scalar ymax = {f(c['ymax'])};
constexpr scalar zmin = {f(c['zmin'])};
constexpr scalar zmax = {f(c['zmax'])};
constexpr scalar thermalConductivity = 1;
constexpr scalar specificHeatCapacity = 1;
constexpr scalar density = {f(c['density'])};
constexpr scalar dynamicViscosity = {f(c['dynamicViscosity'])};
constexpr scalar thermalDiffusivity = thermalConductivity / specificHeatCapacity / density;
struct velBCs {{
    static constexpr int type[6] = {{{vt}}};
    static constexpr scalar val[6][3] = {{{vv}}};
}};
struct TempBCs {{
    static constexpr int type[6] = {{1, 1, 0, 0, 1, 1}};
    static constexpr scalar val[6] = {{0.0, 0.0, 293.0, 373.0, 0.0, 0.0}};
}};
constexpr int numOuterIter = {num_outer};
constexpr int nIter_u = {c['nIter_u']};
constexpr int nIter_v = {c['nIter_v']};
constexpr int nIter_w = {c['nIter_w']};
constexpr int nIter_p = {c['nIter_p']};
constexpr scalar relax_u = {f(c['relax_u'])};
constexpr scalar relax_v = {f(c['relax_v'])};
constexpr scalar relax_w = {f(c['relax_w'])};
constexpr scalar relax_p = {f(c['relax_p'])};
constexpr scalar tol_u = {f(tol)};
constexpr scalar tol_v = {f(tol)};
constexpr scalar tol_w = {f(tol)};
constexpr scalar tol_p = {f(tol_p)};
constexpr scalar tol_mass = {f(tol_mass)};
#endif
"""


def kernel_cases():
    """Small 2D cases whose kernels the harness ref_kernels.cu runs one by one."""
    import ifc

    mixed = ifc.channel2d(20, 13, density=3.0, dynamicViscosity=0.05, relax_u=0.7, relax_v=0.6, relax_p=0.3)
    mixed["velBC_type"] = [ifc.OUTLET, ifc.INLET, ifc.INLET, ifc.WALL, ifc.WALL, ifc.WALL]
    mixed["velBC_val"] = [[0, 0, 0], [0.3, 0.05, 0], [0.2, -0.1, 0], [0, 0, 0], [0, 0, 0], [0, 0, 0]]
    cav = ifc.cavity2d(17, ny=19, relax_u=0.7, relax_v=0.7, relax_p=0.3)
    return {"mixed20x13": mixed, "cavity17x19": cav}


def cases():
    import ifc

    return {
        # throughput: fixed 100 outer iterations per solve() call (tolerances 0)
        "channel512x128": (ifc.channel2d(512, 128), 100, 0.0, 0.0, 0.0),
        # converged runs for the golden fields: fixed iteration counts well past
        # convergence (the reference's own stopping rule is defective, D6/D7)
        "cavity64": (ifc.cavity2d(64), 3000, 0.0, 0.0, 0.0),
        "channel128x32": (ifc.channel2d(128, 32), 3000, 0.0, 0.0, 0.0),
        # the bench case itself, 10000 outer iterations from rest in one
        # solve() call (the oracle converges it in about 6300)
        "channel512x128_long": (ifc.channel2d(512, 128), 10000, 0.0, 0.0, 0.0),
        # time to convergence by the reference's own stopping rule (configs[0]:
        # the 64^2 cavity at tolerance 1e-5, no mass-norm stop)
        "cavity64_converge": (ifc.cavity2d(64), 20000, 1e-5, 1e-5, 0.0),
    }


def vtk_cases():
    """Cases whose seeded fields the harness ref_vtk.cpp writes with the
    reference's Solver::writeVTK: a 2D grid with non-unit extents and a small
    3D box (the writer is host code; the Solver's constructor only allocates)."""
    import ifc

    mixed = kernel_cases()["mixed20x13"]
    box = ifc.cavity3d(5, nx=5, ny=4, nz=3, xmin=-0.3, xmax=0.7, ymin=0.05, ymax=0.125, zmin=-1.5, zmax=2.25)
    return {"vtk_mixed20x13": mixed, "vtk_box5x4x3": box}


def build(ref_root: str, only=None):
    os.makedirs(OUT, exist_ok=True)
    inc = os.path.join(ref_root, "include")
    src = os.path.join(ref_root, "src", "Solver.cu")
    if not os.path.exists(src):
        raise SystemExit(f"reference sources not found under {ref_root}")
    built = []
    for name, (c, n_outer, tol, tol_p, tol_mass) in cases().items():
        if only and name not in only:
            continue
        d = os.path.join(OUT, f"cfg_{name}")
        os.makedirs(d, exist_ok=True)
        with open(os.path.join(d, "config.h"), "w") as fh:
            fh.write(config_h(c, n_outer, tol, tol_p, tol_mass))
        exe = os.path.join(OUT, f"ref_bench_{name}")
        cmd = NVCC + [f"-I{d}", f"-I{inc}", src, os.path.join(HERE, "ref_bench.cpp"), "-o", exe]
        subprocess.run(cmd, check=True)
        built.append(exe)
    for name, c in kernel_cases().items():
        if only and name not in only:
            continue
        d = os.path.join(OUT, f"cfg_{name}")
        os.makedirs(d, exist_ok=True)
        with open(os.path.join(d, "config.h"), "w") as fh:
            fh.write(config_h(c, 1, 0.0, 0.0, 0.0))
        kexe = os.path.join(OUT, f"ref_kernels_{name}")
        subprocess.run(NVCC + [f"-I{d}", f"-I{inc}", os.path.join(HERE, "ref_kernels.cu"), "-o", kexe], check=True)
        built.append(kexe)
    for name, c in vtk_cases().items():
        if only and name not in only:
            continue
        d = os.path.join(OUT, f"cfg_{name}")
        os.makedirs(d, exist_ok=True)
        with open(os.path.join(d, "config.h"), "w") as fh:
            fh.write(config_h(c, 1, 0.0, 0.0, 0.0))
        vexe = os.path.join(OUT, f"ref_{name}")
        subprocess.run(NVCC + [f"-I{d}", f"-I{inc}", src, os.path.join(HERE, "ref_vtk.cpp"), "-o", vexe], check=True)
        built.append(vexe)
    return built


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default=DEFAULT_REF_ROOT)
    ap.add_argument("--only", nargs="*")
    a = ap.parse_args()
    for b in build(a.ref_root, a.only):
        print(b)

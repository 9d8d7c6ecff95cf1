#!/usr/bin/env python
"""Regenerate the golden fixtures from the reference's own build (run on a GPU
machine after `python oracle/build_ref.py` has compiled oracle/_ref/).

  python tests/golden/make_golden.py --out DIR

* ref_kernels_<case>.npz: seeded inputs and the outputs of the reference's
  kernels (include/kernels.cuh) run one by one by oracle/ref_kernels.cu.
* ref_solve_<case>.npz: u, v, p of the reference's Solver::solve() after a
  fixed number of outer iterations well past convergence, read back from its
  VTK output (6 significant digits).
* ref_vtk_<case>.npz (--vtk-only; runs on a machine without a GPU, since the
  writer is host code and the Solver's constructor only allocates): seeded
  float32 fields and the bytes the reference's Solver::writeVTK wrote from
  them (oracle/ref_vtk.cpp).
* oracle_channel512x128.npz (--oracle-only): the 512 x 128 channel solved by
  the FP64 oracle with lexicographic sweeps, the FP64 answer for that case.
* oracle_cavity3d16.npz (--oracle-only needs no GPU): the 16^3 lid-driven
  cavity solved by the FP64 oracle (red-black Gauss-Seidel, per-field rule
  1e-5).  The reference's 3D build cannot run (it launches 2048-thread blocks
  and indexes out of bounds), so this is the 3D pin.
Copy the files into tests/golden/ to update the fixtures.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF = os.path.join(ROOT, "oracle", "_ref")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "incompflow-cuda_b200", "python"))


def kernel_inputs(cfg: dict, seed: int) -> dict:
    rng = np.random.default_rng(seed)
    nx, ny = cfg["nx"], cfg["ny"]
    n = nx * ny
    a_nb = -rng.uniform(0.5, 2.0, (4, n))
    coef = np.concatenate([(-a_nb.sum(0) + rng.uniform(0.1, 1.0, n))[None], a_nb]).ravel()
    f = lambda k: rng.uniform(-1, 1, k)
    return {k: v.astype(np.float32) for k, v in dict(
        u=f(n), v=f(n), p=f(n), pc=f(n), uf=f((nx + 1) * ny), vf=f(nx * (ny + 1)), coef=coef).items()}


def run_kernel_case(name: str, cfg: dict, out: str):
    ins = kernel_inputs(cfg, seed=2024)
    with tempfile.TemporaryDirectory() as tmp:
        din, dout = os.path.join(tmp, "in"), os.path.join(tmp, "out")
        os.makedirs(din)
        os.makedirs(dout)
        for k, v in ins.items():
            v.tofile(os.path.join(din, f"{k}.bin"))
        subprocess.run([os.path.join(REF, f"ref_kernels_{name}"), din, dout], check=True)
        res = {f"out_{f[:-4]}": np.fromfile(os.path.join(dout, f), dtype=np.float32) for f in os.listdir(dout)}
    np.savez_compressed(os.path.join(out, f"ref_kernels_{name}.npz"), **{f"in_{k}": v for k, v in ins.items()}, **res)


def read_vtk(path: str, n: int):
    toks = open(path).read().split()
    i = toks.index("velocity")
    vel = np.array(toks[i + 4:i + 4 + 3 * n], dtype=np.float64).reshape(n, 3)
    i = toks.index("pressure")
    p = np.array(toks[i + 4:i + 4 + n], dtype=np.float64)
    return vel[:, 0], vel[:, 1], p


def run_solve_case(name: str, n_cells: int, out: str):
    with tempfile.TemporaryDirectory() as tmp:
        r = subprocess.run([os.path.join(REF, f"ref_bench_{name}"), "0", "1", f"{name}.vtk"], cwd=tmp,
                           capture_output=True, text=True, check=True)
        u, v, p = read_vtk(os.path.join(tmp, "output", f"{name}.vtk"), n_cells)
    np.savez_compressed(os.path.join(out, f"ref_solve_{name}.npz"), u=u, v=v, p=p, log=np.array(r.stdout[-2000:]))


def vtk_fields(cfg: dict, seed: int) -> dict:
    """Seeded float32 fields spanning many magnitudes (mantissas times 10^-9 ..
    10^9, zeros, small integers, negative values), so the reference's %g-like
    output meets fixed and exponent forms, trailing-zero removal and rounding."""
    rng = np.random.default_rng(seed)
    nz = cfg.get("nz", 1) if cfg["dim"] == 3 else 1
    n = cfg["nx"] * cfg["ny"] * nz
    out = {}
    for k in ("u", "v", "w", "p", "T"):
        x = rng.uniform(-10, 10, n) * 10.0 ** rng.integers(-9, 10, n)
        pick = rng.random(n)
        x[pick < 0.05] = 0.0
        sel = (pick >= 0.05) & (pick < 0.12)
        x[sel] = rng.integers(-1000, 1000, int(sel.sum()))
        out[k] = x.astype(np.float32)
    return out


def run_vtk_case(name: str, cfg: dict, out: str):
    """The reference's Solver::writeVTK on seeded fields (ref_vtk.cpp): the
    file's bytes and the fields they were written from."""
    f = vtk_fields(cfg, seed=7)
    with tempfile.TemporaryDirectory() as tmp:
        din = os.path.join(tmp, "in")
        os.makedirs(din)
        for k, v in f.items():
            v.tofile(os.path.join(din, f"{k}.bin"))
        subprocess.run([os.path.join(REF, f"ref_{name}"), din, f"{name}.vtk"], cwd=tmp, check=True,
                       capture_output=True)
        data = open(os.path.join(tmp, "output", f"{name}.vtk"), "rb").read()
    np.savez_compressed(os.path.join(out, f"ref_{name}.npz"), **f, vtk=np.frombuffer(data, dtype=np.uint8))


def oracle_cavity3d(out: str):
    import ifc
    import oracle as O

    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import to_oracle_cfg

    cfg = ifc.cavity3d(16)
    o = O.Oracle(to_oracle_cfg(cfg), "d")
    n, nm = o.solve()
    f = {k: o.field(k).astype(np.float64).copy() for k in ("u", "v", "w", "p")}
    np.savez_compressed(os.path.join(out, "oracle_cavity3d16.npz"), **f, iterations=np.array(n),
                        converged=np.array(nm["converged"]))


def oracle_channel512x128(out: str):
    """The 512 x 128 channel (the README's default case): 10000 outer
    iterations of the FP64 oracle with lexicographic Gauss-Seidel, well past
    convergence (the per-field rule at 1e-5 stops it at 3620): the FP64
    answer the FP32 device solve of that case is held to (1e-4).  Stored as
    float32 (relative resolution 6e-8)."""
    import ifc
    import oracle as O

    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import to_oracle_cfg

    cfg = dict(ifc.channel2d(512, 128), tol_u=0.0, tol_v=0.0, tol_p=0.0, tol_mass=0.0)
    o = O.Oracle(to_oracle_cfg(dict(cfg, sweep_mode=O.GS_LEX)), "d")
    n, _ = o.solve(10000)
    f = {k: o.field(k).astype(np.float32) for k in ("u", "v", "p")}
    np.savez_compressed(os.path.join(out, "oracle_channel512x128.npz"), **f, iterations=np.array(n))


def main():
    import build_ref

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--oracle-only", action="store_true")
    ap.add_argument("--vtk-only", action="store_true", help="only the writeVTK fixtures (host code; no GPU needed)")
    ap.add_argument("--only", nargs="*", help="only these converged-solve cases of the reference's build")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    if a.only:
        for name in a.only:
            cfg = build_ref.cases()[name][0]
            run_solve_case(name, cfg["nx"] * cfg["ny"], a.out)
        return
    for name, cfg in build_ref.vtk_cases().items():
        run_vtk_case(name, cfg, a.out)
    if a.vtk_only:
        return
    oracle_cavity3d(a.out)
    oracle_channel512x128(a.out)
    if a.oracle_only:
        return
    for name, cfg in build_ref.kernel_cases().items():
        run_kernel_case(name, cfg, a.out)
    for name, (cfg, *_rest) in build_ref.cases().items():
        if name == "channel512x128" or name.endswith("_converge"):
            continue
        run_solve_case(name, cfg["nx"] * cfg["ny"], a.out)
    print("golden fixtures written to", a.out)


if __name__ == "__main__":
    main()

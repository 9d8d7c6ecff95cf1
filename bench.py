#!/usr/bin/env python
"""Throughput benchmark of the B200 SIMPLE solver.

Workload: the reference's default case as its README states it:
a 2D channel of 512 x 128 cells on [-0.0625, 0.0625] x [-0.0125, 0.0125],
water (rho 998.2, mu 1.002e-3), west inlet 0.001 m/s, east outlet, no-slip
north/south walls, SIMPLE with alpha_u 0.75 / alpha_p 0.25 and 10/10/20
red-black Gauss-Seidel sweeps per outer iteration, FP32.  Inputs are
synthetic: the flow starts from rest and is advanced by the warm-up steps.

One step = OUTER_PER_STEP SIMPLE outer iterations (fixed work: the
convergence test runs but does not stop the loop).  The metric is
cell-updates/s, one cell-update being one relaxed point update of one unknown
(u, v or p') at one cell.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun, one rank per GPU) every rank runs an independent
replica: the plain solve does not shard (one grid per GPU), so the scaling is
weak and `value` sums all ranks' cell-updates over the slowest rank's time.

--impl reference times the reference's own implementation of this workload:
its CUDA build (oracle/_ref/, compiled from the reference's sources with the
same case written into its config.h) when present, else the serial CPU
restatement of its kernels.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "incompflow-cuda_b200", "python"))

WORKLOAD = "channel2d_512x128"
OUTER_PER_STEP = 100
BYTES_PER_UPDATE_2D = 32      # stored-coefficient GS update, FP32: 4*(2*dim+4)
METRIC = "cell-updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the compact precision / batch / adjoint / slabs records of the default line")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--form", default="plain",
                    choices=["plain", "adjoint", "precision", "batch", "convergence", "energy", "slabs"],
                    help="plain: the headline throughput line; adjoint: the differentiation form")
    ap.add_argument("--profiles", type=int, default=32, help="adjoint form: seeded inlet profiles")
    ap.add_argument("--fd-profiles", type=int, default=1,
                    help="adjoint form: profiles whose 65 parameters are checked by central differences")
    ap.add_argument("--fd-iters", type=int, default=3000,
                    help="adjoint form: outer iterations of each warm-started FP64 finite-difference solve")
    ap.add_argument("--n3d", type=int, default=128, help="precision form: cells per direction")
    ap.add_argument("--max-outer", type=int, default=8000, help="precision form: outer-iteration cap")
    ap.add_argument("--cases", type=int, default=256, help="batch form: cases")
    ap.add_argument("--convection", default="upwind",
                    choices=["upwind", "central", "sou", "quick", "minmod", "van_leer"],
                    help="plain form: convection scheme (upwind is the reference's; the others run by "
                         "deferred correction)")
    return ap.parse_args()


CONVECTION = "upwind"


def workload_cfg():
    import ifc

    return ifc.channel2d(512, 128, convection_scheme=CONVECTION)


def workload_name():
    return WORKLOAD if CONVECTION == "upwind" else f"{WORKLOAD}_{CONVECTION}"


def workload_config() -> dict:
    """The workload as both arms report it (the same dict in each line)."""
    cfg = workload_cfg()
    return {"workload": workload_name(), "nx": 512, "ny": 128, "outer_iterations_per_step": OUTER_PER_STEP,
            "convection": CONVECTION, "sweeps_u_v_p": [cfg["nIter_u"], cfg["nIter_v"], cfg["nIter_p"]],
            "relax_u_p": [cfg["relax_u"], cfg["relax_p"]], "start": "from rest", "scalar": "fp32"}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def profiled_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` recorded by the committed ncu summary
    (profiles/*.md line "traffic_bytes_per_launch <kernel> <bytes>"), or None."""
    import glob

    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        for line in open(path):
            parts = line.strip().strip("`").split()
            if len(parts) == 3 and parts[0] == "traffic_bytes_per_launch" and parts[1] == kernel:
                try:
                    return float(parts[2])
                except ValueError:
                    pass
    return None


def host_cpu() -> str:
    """CPU model and logical core count of this host (for the baseline label)."""
    model = "unknown CPU"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return f"{model} ({os.cpu_count()} logical cores)"


def cpu_baseline(seconds: float):
    """The serial CPU restatement of the reference's kernels (oracle, FP32,
    1 core) on a bounded sample of the same workload: outer iterations from
    rest until `seconds` of CPU time have passed."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle as O
    from helpers import to_oracle_cfg

    cfg = to_oracle_cfg(workload_cfg())
    o = O.Oracle(cfg, "f")
    t0 = time.perf_counter()
    its, updates = 0, 0
    while time.perf_counter() - t0 < seconds:
        nm = o.outer_iteration()
        its += 1
        updates += o.N * (nm["sweeps"][0] + nm["sweeps"][1] + nm["sweeps"][3])
    dt = time.perf_counter() - t0
    return {"value": updates / dt, "unit": METRIC, "cores": 1, "kind": "port",
            "sample": f"{its} outer iterations of {workload_name()} from rest, serial C oracle (FP32, red-black GS, "
                      f"gcc -O2), {dt:.1f} s on one core of {host_cpu()}"}


def cpu_baseline_all_cores(seconds: float):
    """The same restatement built with OpenMP row loops
    (oracle/_build/libifc_oracle_omp.so) on every host core, timed by
    oracle/time_port.py in a child process (the parallel build's FP64 sweep
    sums add in another order; each cell is computed as in the serial
    build).  A separate record beside the one-core baseline."""
    import subprocess

    threads = os.cpu_count() or 1
    lib = os.path.join(ROOT, "oracle", "_build", "libifc_oracle_omp.so")
    env = dict(os.environ, IFC_ORACLE_LIB=lib, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="true")
    cfg = workload_cfg()
    r = subprocess.run([sys.executable, os.path.join(ROOT, "oracle", "time_port.py"), "--seconds", str(seconds),
                        "--nx", str(cfg["nx"]), "--ny", str(cfg["ny"])],
                       env=env, capture_output=True, text=True, timeout=seconds * 6 + 120)
    if r.returncode != 0:
        return {"error": (r.stderr or r.stdout)[-300:]}
    d = json.loads(r.stdout.strip().splitlines()[-1])
    return {"value": d["cell_updates"] / d["seconds"], "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"{d['outer_iterations']} outer iterations of {workload_name()} from rest, C oracle with "
                      f"OpenMP row loops (FP32, red-black GS, gcc -O2), {d['seconds']:.1f} s on {threads} threads of "
                      f"{host_cpu()}"}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_ours(args):
    import torch
    import torch.distributed as dist

    import ifc

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    stream = torch.cuda.Stream()
    cfg = workload_cfg()
    cfg["stream"] = stream.cuda_stream
    s = ifc.Solver(cfg)
    N = s.N
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        s.iterate(OUTER_PER_STEP)
    # Device-resident throughput: K steps, each timed with CUDA events on the
    # solver's stream; the L2 is flushed between steps (outside the events).
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    updates, launches = 0, 0
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(float(k))
        ev[k][0].record(stream)
        st = s.iterate(OUTER_PER_STEP)
        ev[k][1].record(stream)
        updates += st["cell_updates"]
        launches += st["kernel_launches"]
    barrier()
    clk = clocks.stop()
    ms = sum(a.elapsed_time(b) for a, b in ev)

    # End to end through the public C ABI with host buffers: every step
    # uploads u, v, p from pinned host memory, runs the step, reads them back.
    host_in = {k: torch.from_numpy(s.get(k)).pin_memory() for k in ("u", "v", "p")}
    host_out = {k: torch.empty_like(v).pin_memory() for k, v in host_in.items()}
    lib = ifc.load()
    fid = {k: ifc.FIELDS.index(k) for k in host_in}
    nbytes = N * 4
    e2e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    e2e_updates = 0
    barrier()
    for k in range(args.steps):
        e2e_ev[k][0].record(stream)
        for name, t in host_in.items():
            assert lib.ifc_set_field(s._h, fid[name], C.c_void_p(t.data_ptr()), nbytes) == 0
        st = s.iterate(OUTER_PER_STEP)
        for name, t in host_out.items():
            assert lib.ifc_get_field(s._h, fid[name], C.c_void_p(t.data_ptr()), nbytes) == 0
        e2e_ev[k][1].record(stream)
        e2e_updates += st["cell_updates"]
    barrier()
    e2e_ms = sum(a.elapsed_time(b) for a, b in e2e_ev)

    # Roofline of the dominant kernel.  At this size the whole SIMPLE loop of a
    # step runs as one cooperative launch (k_simple2d); its duration is the
    # step's event time minus two tiny setup kernels.  Algorithmic bytes: the
    # reference-form traffic of one outer iteration, (220 + 32 (n_u+n_v+n_p))
    # bytes per cell in 2D FP32, times the cells and the iterations per launch.
    step_ms = [a.elapsed_time(b) for a, b in ev]
    launch_ms = statistics.mean(step_ms)
    alg_bytes = (220 + BYTES_PER_UPDATE_2D * (cfg["nIter_u"] + cfg["nIter_v"] + cfg["nIter_p"])) * N * OUTER_PER_STEP
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (launch_ms * 1e-3) / 1e9
    traffic = profiled_traffic("k_simple2d")
    t_max = torch.tensor([ms, e2e_ms], dtype=torch.float64, device="cuda")
    tot = torch.tensor([float(updates), float(e2e_updates)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
        dist.all_reduce(tot, op=dist.ReduceOp.SUM)
    ms_all, e2e_all = t_max.tolist()
    upd_all, e2e_upd_all = tot.tolist()

    cpu = None
    cpu_all = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.cpu_seconds)
        cpu_all = cpu_baseline_all_cores(args.cpu_seconds)
    if rank == 0:
        line = {
            "metric": METRIC,
            "value": upd_all / (ms_all * 1e-3),
            "unit": METRIC,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_all / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic: flow from rest, advanced by the warm-up steps",
            "config": workload_config(),
            "impl_notes": {"linear_solver": "red-black Gauss-Seidel", "precision": "fp32 sweeps, fp64 norms",
                           "l2": "flushed (256 MB write) between timed steps",
                           "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e_upd_all / (e2e_all * 1e-3), "unit": METRIC,
                    "h2d_bytes_per_step": 3 * nbytes, "d2h_bytes_per_step": 3 * nbytes},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": "k_simple2d (the whole SIMPLE loop of a step, one cooperative launch)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "traffic": traffic,
                         "algorithmic_bytes_per_launch": alg_bytes, "launch_ms": launch_ms,
                         "note": "reference-form bytes; the 3 MB working set lives in L2, so DRAM traffic is ~0 "
                                 "and the kernel is latency-bound (grid barriers, dependent sweeps)"},
            "ref_equivalent_gbs": upd_all / (ms_all * 1e-3) * BYTES_PER_UPDATE_2D / 1e9,
            "clocks": clk,
        }
        if cpu:
            line["cpu_baseline"] = cpu
        if cpu_all:
            line["cpu_baseline_all_cores"] = cpu_all
        if world == 1 and not args.no_forms and CONVECTION == "upwind":
            forms = {}
            for name, fn in (("precision", lambda: precision_summary(args.n3d)),
                             ("batch", lambda: batch_summary(4)), ("adjoint", lambda: adjoint_summary(4, 8)),
                             ("slabs", slabs_summary)):
                t0 = time.perf_counter()
                try:
                    forms[name] = fn()
                except Exception as e:  # a form's failure must not cost the headline line
                    forms[name] = {"error": f"{type(e).__name__}: {e}"}
                forms[name]["wall_s"] = round(time.perf_counter() - t0, 1)
            line["forms"] = forms
        print(json.dumps(line), flush=True)
    s.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ---- compact records of the further forms in the default line --------------
# Each runs after the headline's timed region, on rank 0 at N = 1, and takes
# seconds; the full forms are bench.py --form precision|batch|adjoint|slabs.

def rel_l2(a, b):
    import numpy as np

    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def prec_byte_model(cfg: dict, N: int) -> dict:
    """Compulsory unique bytes of each 3D stage launch sequence (FP32, whole
    arrays per pass: a half sweep reads whole cache lines of both colours)."""
    nu, npc = cfg["nIter_u"], cfg["nIter_p"]
    return {
        "mom_solve": (nu * 2 * (3 * 4 + 4 + 6 * 4)) * N,          # per half: faces, p, u/v/w read+write
        "rhie_chow": (3 * 4 + 4 + 4 + 3 * 4 + 3 * 4 + 4) * N,     # u v w, p, aC in; faces, b_p out
        "pcorr_solve": (4 + 4 + npc * 2 * (4 + 4 + 4 + 4)) * N,   # 1/aC once; per half 1/aC, p', b_p, p' write
        "update": (4 + 4 + 4 * 3 + 3 * 4 + 4 + 3 * 4 * 2 + 4) * N,
    }


def precision_summary(n: int) -> dict:
    """The 128^3 cavity at Re 400: FP32 time to convergence, ms per outer
    iteration, each stage's compulsory bytes over its device time against the
    measured HBM peak, and the FP32 fields against the FP64 build after the
    same number of outer iterations."""
    import numpy as np

    import ifc

    cfg = ifc.cavity3d(n, re=400.0, numOuterIter=8000, criterion=ifc.CRIT_REFERENCE)
    s32 = ifc.Solver(dict(cfg, precision="f"))
    st = s32.solve()
    k = st["outer_iterations"]
    peak, _ = measured_peaks()
    model = prec_byte_model(cfg, n ** 3)
    stages = {}
    for name in ("mom_solve", "rhie_chow", "pcorr_solve", "update"):
        ms_, nl = s32.time_stage(name, reps=3)
        gbs = model[name] / (ms_ * 1e-3) / 1e9
        stages[name] = {"ms": round(ms_, 4), "launches": nl, "gbs": round(gbs, 1), "frac_of_peak": round(gbs / peak, 3)}
    a = {f: s32.get(f).astype(np.float64) for f in ("u", "v", "w", "p")}
    s32.close()
    s64 = ifc.Solver(dict(cfg, precision="d"))
    st64 = s64.iterate(k)
    b = {f: s64.get(f) for f in ("u", "v", "w", "p")}
    s64.close()
    a["p"] -= a["p"].mean()
    b["p"] = b["p"] - b["p"].mean()
    return {"workload": f"cavity3d_{n}_re400",
            "criterion": "the reference's rule (every norm over the p-norm max), 1e-5",
            "fp32_converged": bool(st["converged"]), "outer_iterations": k,
            "seconds_to_convergence": st["device_ms"] / 1e3, "ms_per_outer_iteration": st["device_ms"] / max(k, 1),
            "fp64_ms_per_outer_iteration": st64["device_ms"] / max(k, 1),
            "rel_l2_vs_fp64_build_equal_iterations": {f: rel_l2(a[f], b[f]) for f in a},
            "stages_at_convergence": stages, "hbm_peak_gbs": peak,
            "gpu_launches": st["kernel_launches"] + st64["kernel_launches"]}


def batch_summary(every: int) -> dict:
    """The seeded 256-case cavity batch in one batched solve, against the plain
    per-case loop timed on every `every`-th case (sum of per-case device times)
    and scaled to all 256 by cell-iterations (cells x outer iterations of each
    case, from the batched solve, which takes the same iterations): the plain
    loop's time per cell-iteration of the sample times the batch's total.  The
    batched fields of the sampled cases are compared with the plain solves'."""
    import ifc

    cases = ifc.batch_cases(256, seed=0)
    ifc.batch_solve([ifc.cavity2d(32), ifc.cavity2d(128), ifc.cavity2d(256)], want_fields=False)  # autotune
    res, fields, bms = ifc.batch_solve(cases)
    sample = list(range(0, len(cases), every))
    plain_ms, worst, conv_p = 0.0, 0.0, 0
    for q in sample:
        s = ifc.Solver(cases[q])
        st = s.solve()
        plain_ms += st["device_ms"]
        conv_p += int(st["converged"])
        for f in ("u", "v"):
            worst = max(worst, rel_l2(fields[q][f], s.get(f)))
        s.close()
    work = [r["outer_iterations"] * c["nx"] * c["ny"] for r, c in zip(res, cases)]
    plain_est = plain_ms * sum(work) / sum(work[q] for q in sample)
    return {"workload": "batch_cavity2d_256", "cases": len(cases),
            "solves_per_s": len(cases) / (bms * 1e-3), "batch_ms": bms,
            "plain_loop": {"cases_timed": len(sample), "which": f"every {every}th case", "device_ms": plain_ms,
                           "device_ms_scaled_to_all": plain_est,
                           "scaling": "by cell-iterations: sum over all cases / sum over the sampled cases",
                           "solves_per_s": len(sample) / (plain_ms * 1e-3)},
            "speedup_vs_plain": plain_est / bms,
            "converged": {"batch": int(sum(r["converged"] for r in res)), "of": len(cases),
                          "plain_sampled": conv_p},
            "max_rel_l2_batch_vs_plain_uv_sampled": worst, "criterion": "per-field relative 1e-5"}


def adjoint_summary(nprof: int, fd_every: int) -> dict:
    """nprof seeded inlet profiles of the 256 x 64 channel: FP32 primal solve
    and FP64 adjoint device times; the first profile's gradient against FP64
    central differences for every fd_every-th inlet parameter and mu."""
    import numpy as np

    import ifc

    nx, ny = 256, 64
    base = ifc.channel2d(nx, ny, inlet_profile=adjoint_profile(0))
    s32 = ifc.Solver(base)
    s32.solve()
    s32.adjoint(tol=1e-8)  # warm-up
    rows = []
    for k in range(nprof):
        s32.set_inlet_profile(adjoint_profile(k, ny))
        s32.set_uniform()
        st = s32.solve()
        dth, res = s32.adjoint(tol=1e-8)
        rows.append((st["device_ms"], res["device_ms"], dth, res["dJ_dmu"], st["converged"] and res["converged"]))
    s32.close()
    theta = adjoint_profile(0, ny)
    c64 = dict(base, precision="d", inlet_profile=theta)
    s64 = ifc.Solver(c64)
    s64.solve()
    s64.iterate(4000)
    keys = ("u", "v", "p", "uf", "vf")
    state = {f: s64.get(f) for f in keys}

    def J_from(sol):
        for f, a_ in state.items():
            sol.set(f, a_)
        sol.iterate(3000)
        p_ = sol.get("p").reshape(ny, nx)
        return float(p_[:, 0].mean() - p_[:, -1].mean())

    errs = []
    for j in range(0, ny, fd_every):
        h = 1e-3 * theta[j]
        Js = []
        for sgn in (1.0, -1.0):
            tt = theta.copy()
            tt[j] += sgn * h
            s64.set_inlet_profile(tt)
            Js.append(J_from(s64))
        fd = (Js[0] - Js[1]) / (2 * h)
        errs.append(abs(rows[0][2][j] - fd) / abs(fd))
    s64.close()
    mu = base["dynamicViscosity"]
    Jm = []
    for sgn in (1.0, -1.0):
        sm = ifc.Solver(dict(c64, dynamicViscosity=mu + sgn * 1e-3 * mu))
        Jm.append(J_from(sm))
        sm.close()
    fdmu = (Jm[0] - Jm[1]) / (2e-3 * mu)
    errs.append(abs(rows[0][3] - fdmu) / abs(fdmu))
    ratio = np.array([r[1] / r[0] for r in rows])
    return {"workload": "channel2d_256x64_adjoint", "profiles": nprof,
            "adjoint_over_primal": float(ratio.mean()), "ratio_max": float(ratio.max()), "bound": 3.0,
            "primal_ms_mean": float(np.mean([r[0] for r in rows])),
            "adjoint_ms_mean": float(np.mean([r[1] for r in rows])),
            "all_converged": bool(all(r[4] for r in rows)),
            "fd_check": {"profile": 0, "parameters": len(errs), "which": f"theta[::{fd_every}] and mu",
                         "fd": "FP64 central, relative step 1e-3", "max_rel_err": float(max(errs)),
                         "bound": 1e-4}}


ADJ_WORKLOAD = "channel2d_256x64_adjoint"


def adjoint_profile(k: int, ny: int = 64):
    import numpy as np

    return 0.001 + np.random.default_rng(k).normal(0.0, 1e-4, ny)


def run_adjoint(args):
    """Differentiation form: for each seeded inlet profile theta (64 values,
    0.001 m/s + N(0, 1e-4)) an FP32 primal solve of the 256 x 64 channel to
    the standard per-field criterion 1e-5, then the FP64 discrete adjoint
    (tol 1e-8) giving dJ/dtheta and dJ/dmu of J = inlet-minus-outlet mean
    pressure drop.  The metric is adjoint device time / primal device time.
    A second gradient is taken after POLISH further primal iterations (its
    error shows how much of the first one's is the primal's stopping point).
    The first --fd-profiles profiles are checked against central finite
    differences (relative step 1e-3) of FP64 solves warm-started from the
    converged FP64 state, for all 65 parameters (two host threads, each with
    its own handle and stream)."""
    import threading

    import numpy as np
    import torch

    import ifc

    POLISH = 300
    world, rank, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    nx, ny = 256, 64
    base_cfg = ifc.channel2d(nx, ny, inlet_profile=adjoint_profile(0))
    s32 = ifc.Solver(base_cfg)
    # warm-up: one untimed primal + adjoint
    s32.solve()
    s32.adjoint(tol=1e-8)
    rows = []
    clocks = ClockSampler(local)
    clocks.start()
    for k in range(args.profiles):
        theta = adjoint_profile(k, ny)
        t0 = time.perf_counter()
        s32.set_inlet_profile(theta)
        s32.set_uniform()
        st = s32.solve()
        dth, res = s32.adjoint(tol=1e-8)
        wall = time.perf_counter() - t0
        stp = s32.iterate(POLISH)
        dth_p, res_p = s32.adjoint(tol=1e-8)
        rows.append({"theta": theta, "primal_ms": st["device_ms"], "primal_its": st["outer_iterations"],
                     "primal_converged": st["converged"], "adj_ms": res["device_ms"], "adj_its": res["iterations"],
                     "adj_converged": res["converged"], "dth": dth, "dmu": res["dJ_dmu"], "J": res["objective"],
                     "wall_ms": wall * 1e3, "launches": st["kernel_launches"] + res["kernel_launches"],
                     "polish_ms": stp["device_ms"], "dth_p": dth_p, "dmu_p": res_p["dJ_dmu"]})
    clk = clocks.stop()

    mu = base_cfg["dynamicViscosity"]
    keys = ("u", "v", "p", "uf", "vf")

    def J_of(sol):
        p = sol.get("p").reshape(ny, nx)
        return float(p[:, 0].mean() - p[:, -1].mean())

    def run_from(sol, base):
        for f, a in base.items():
            sol.set(f, a)
        sol.iterate(args.fd_iters)
        return J_of(sol)

    fd_rows = []
    t_fd = time.perf_counter()
    for k in range(min(args.fd_profiles, args.profiles)):
        theta = rows[k]["theta"]
        c64 = dict(base_cfg, precision="d", inlet_profile=theta)
        s64 = ifc.Solver(c64)
        s64.solve()
        s64.iterate(4000)
        base = {f: s64.get(f) for f in keys}
        s64.close()
        fd = np.empty(ny)
        fdmu = [0.0]

        def worker(js, with_mu):
            sol = ifc.Solver(c64)
            for j in js:
                h = 1e-3 * theta[j]
                Js = []
                for sgn in (1.0, -1.0):
                    tt = theta.copy()
                    tt[j] += sgn * h
                    sol.set_inlet_profile(tt)
                    Js.append(run_from(sol, base))
                fd[j] = (Js[0] - Js[1]) / (2 * h)
            sol.close()
            if with_mu:
                h = 1e-3 * mu
                Jm = []
                for sgn in (1.0, -1.0):
                    sm = ifc.Solver(dict(c64, dynamicViscosity=mu + sgn * h))
                    Jm.append(run_from(sm, base))
                    sm.close()
                fdmu[0] = (Jm[0] - Jm[1]) / (2 * h)

        th = [threading.Thread(target=worker, args=(list(range(0, ny, 2)), True)),
              threading.Thread(target=worker, args=(list(range(1, ny, 2)), False))]
        for t in th:
            t.start()
        for t in th:
            t.join()
        rec = {"profile": k}
        for tag, dth, dmu in (("", rows[k]["dth"], rows[k]["dmu"]), ("polished_", rows[k]["dth_p"], rows[k]["dmu_p"])):
            rec[tag + "max_rel_err_theta"] = float((np.abs(dth - fd) / np.abs(fd)).max())
            rec[tag + "rel_err_mu"] = float(abs(dmu - fdmu[0]) / abs(fdmu[0]))
        fd_rows.append(rec)
    t_fd = time.perf_counter() - t_fd
    s32.close()

    pm = np.array([r["primal_ms"] for r in rows])
    am = np.array([r["adj_ms"] for r in rows])
    ratio = am / pm
    errs = [max(r["max_rel_err_theta"], r["rel_err_mu"]) for r in fd_rows]
    errs_p = [max(r["polished_max_rel_err_theta"], r["polished_rel_err_mu"]) for r in fd_rows]
    line = {
        "metric": "adjoint/primal device time", "value": float(ratio.mean()), "unit": "x",
        "higher_is_better": False, "n_gpus": 1, "steps": args.profiles, "warmup": 1,
        "ms_per_step": float((pm + am).mean()), "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 primal, f64 adjoint", "data": "synthetic: seeded inlet profiles 0.001 + N(0, 1e-4) m/s",
        "config": {"workload": ADJ_WORKLOAD, "nx": nx, "ny": ny, "parameters": ny + 1,
                   "objective": "mean p(first column) - mean p(last column)",
                   "primal": "FP32, per-field criterion 1e-5 from rest", "adjoint_tol": 1e-8,
                   "form": "single-launch adjoint solve (k_adjoint2d)"},
        "primal_ms_mean": float(pm.mean()), "adjoint_ms_mean": float(am.mean()),
        "ratio_max": float(ratio.max()),
        "primal_iterations_mean": float(np.mean([r["primal_its"] for r in rows])),
        "adjoint_iterations_mean": float(np.mean([r["adj_its"] for r in rows])),
        "polish": {"outer_iterations": POLISH, "ms_mean": float(np.mean([r["polish_ms"] for r in rows]))},
        "all_converged": bool(all(r["primal_converged"] and r["adj_converged"] for r in rows)),
        "e2e": {"value": float(np.mean([r["wall_ms"] for r in rows])), "unit": "ms per gradient (host wall clock)",
                "h2d_bytes_per_step": ny * 8, "d2h_bytes_per_step": (ny + 1) * 8},
        "grad_vs_fd": {"profiles_checked": len(fd_rows), "parameters_each": ny + 1, "fd_step": "1e-3 relative",
                       "fd_precision": "FP64", "fd_iters_from_base": args.fd_iters, "fd_seconds": t_fd,
                       "max_rel_err": float(max(errs)) if errs else None,
                       "max_rel_err_polished": float(max(errs_p)) if errs_p else None,
                       "bound": 1e-4, "per_profile": fd_rows},
        "gpu_launches": int(sum(r["launches"] for r in rows)),
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)


PREC_WORKLOAD = "cavity3d_128_re400"


def run_precision(args):
    """Precision form: the 3D lid-driven cavity (128^3, Re 400, lid u=1 on the
    top wall, solver settings of the 2D cavity: alpha 0.7/0.3, GS 5/5/5/50).
    FP32 sweeps and assembly, FP64 norms, mass imbalance and p' pinning.
      (a) FP32 from rest to convergence by the reference's own rule (every
          relative norm over the running max of the pressure norm, 1e-5) --
          the time to convergence;
      (b) FP32 by the per-field rule on FP64 residuals (each momentum residual
          and the mass imbalance over its own running max, 1e-5), up to
          --max-outer iterations, with the ratios it reaches;
      (c) the same solver built in double, from rest, to the rule of (b);
      (d) the double build for exactly as many iterations as (a): the L2/Linf
          error of (a)'s u, v, w, p (p modulo its mean) against it;
    and the device time and compulsory bytes of each stage of one outer
    iteration of the FP32 handle."""
    import numpy as np
    import torch

    import ifc

    world, rank, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    n = args.n3d
    cfg = ifc.cavity3d(n, re=400.0, numOuterIter=args.max_outer, convection_scheme=CONVECTION,
                       criterion=ifc.CRIT_RESIDUAL)
    clocks = ClockSampler(local)
    clocks.start()
    sres = ifc.Solver(dict(cfg, precision="f"))
    stres = sres.solve()
    sres.close()
    s32 = ifc.Solver(dict(cfg, precision="f", criterion=ifc.CRIT_REFERENCE))
    st32 = s32.solve()
    k32 = st32["outer_iterations"]
    s64 = ifc.Solver(dict(cfg, precision="d"))
    st64 = s64.solve()
    s64.close()
    s64 = ifc.Solver(dict(cfg, precision="d"))
    st64e = s64.iterate(k32)
    clk = clocks.stop()

    def fields(s):
        f = {k: s.get(k).astype(np.float64) for k in ("u", "v", "w", "p")}
        f["p"] -= f["p"].mean()
        return f

    a, b = fields(s32), fields(s64)
    err = {k: {"rel_l2": float(np.linalg.norm(a[k] - b[k]) / np.linalg.norm(b[k])),
               "linf_rel": float(np.abs(a[k] - b[k]).max() / np.abs(b[k]).max())} for k in a}
    N = n ** 3
    byte_model = prec_byte_model(cfg, N)
    peak, peak_kind = measured_peaks()
    stages = {}
    for name in ("mom_solve", "rhie_chow", "pcorr_solve", "update"):
        ms_, nl = s32.time_stage(name, reps=5)
        gbs = byte_model[name] / (ms_ * 1e-3) / 1e9
        stages[name] = {"ms": ms_, "launches": nl, "compulsory_bytes": byte_model[name], "gbs": gbs,
                        "frac_of_peak": gbs / peak}
    line = {
        "metric": "time to convergence", "value": st32["device_ms"] / 1e3, "unit": "s", "higher_is_better": False,
        "n_gpus": 1, "steps": 1, "warmup": 0, "ms_per_step": st32["device_ms"], "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 sweeps, f64 reductions", "data": "synthetic: flow from rest",
        "config": {"workload": PREC_WORKLOAD if CONVECTION == "upwind" else f"{PREC_WORKLOAD}_{CONVECTION}", "n": n,
                   "criterion": "the reference's rule (every norm over the p-norm max), 1e-5",
                   "max_outer": args.max_outer, "convection": CONVECTION},
        "fp32": {"converged": bool(st32["converged"]), "outer_iterations": k32,
                 "ms_per_outer_iteration": st32["device_ms"] / max(k32, 1),
                 "cell_updates_per_s": st32["cell_updates"] / (st32["device_ms"] * 1e-3)},
        "fp32_residual_rule": {"converged": bool(stres["converged"]), "outer_iterations": stres["outer_iterations"],
                               "seconds": stres["device_ms"] / 1e3,
                               "ratios_reached": {q: stres[f"rel_{q}"] for q in ("u", "v", "w", "p")}},
        "fp64_same_rule": {"converged": bool(st64["converged"]), "outer_iterations": st64["outer_iterations"],
                           "seconds": st64["device_ms"] / 1e3,
                           "ms_per_outer_iteration": st64["device_ms"] / max(st64["outer_iterations"], 1)},
        "error_vs_fp64_build_equal_iterations": err,
        "stages_fp32": stages, "hbm_peak_gbs": peak, "peak_kind": peak_kind,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    s32.close()
    s64.close()


def run_batch(args):
    """Batched form: --cases lid-driven cavities (nx, ny drawn from 32..256 in
    steps of 32, Re log-uniform in [10, 1000], seed 0), each to the per-field
    criterion 1e-5, in one persistent launch (ifc_batch_solve), against the
    plain per-case loop (one handle per case, ifc_solve); solves/s of both and
    the largest field difference between them."""
    import numpy as np
    import torch

    import ifc

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    cases = ifc.batch_cases(args.cases, seed=0)
    mine = ifc.shard_cases([ifc.case_weight(c) for c in cases], rank, world) if world > 1 else list(range(len(cases)))
    sub = [cases[i] for i in mine]
    # warm-up: one case of every size class, which also runs the autotuner
    # (it times each variant once per class and process); its time is reported
    t0 = time.perf_counter()
    ifc.batch_solve([ifc.cavity2d(32), ifc.cavity2d(128), ifc.cavity2d(256)], want_fields=False)
    tune_s = time.perf_counter() - t0
    clocks = ClockSampler(local)
    clocks.start()
    res, fields, bms = ifc.batch_solve(sub)
    clk = clocks.stop()
    case_its = sum(r["outer_iterations"] for r in res)
    updates = sum(r["outer_iterations"] * c["nx"] * c["ny"] * (c["nIter_u"] + c["nIter_v"] + c["nIter_p"])
                  for r, c in zip(res, sub))
    variants = {}
    for r, c in zip(res, sub):
        key = f"{r['tile_x']}x{r['tile_y']}/ks{r['sweeps_per_pass']}" if r["tile_x"] else "rows/ks1"
        variants[key] = variants.get(key, 0) + 1
    plain_ms, worst, nconv_b, nconv_p = 0.0, 0.0, 0, 0
    for k, c in enumerate(sub):
        s = ifc.Solver(c)
        st = s.solve()
        plain_ms += st["device_ms"]
        nconv_p += int(st["converged"])
        nconv_b += int(res[k]["converged"])
        for f in ("u", "v"):
            a = fields[k][f].astype(np.float64)
            b = s.get(f).astype(np.float64)
            worst = max(worst, float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)))
        s.close()
    local_res = {"solves": len(sub), "updates": updates, "case_its": case_its, "conv_batch": nconv_b,
                 "conv_plain": nconv_p, "batch_ms": bms, "plain_ms": plain_ms, "worst": worst}
    tot = batch_totals(local_res, world, torch.device("cuda", local))
    line = {
        "metric": "converged solves/s", "value": tot["solves"] / (tot["batch_ms"] * 1e-3), "unit": "solves/s",
        "higher_is_better": True, "n_gpus": world, "steps": 1, "warmup": 1, "ms_per_step": tot["batch_ms"],
        "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic: seeded cavity cases from rest",
        "config": {"workload": f"batch_cavity2d_{args.cases}", "cases": int(tot["solves"]),
                   "sizes": "nx, ny in {32..256 step 32}", "re": "log-uniform [10, 1000]",
                   "criterion": "per-field relative 1e-5",
                   "sharding": "greedy longest-first by ifc.case_weight, no data-path collective"},
        "plain_loop": {"solves_per_s": tot["solves"] / (tot["plain_ms"] * 1e-3), "device_ms": tot["plain_ms"],
                       "note": "per rank the sum of per-case ifc_solve device times (handle creation excluded), "
                               "max over ranks"},
        "speedup_vs_plain": tot["plain_ms"] / tot["batch_ms"],
        "case_outer_iterations": int(tot["case_its"]),
        "cell_updates_per_s": tot["updates"] / (tot["batch_ms"] * 1e-3),
        "variants_used_rank0": variants,
        "autotune_and_warmup_seconds": tune_s,
        "converged": {"batch": int(tot["conv_batch"]), "plain": int(tot["conv_plain"]), "of": int(tot["solves"])},
        "max_rel_l2_batch_vs_plain_uv": tot["worst"],
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


def batch_totals(local: dict, world: int, device) -> dict:
    """Whole-job totals of the batch form over the ranks of the process group:
    solves, cell-updates, case iterations and converged counts are summed;
    device times (each rank's batch and plain-loop time) and the worst field
    difference take the maximum.  world == 1 returns the local values."""
    if world == 1:
        return dict(local)
    import torch
    import torch.distributed as dist

    sums = ("solves", "updates", "case_its", "conv_batch", "conv_plain")
    maxes = ("batch_ms", "plain_ms", "worst")
    a = torch.tensor([float(local[k]) for k in sums], dtype=torch.float64, device=device)
    b = torch.tensor([float(local[k]) for k in maxes], dtype=torch.float64, device=device)
    dist.all_reduce(a, op=dist.ReduceOp.SUM)
    dist.all_reduce(b, op=dist.ReduceOp.MAX)
    out = dict(zip(sums, a.tolist()))
    out.update(zip(maxes, b.tolist()))
    return out


ENERGY_SWEEPS = 2000


def run_energy(args):
    """Energy form: the temperature on the developed 512 x 128 channel flow
    (600 outer iterations from rest), TempBCs of the reference's config.h
    (293 K south wall, 373 K north wall, zero gradient elsewhere).  A step is
    one ifc_solve_energy call of ENERGY_SWEEPS unrelaxed red-black sweeps
    (tol 0: fixed work), continuing from the previous step's T; the metric is
    temperature cell-updates/s.  e2e uploads T from pinned host memory before
    and reads it back after every call."""
    import numpy as np
    import torch

    import ifc

    world, rank, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    cfg = ifc.channel2d(512, 128, TempBC_type=[1, 1, 0, 0, 1, 1], TempBC_val=[0.0, 0.0, 293.0, 373.0, 0.0, 0.0])
    s = ifc.Solver(cfg)
    s.iterate(600)
    N = s.N
    for _ in range(max(args.warmup, 1)):
        s.solve_energy(max_sweeps=ENERGY_SWEEPS, tol=0.0)
    clocks = ClockSampler(local)
    clocks.start()
    ms = []
    for _ in range(args.steps):
        r = s.solve_energy(max_sweeps=ENERGY_SWEEPS, tol=0.0)
        ms.append(r["device_ms"])
    clk = clocks.stop()
    # end to end: T from pinned host memory, the solve, T back to the host
    t_host = torch.from_numpy(s.get("T")).pin_memory()
    t_back = torch.empty_like(t_host).pin_memory()
    lib = ifc.load()
    fid = ifc.FIELDS.index("T")
    nbytes = N * 4
    e2e_ms = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        assert lib.ifc_set_field(s._h, fid, C.c_void_p(t_host.data_ptr()), nbytes) == 0
        s.solve_energy(max_sweeps=ENERGY_SWEEPS, tol=0.0)
        assert lib.ifc_get_field(s._h, fid, C.c_void_p(t_back.data_ptr()), nbytes) == 0
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    updates = N * ENERGY_SWEEPS
    value = updates * len(ms) / (sum(ms) * 1e-3)
    peak, peak_kind = measured_peaks()
    achieved = BYTES_PER_UPDATE_2D * updates / (statistics.mean(ms) * 1e-3) / 1e9
    cpu = None
    if not args.no_cpu_baseline:
        # the oracle's numpy restatement of the same sweeps, one core, on the
        # same coefficients, for a bounded number of sweeps
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O

        coef, src = O.energy_assemble(cfg, s.get("uf"), s.get("vf"), None, "f")
        t = s.get("T").copy()
        t0 = time.perf_counter()
        nsw = 0
        while time.perf_counter() - t0 < args.cpu_seconds:
            t, _ = O.energy_sweeps(cfg, coef, src, t, 20, "f")
            nsw += 20
        dt = time.perf_counter() - t0
        cpu = {"value": N * nsw / dt, "unit": "cell-updates/s", "cores": 1, "kind": "port",
               "sample": f"{nsw} red-black sweeps of the same system, numpy restatement (oracle.energy_sweeps), "
                         f"{dt:.1f} s on one core of {host_cpu()}"}
    line = {
        "metric": "temperature cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": statistics.mean(ms), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic: channel flow from rest, 600 outer iterations",
        "config": {"workload": "energy_channel2d_512x128", "sweeps_per_step": ENERGY_SWEEPS,
                   "linear_solver": "red-black Gauss-Seidel, 5 sweeps per blocked pass, one cooperative launch",
                   "l2": "not flushed: the 1.6 MB system stays in L2 by design"},
        "e2e": {"value": updates * len(e2e_ms) / (sum(e2e_ms) * 1e-3), "unit": "cell-updates/s",
                "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes},
        "roofline": {"bound": "hbm", "kernel": "k_coef_solve2d (the whole solve, one cooperative launch)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": profiled_traffic("k_coef_solve2d"),
                     "note": "reference-form 32 B per cell-update; the system lives in L2"},
        "clocks": clk,
    }
    if cpu:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    s.close()


SLAB_WORKLOADS = (
    # (name, config, slab counts, sweeps per exchange, outer iterations timed)
    ("channel2d_4096x2048", lambda ifc: ifc.channel2d(4096, 2048), (2, 4), None, 6),
    ("cavity3d_128x128x512", lambda ifc: ifc.cavity3d(128, nz=512), (2, 4), 4, 3),
)


def slab_record(cfg: dict, counts, k, n: int, warm: int) -> dict:
    """One slab workload: the whole grid by ifc_iterate, then the same solve
    through ifc_slabs in 1 slab (the steps one stage at a time) and in each
    count of overlapping slabs on this GPU, ms per outer iteration (host clock
    around synchronised iterations: the slabs' steps are host-orchestrated),
    with the halo traffic and a bit-for-bit check of u against the whole
    grid's after the same iterations."""
    import numpy as np
    import torch

    import ifc
    import ifc_slabs as S

    def timed(fn, reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fn(reps)
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) * 1e3 / reps

    dim = cfg["dim"]
    sweeps = cfg["nIter_u"] + cfg["nIter_v"] + (cfg["nIter_w"] if dim == 3 else 0) + cfg["nIter_p"]
    cells = cfg["nx"] * cfg["ny"] * (cfg["nz"] if dim == 3 else 1)
    whole_cfg = dict(cfg, tol_u=0.0, tol_v=0.0, tol_w=0.0, tol_p=0.0, tol_mass=0.0, pin_pressure=0)
    s = ifc.Solver(whole_cfg)
    s.iterate(warm)
    ms_whole = timed(s.iterate, n)
    ref_u = s.get("u")
    s.close()
    rec = {"cells": cells, "sweeps_per_outer": sweeps, "outer_iterations_timed": n,
           "sweeps_per_exchange": k or "whole stages", "whole_ifc_iterate_ms_per_outer": ms_whole}
    for parts in (1,) + tuple(counts):
        with S.SlabSolver(cfg, parts=parts, sweeps_per_exchange=k) as ss:
            ss.iterate(warm)
            x0 = ss.exchanges
            b0 = ss.halo.bytes if ss.halo is not None else 0
            ms = timed(ss.iterate, n)
            held = sum(g1 - g0 for g0, g1 in ss.plan.span)
            rec["stages_1_slab" if parts == 1 else f"slabs_{parts}"] = {
                "ms_per_outer": ms, "cell_updates_per_s": cells * sweeps / (ms * 1e-3),
                "halo_rows": ss.plan.halo, "rows_held_over_rows": held / ss.plan.cells,
                "exchanges_per_outer": (ss.exchanges - x0) / n,
                "halo_bytes_per_outer": ((ss.halo.bytes if ss.halo is not None else 0) - b0) / n,
                "bitwise_equal_to_whole": bool(np.array_equal(ss.gather("u"), ref_u))}
    return rec


def slabs_summary() -> dict:
    """The compact slab record of the default line: the 4096 x 2048 channel,
    whole and in 2 and 4 slabs, 3 outer iterations each."""
    import ifc

    name, make, counts, k, _ = SLAB_WORKLOADS[0]
    return {"workload": name, **slab_record(make(ifc), counts, k, 3, 1)}


def run_slabs(args):
    """Slab decomposition on one GPU (ifc_slabs): each workload's grid solved
    whole (ifc_iterate, and the same steps one stage at a time) and cut into
    2 and 4 overlapping slabs whose halos are refreshed by device copies after
    every step.  The slabs share one device, so their time is the sum of the
    slabs' steps, the halo copies and the host's step-by-step orchestration:
    the cost of the decomposition itself, the part a multi-GPU run adds to
    each GPU's share of the work.  Each decomposed solve is checked bit for
    bit against the whole grid's after the same iterations."""
    import torch

    import ifc

    world, rank, local = dist_env()
    if world > 1:
        run_slabs_ranks(args, world, rank, local)
        return
    torch.cuda.set_device(local)
    clocks = ClockSampler(local)
    clocks.start()
    records = {name: slab_record(make(ifc), counts, k, n, max(args.warmup, 1))
               for name, make, counts, k, n in SLAB_WORKLOADS}
    clk = clocks.stop()
    base = records[SLAB_WORKLOADS[0][0]]
    line = {
        "metric": METRIC, "value": base["slabs_4"]["cell_updates_per_s"], "unit": METRIC, "n_gpus": 1,
        "steps": SLAB_WORKLOADS[0][4], "warmup": args.warmup, "ms_per_step": base["slabs_4"]["ms_per_outer"],
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: flows from rest",
        "config": {"workload": "slabs: " + ", ".join(w[0] for w in SLAB_WORKLOADS),
                   "headline_value": "channel2d_4096x2048 in 4 slabs on one GPU",
                   "timing": "host wall clock around synchronised outer iterations (the slabs' steps are host-orchestrated)"},
        "records": records,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def run_slabs_ranks(args, world: int, rank: int, local: int):
    """Slab form on N GPUs (torchrun, one process per GPU): each workload's
    grid cut into N slabs, one per rank, halos swapped with the two neighbour
    ranks by NCCL send/receive after every step (ifc_slabs.DistHalo).  Time
    per outer iteration is the max over ranks of host-clock time around
    synchronised iterations (barrier on both sides); strong scaling (the grid
    is fixed).  Rank 0 then checks u bit for bit against the whole grid solved
    on its own GPU."""
    from datetime import timedelta

    import numpy as np
    import torch
    import torch.distributed as dist

    import ifc
    import ifc_slabs as S

    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    records = {}
    for name, make, _, k, n in SLAB_WORKLOADS:
        cfg = make(ifc)
        dim = cfg["dim"]
        sweeps = cfg["nIter_u"] + cfg["nIter_v"] + (cfg["nIter_w"] if dim == 3 else 0) + cfg["nIter_p"]
        cells = cfg["nx"] * cfg["ny"] * (cfg["nz"] if dim == 3 else 1)
        ss = S.SlabSolver(cfg, sweeps_per_exchange=k, group=dist.group.WORLD)
        warm = max(args.warmup, 1)
        ss.iterate(warm)
        x0, b0 = ss.exchanges, ss.halo.bytes
        torch.cuda.synchronize()
        dist.barrier()
        t0 = time.perf_counter()
        ss.iterate(n)
        torch.cuda.synchronize()
        dist.barrier()
        ms = torch.tensor([(time.perf_counter() - t0) * 1e3 / n], dtype=torch.float64, device="cuda")
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
        u = ss.gather("u")
        rec = {"cells": cells, "slabs": world, "halo_rows": ss.plan.halo,
               "sweeps_per_exchange": k or "whole stages", "ms_per_outer": float(ms[0]),
               "cell_updates_per_s": cells * sweeps / (float(ms[0]) * 1e-3),
               "exchanges_per_outer": (ss.exchanges - x0) / n,
               "halo_bytes_per_outer_this_rank": (ss.halo.bytes - b0) / n}
        ss.close()
        if rank == 0:
            w = ifc.Solver(dict(cfg, tol_u=0.0, tol_v=0.0, tol_w=0.0, tol_p=0.0, tol_mass=0.0, pin_pressure=0))
            w.iterate(warm + n)
            rec["bitwise_equal_to_whole"] = bool(np.array_equal(u, w.get("u")))
            w.close()
        records[name] = rec
        dist.barrier()
    if rank == 0:
        base = records[SLAB_WORKLOADS[0][0]]
        print(json.dumps({
            "metric": METRIC, "value": base["cell_updates_per_s"], "unit": METRIC, "n_gpus": world,
            "steps": SLAB_WORKLOADS[0][4], "warmup": args.warmup, "ms_per_step": base["ms_per_outer"],
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: flows from rest",
            "config": {"workload": "slabs: " + ", ".join(w[0] for w in SLAB_WORKLOADS),
                       "headline_value": f"channel2d_4096x2048 in {world} slabs, one per GPU",
                       "timing": "host clock around synchronised outer iterations, max over ranks"},
            "records": records}), flush=True)
    dist.barrier()
    dist.destroy_process_group()


def run_convergence(args):
    """Time to convergence on the 64^2 lid-driven cavity (Re 100, alpha
    0.7/0.3, GS 5/5/50, tolerance 1e-5, from rest): this library under the
    reference's own stopping rule and under the per-field rule, the
    reference's CUDA build under its own rule (oracle/_ref, one
    Solver::solve() call from a new Solver, wall clock), and the serial
    oracle under the per-field rule.  Red-black and the reference's chaotic
    Gauss-Seidel take different iteration counts, so times are compared at
    convergence, each by its own count."""
    import re
    import numpy as np
    import torch

    import ifc

    world, rank, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    cfg = ifc.cavity2d(64)
    ours = {}
    for name, crit in (("reference_rule", ifc.CRIT_REFERENCE), ("per_field_rule", ifc.CRIT_PER_FIELD)):
        ifc.Solver(dict(cfg, criterion=crit)).solve()  # warm-up (graph build, first launch)
        runs = []
        for _ in range(3):
            s = ifc.Solver(dict(cfg, criterion=crit))
            st = s.solve()
            runs.append((st["device_ms"], st["outer_iterations"], st["converged"]))
            s.close()
        ms = sorted(r[0] for r in runs)[1]
        ours[name] = {"ms": ms, "outer_iterations": runs[0][1], "converged": bool(runs[0][2]),
                      "ms_per_iteration": ms / max(runs[0][1], 1)}
    ref = {"unavailable": "reference build not present (oracle/_ref)"}
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_bench_cavity64_converge")
    if os.path.exists(exe):
        times, its = [], None
        for _ in range(3):
            out = subprocess.run([exe, "0", "1"], capture_output=True, text=True, timeout=600)
            if out.returncode != 0:
                break
            rec = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][-1])
            iters = [int(m) for m in re.findall(r"^iter: (\d+)", out.stdout, re.M)]
            its = iters[-1] if iters else None
            times.append(rec["step_ms"][0])
        if times:
            t = sorted(times)[len(times) // 2]
            ref = {"ms": t, "outer_iterations": its, "ms_per_iteration": t / its if its else None,
                   "timing": "wall clock around one Solver::solve() from rest (its own stopping rule)"}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle as O
    from helpers import to_oracle_cfg

    o = O.Oracle(to_oracle_cfg(cfg), "f")
    t0 = time.perf_counter()
    n, nm = o.solve()
    cpu_ms = (time.perf_counter() - t0) * 1e3
    line = {
        "metric": "time to convergence", "value": ours["reference_rule"]["ms"] / 1e3, "unit": "s",
        "higher_is_better": False, "n_gpus": 1, "steps": 3, "warmup": 1,
        "ms_per_step": ours["reference_rule"]["ms"], "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: flow from rest",
        "config": {"workload": "cavity2d_64_re100", "tolerance": 1e-5, "sweeps_u_v_p": [5, 5, 50]},
        "ours": ours, "reference_cuda_build": ref,
        "speedup_vs_reference_build": (ref["ms"] / ours["reference_rule"]["ms"]) if "ms" in ref else None,
        "cpu_baseline": {"value": cpu_ms / 1e3, "unit": "s", "cores": 1, "kind": "port",
                         "sample": f"serial C oracle, FP32 red-black, per-field rule: {n} outer iterations"},
    }
    print(json.dumps(line), flush=True)


def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return
    if CONVECTION != "upwind":
        print(json.dumps({"impl": "reference",
                          "unavailable": "the reference has first-order upwind convection only"}))
        return
    ref_bin = os.path.join(ROOT, "oracle", "_ref", "ref_bench_channel512x128")
    if os.path.exists(ref_bin):
        out = subprocess.run([ref_bin, str(args.warmup), str(args.steps)], capture_output=True, text=True,
                             timeout=1800)
        if out.returncode != 0:
            print(json.dumps({"impl": "reference", "unavailable": f"reference build exited {out.returncode}"}))
            return
        rec = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][-1])
        cfg = workload_cfg()
        N = 512 * 128
        upd = N * (cfg["nIter_u"] + cfg["nIter_v"] + cfg["nIter_p"]) * rec["outer_per_step"]
        step_ms = rec["step_ms"]
        value = upd * len(step_ms) / (sum(step_ms) * 1e-3)
        kind, cores = "reference", 1
        sample = (f"reference CUDA build (src/Solver.cu + include/kernels.cuh, -O2, sm_100a), "
                  f"{rec['outer_per_step']} outer iterations per Solver::solve() call")
        ms_per_step = statistics.mean(step_ms)
    else:
        cpu = cpu_baseline(args.cpu_seconds)
        value = cpu["value"]
        kind, cores, sample = "port", 1, cpu["sample"]
        N = 512 * 128
        ms_per_step = OUTER_PER_STEP * 40 * N / value * 1e3
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic: flow from rest",
        "config": workload_config(),
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    global CONVECTION
    args = parse()
    CONVECTION = args.convection
    if args.impl == "reference":
        run_reference(args)
    elif args.form == "adjoint":
        run_adjoint(args)
    elif args.form == "precision":
        run_precision(args)
    elif args.form == "batch":
        run_batch(args)
    elif args.form == "convergence":
        run_convergence(args)
    elif args.form == "energy":
        run_energy(args)
    elif args.form == "slabs":
        run_slabs(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

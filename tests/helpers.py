"""Shared helpers of the parity tests: seeded states, oracle <-> device
transfers and comparison with an explicit tolerance."""
import numpy as np

import ifc
import oracle as O


def fused_sweeps_per_pass(cfg: dict) -> int:
    """Sweeps per pass of the fused 2D kernels (the library default is 5;
    requests round down to a supported value: 1 2 3 4 5 6 8)."""
    want = int(cfg.get("sweeps_per_pass", 0)) or 5
    for k in (8, 6, 5, 4, 3, 2):
        if want >= k:
            return k
    return 1


def to_oracle_cfg(cfg: dict) -> dict:
    """Oracle config for a library config (same keys; red-black sweeps; the
    inner early-exit rule evaluated at the granularity the device uses: after
    every pass of the fused 2D kernels, after every sweep otherwise)."""
    c = dict(cfg)
    gs = cfg.get("linear_solver", 0) == 0
    c.setdefault("sweep_mode", O.GS_REDBLACK if gs else O.JACOBI)
    c.setdefault("check_every", fused_sweeps_per_pass(cfg) if (gs and cfg["dim"] == 2) else 1)
    c["criterion"] = cfg.get("criterion", O.CRIT_PER_FIELD)
    if "pin_pressure" not in cfg or cfg["pin_pressure"] < 0:
        closed = all(t != ifc.OUTLET for t in cfg["velBC_type"][: 2 * cfg["dim"]])
        c["pin_pressure"] = 1 if closed else 0
    return c


def seeded_state(cfg: dict, seed: int, dtype):
    """Random cell and face fields of moderate size (keeps aC well away from 0)."""
    rng = np.random.default_rng(seed)
    nx, ny = cfg["nx"], cfg["ny"]
    nz = cfg.get("nz", 1) if cfg["dim"] == 3 else 1
    N = nx * ny * nz
    s = {
        "u": rng.uniform(-1, 1, N), "v": rng.uniform(-1, 1, N), "w": rng.uniform(-1, 1, N),
        "p": rng.uniform(-1, 1, N),
        "uf": rng.uniform(-1, 1, (nx + 1) * ny * nz), "vf": rng.uniform(-1, 1, nx * (ny + 1) * nz),
        "wf": rng.uniform(-1, 1, nx * ny * (nz + 1)),
    }
    if cfg["dim"] == 2:
        s["wf"][:] = 0.0
        s["w"][:] = 0.0
    return {k: v.astype(dtype) for k, v in s.items()}


def load_both(o: "O.Oracle", s: "ifc.Solver", state: dict):
    for k, v in state.items():
        o.field(k)[:] = v
        s.set(k, v)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def assert_bitwise(dev, ref, what=""):
    dev = np.asarray(dev)
    ref = np.asarray(ref)
    assert dev.shape == ref.shape, (what, dev.shape, ref.shape)
    bad = np.flatnonzero((dev != ref) & ~(np.isnan(dev) & np.isnan(ref)))
    if bad.size:
        q = bad[0]
        raise AssertionError(f"{what}: {bad.size} of {dev.size} values differ; first at {q}: "
                             f"device {dev[q]!r} oracle {ref[q]!r} (rel L2 {rel_l2(dev, ref):.3e})")

"""Overlapping-slab decomposition of one SIMPLE solve over several handles.

A grid too large for one device is cut along its last axis (y in 2D, z in 3D)
into slabs of whole rows (planes).  Every slab is an ordinary solver handle
over the rows it owns plus ``halo`` rows on each side that its neighbours own;
the handle takes the whole grid's spacing along the cut axis
(``ifc_config.slab_axis_cells``), so its arithmetic on a cell is the
undecomposed solver's.  The outer iteration of the reference
(src/Solver.cu:160-198) runs step by step on every slab, and after each step
the halo rows of every field that step wrote are overwritten with the rows the
neighbours own: one exchange per step, each a single message per neighbour.

Exactness.  Each step computes a value from a bounded stencil.  At a cut edge
the slab's handle sees a domain boundary and computes wrong values next to
it; inside one step that error moves inward by at most one row per red-black
half sweep (two per sweep) and by at most two rows in an assembly, Rhie-Chow,
face or update step.  With the halo deeper than the furthest such reach of
any step, the owned rows never see it, and every owned value equals the
undecomposed solve's bit for bit: ``halo_depth`` gives 2 k + 4 rows for steps
of at most k sweeps.  Two granularities:

* ``sweeps_per_exchange=None``: the stages of ``ifc_run_stage`` (momentum
  assembly fused with all its sweeps, Rhie-Chow, the whole p' solve, update),
  i.e. the device's fastest kernels, four exchanges per outer iteration and
  a halo of 2 max(nIter) + 4 rows.
* ``sweeps_per_exchange=k``: materialised coefficients
  (``IFC_STAGE_MOM_ASSEMBLE`` / ``IFC_STAGE_PCORR_COEF``) and ``ifc_sweep``
  in chunks of k sweeps with an exchange after each; a halo of 2 k + 4 rows,
  for deep p' solves on slabs that are thin against 2 nIter_p.

Red-black colours are global: every slab starts on an even global row.  The
inner early exit of the reference's sweeps compares norms over the whole grid,
so the slabs run every inner sweep (tolerances 0), and pressure pinning (a
mean over the whole grid) is off; the outer loop runs a given number of
iterations and reports the mass imbalance over the whole grid.

Two exchanges: ``LocalHalo`` for slabs held by one process (device copies on
one stream), ``DistHalo`` for one slab per rank of a ``torch.distributed``
group (NCCL point-to-point over NVLink between GPUs; gloo for CPU tensors).
Slabs are created by a factory, by default ``DeviceSlab`` (an ``ifc.Solver``
with torch views of its device fields).  Device slabs enqueue their steps
without a host wait (``ifc_run_stage_async``, ``ifc_sweep_async``), so steps,
halo copies and NCCL transfers follow one another on one stream and the host
waits once per ``iterate`` call.  ``solve`` stops on the whole grid's mass
imbalance; ``gather`` and ``write_vtk`` give the whole grid's fields and VTK
file, byte for byte those of an undecomposed handle.
"""
from __future__ import annotations

import contextlib
import dataclasses

import numpy as np
import torch

import ifc

# Fields each step writes (and that a later step reads), by ifc field name.
_VEL = {2: ["u", "v"], 3: ["u", "v", "w"]}
_FACES = {2: ["uf", "vf"], 3: ["uf", "vf", "wf"]}
_PLANAR = ("mcoef", "pcoef")           # 2*dim+1 coefficient planes of N values each


def step_writes(step: str, dim: int) -> list[str]:
    """Fields written by one step that later steps read."""
    vel, faces = _VEL[dim], _FACES[dim]
    return {
        "face_bc": faces,
        "mom_solve": vel + ["ac"],
        "mom_assemble": ["mcoef", "ac"] + ["src_" + c for c in vel],
        "rhie_chow": faces + ["src_p"],
        "pcorr_coef": ["pcoef"],
        "pcorr_solve": ["pc"],
        "update": ["p"] + vel + faces,
    }[step]


def halo_depth(cfg: dict, sweeps_per_exchange: int | None = None) -> int:
    """Halo rows that keep the owned rows exact: 2 k + 4 (rounded up to even)
    for steps of at most k sweeps (k = the largest nIter, or the chunk)."""
    dim = cfg["dim"]
    counts = [cfg["nIter_u"], cfg["nIter_v"]] + ([cfg["nIter_w"]] if dim == 3 else []) + [cfg["nIter_p"]]
    k = max(counts)
    if sweeps_per_exchange:
        if sweeps_per_exchange < 1:
            raise ValueError("sweeps_per_exchange must be >= 1")
        k = min(k, int(sweeps_per_exchange))
    d = 2 * k + 4
    return d + (d & 1)


@dataclasses.dataclass(frozen=True)
class SlabPlan:
    """Rows (planes) of each slab along the cut axis: ``own[s]`` = [o0, o1)
    owned, ``span[s]`` = [g0, g1) held (owned plus halos)."""
    cells: int
    halo: int
    own: tuple
    span: tuple

    @property
    def parts(self) -> int:
        return len(self.own)

    def halo_lo(self, s: int) -> int:
        return self.own[s][0] - self.span[s][0]

    def halo_hi(self, s: int) -> int:
        return self.span[s][1] - self.own[s][1]


def plan_slabs(cells: int, parts: int, halo: int) -> SlabPlan:
    """Cut ``cells`` rows into ``parts`` slabs of near-equal even-aligned
    ownership.  Every slab must own at least ``halo`` rows (a neighbour's
    halo is then owned by one slab); ValueError otherwise."""
    if parts < 1 or cells < 3:
        raise ValueError("need parts >= 1 and at least 3 cells along the cut axis")
    if parts == 1:
        return SlabPlan(cells, 0, ((0, cells),), ((0, cells),))
    if halo < 2 or halo % 2:
        raise ValueError("halo must be even and >= 2")
    cuts = [0] + [(k * cells // parts) & ~1 for k in range(1, parts)] + [cells]
    own = tuple((cuts[s], cuts[s + 1]) for s in range(parts))
    for o0, o1 in own:
        if o1 - o0 < halo:
            raise ValueError(f"slab of {o1 - o0} rows is thinner than the halo ({halo}): "
                             f"{cells} rows allow at most {cells // halo} slabs at this halo")
    span = tuple((max(0, o0 - halo), min(cells, o1 + halo)) for o0, o1 in own)
    return SlabPlan(cells, halo, own, span)


def slab_config(cfg: dict, plan: SlabPlan, s: int) -> dict:
    """Config of slab s's handle: its rows, the whole grid's spacing and
    extents, every inner sweep run, no pinning."""
    dim = cfg["dim"]
    g0, g1 = plan.span[s]
    c = dict(cfg)
    c["ny" if dim == 2 else "nz"] = g1 - g0
    c["slab_axis_cells"] = plan.cells if plan.parts > 1 else 0
    for q in "uvwp":
        c[f"tol_{q}"] = 0.0
    c["tol_mass"] = 0.0
    c["pin_pressure"] = 0
    c["log_level"] = 0
    prof = cfg.get("inlet_profile")
    if prof is not None:
        prof = np.asarray(prof, dtype=np.float64)
        row = 1 if dim == 2 else cfg["ny"]
        c["inlet_profile"] = prof[g0 * row:g1 * row].copy()
    return c


def field_rows(name: str, dim: int, nx: int, ny: int, nz: int) -> tuple[int, int, int]:
    """(values per row of the cut axis, rows, planes) of a field on a handle of
    nx x ny (x nz) cells: a row is one y-row in 2D, one z-plane in 3D; face
    arrays along the cut axis have one row more; coefficient arrays hold
    2*dim+1 planes of N values, each cut the same way."""
    n = ny if dim == 2 else nz
    row = nx if dim == 2 else nx * ny
    if name == "uf":
        row = nx + 1 if dim == 2 else (nx + 1) * ny
    elif name == "vf":
        if dim == 2:
            return nx, ny + 1, 1
        row = nx * (ny + 1)
    elif name == "wf":
        return nx * ny, nz + 1, 1
    if name in _PLANAR:
        return row, n, 2 * dim + 1
    return row, n, 1


class _DeviceArray:
    """Zero-copy __cuda_array_interface__ over a handle's device field."""

    def __init__(self, ptr: int, n: int, dtype):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": np.dtype(dtype).str,
                                         "data": (ptr, False), "version": 2}


class DeviceSlab:
    """One slab on the current CUDA device: an ifc.Solver handle on the given
    stream and flat torch views of its device fields."""

    def __init__(self, cfg: dict, stream: torch.cuda.Stream | None = None):
        st = stream if stream is not None else torch.cuda.current_stream()
        self.solver = ifc.Solver(dict(cfg, stream=st.cuda_stream))
        self.dtype = self.solver.dtype
        self._views = {}

    def stage(self, name: str):
        # enqueued only: the halo copies or NCCL transfers that follow on the
        # same stream are ordered after it, and sync() reports its outcome
        self.solver.stage(name, wait=False)

    def sync(self):
        self.solver.sync()

    def sweep(self, eq: int, n: int):
        self.solver.sweep(eq, n, norms=False, wait=False)

    def view(self, name: str) -> torch.Tensor:
        v = self._views.get(name)
        if v is None:
            n = self.solver.field_size(name) // np.dtype(self.dtype).itemsize
            v = torch.as_tensor(_DeviceArray(self.solver.device_ptr(name), n, self.dtype), device="cuda")
            self._views[name] = v
        return v

    def zero(self, name: str):
        self.view(name).zero_()

    def close(self):
        self._views.clear()
        self.solver.close()


def _segments(view: torch.Tensor, row: int, planes: int, plane: int, r0: int, r1: int) -> list:
    """Rows [r0, r1) of every plane of a flat field view."""
    return [view[k * plane + r0 * row:k * plane + r1 * row] for k in range(planes)]


class _Layout:
    """Row blocks of slab s for the halo exchange: its halo rows and the owned
    rows its neighbours receive (cell rows; face arrays along the cut axis use
    the same indices for their face rows, the slab's edge face excluded)."""

    def __init__(self, plan: SlabPlan, dim: int, nx: int, ny: int, nz: int):
        self.plan, self.dim = plan, dim
        self.shape = []
        for g0, g1 in plan.span:
            n = g1 - g0
            self.shape.append((nx, n, 1) if dim == 2 else (nx, ny, n))

    def blocks(self, s: int, view: torch.Tensor, name: str) -> dict:
        p, D = self.plan, self.plan.halo
        nx, ny, nz = self.shape[s]
        row, _, planes = field_rows(name, self.dim, nx, ny, nz)
        n = p.span[s][1] - p.span[s][0]
        plane = row * n
        lo, hi = p.halo_lo(s), p.halo_hi(s)
        b = {}
        if lo:
            b["recv_lo"] = _segments(view, row, planes, plane, 0, lo)
            b["send_lo"] = _segments(view, row, planes, plane, lo, lo + D)
        if hi:
            b["recv_hi"] = _segments(view, row, planes, plane, n - hi, n)
            b["send_hi"] = _segments(view, row, planes, plane, n - hi - D, n - hi)
        return b


class LocalHalo:
    """Halo exchange between slabs held by one process: device-to-device
    copies of the owned edge rows into the neighbours' halos, in stream order
    with the slabs' kernels."""

    def __init__(self, layout: _Layout, slabs: dict):
        self.layout, self.slabs = layout, slabs
        self.bytes = 0

    def refresh(self, names: list[str]):
        P = self.layout.plan.parts
        for name in names:
            for s in range(P - 1):
                a = self.layout.blocks(s, self.slabs[s].view(name), name)
                b = self.layout.blocks(s + 1, self.slabs[s + 1].view(name), name)
                for src, dst in zip(a["send_hi"] + b["send_lo"], b["recv_lo"] + a["recv_hi"]):
                    dst.copy_(src)
                    self.bytes += src.numel() * src.element_size()


class DistHalo:
    """Halo exchange for one slab per rank of a process group: the owned edge
    rows of every field of a step are packed into one buffer per neighbour and
    swapped by one grouped send/receive pair (NCCL over NVLink for device
    tensors, gloo for CPU ones), then unpacked into the halo rows."""

    def __init__(self, layout: _Layout, s: int, slab, group=None):
        import torch.distributed as dist

        self.dist, self.layout, self.s, self.slab, self.group = dist, layout, s, slab, group
        P = layout.plan.parts
        g = (lambda r: dist.get_global_rank(group, r)) if group is not None else (lambda r: r)
        self.peer_lo = g(s - 1) if s > 0 else None
        self.peer_hi = g(s + 1) if s < P - 1 else None
        self.bytes = 0
        # every rank of the group takes part in its first collective
        t = torch.zeros(1, dtype=torch.float64, device=slab.view("p").device)
        dist.all_reduce(t, group=group)

    def refresh(self, names: list[str]):
        dist = self.dist
        parts = {"lo": ([], []), "hi": ([], [])}
        for name in names:
            b = self.layout.blocks(self.s, self.slab.view(name), name)
            for side in ("lo", "hi"):
                if "send_" + side in b:
                    parts[side][0].extend(b["send_" + side])
                    parts[side][1].extend(b["recv_" + side])
        ops, unpack = [], []
        for side, peer in (("lo", self.peer_lo), ("hi", self.peer_hi)):
            if peer is None or not parts[side][0]:
                continue
            sbuf = torch.cat(parts[side][0])
            rbuf = torch.empty_like(sbuf)
            ops.append(dist.P2POp(dist.isend, sbuf, peer, self.group))
            ops.append(dist.P2POp(dist.irecv, rbuf, peer, self.group))
            unpack.append((rbuf, parts[side][1]))
            self.bytes += sbuf.numel() * sbuf.element_size()
        if not ops:
            return
        for w in dist.batch_isend_irecv(ops):
            w.wait()
        for rbuf, segs in unpack:
            off = 0
            for seg in segs:
                seg.copy_(rbuf[off:off + seg.numel()])
                off += seg.numel()


class SlabSolver:
    """One SIMPLE solve of ``cfg`` over slabs along its last axis.

    Local form (``group`` None): ``parts`` slabs in this process, on the
    current device.  Distributed form: one slab per rank of ``group`` (a
    torch.distributed process group; slab s on group rank s), each rank
    calling every method in the same order.  ``sweeps_per_exchange``: None
    for whole stages between exchanges, k for chunks of k sweeps.
    ``make_slab(cfg)`` builds one slab (default ``DeviceSlab``)."""

    def __init__(self, cfg: dict, parts: int | None = None, sweeps_per_exchange: int | None = None,
                 group=None, make_slab=None):
        if cfg.get("linear_solver", ifc.GAUSS_SEIDEL) not in (ifc.GAUSS_SEIDEL, ifc.JACOBI):
            raise ValueError("unknown linear solver")
        self.cfg = dict(cfg)
        self.dim = dim = int(cfg["dim"])
        self.k = sweeps_per_exchange
        if group is not None:
            import torch.distributed as dist

            parts, me = dist.get_world_size(group), dist.get_rank(group)
            self.local = [me]
        else:
            parts = 1 if parts is None else int(parts)
            self.local = list(range(parts))
        cells = cfg["ny"] if dim == 2 else cfg["nz"]
        halo = halo_depth(cfg, sweeps_per_exchange) if parts > 1 else 0
        self.plan = plan_slabs(int(cells), parts, halo)
        # Device slabs and their halo copies (or NCCL transfers) share one
        # stream, so every exchange is ordered between the steps around it.
        self.stream = None
        if make_slab is None:
            self.stream = torch.cuda.Stream()
            make_slab = lambda c: DeviceSlab(c, self.stream)  # noqa: E731
        self.slabs = {s: make_slab(slab_config(cfg, self.plan, s)) for s in self.local}
        ny = int(cfg["ny"])
        nz = int(cfg.get("nz", 1)) if dim == 3 else 1
        self.layout = _Layout(self.plan, dim, int(cfg["nx"]), ny, nz)
        self.group = group
        with self._on_stream():
            if group is not None:
                me = self.local[0]
                self.halo = DistHalo(self.layout, me, self.slabs[me], group) if parts > 1 else None
            else:
                self.halo = LocalHalo(self.layout, self.slabs) if parts > 1 else None
        self.iterations = 0
        self.exchanges = 0
        self._faces_set = False
        self._peak_mass = 0.0

    def _on_stream(self):
        return torch.cuda.stream(self.stream) if self.stream is not None else contextlib.nullcontext()

    # ---- one outer iteration, step by step
    def _refresh(self, names):
        if self.halo is not None and names:
            with self._on_stream():
                self.halo.refresh(names)
            self.exchanges += 1

    def _step(self, name: str):
        for s in self.local:
            self.slabs[s].stage(name)
        self._refresh(step_writes(name, self.dim))

    def _sweeps(self, counts: dict):
        """counts: {eq: sweeps}; chunks of k sweeps of every equation, one
        exchange after each chunk."""
        left = dict(counts)
        names = ["u", "v", "w", "pc"]
        while any(n > 0 for n in left.values()):
            written = []
            for eq, n in left.items():
                c = min(self.k, n)
                if c <= 0:
                    continue
                for s in self.local:
                    self.slabs[s].sweep(eq, c)
                left[eq] = n - c
                written.append(names[eq])
            self._refresh(written)

    def iterate(self, n: int) -> dict:
        """n outer iterations (the reference's Solver::solve body,
        src/Solver.cu:160-198, every inner sweep run)."""
        c, vel = self.cfg, list(range(self.dim))
        for _ in range(int(n)):
            if not self._faces_set:
                self._step("face_bc")
                self._faces_set = True
            if self.k is None:
                for st in ("mom_solve", "rhie_chow", "pcorr_solve", "update"):
                    self._step(st)
            else:
                self._step("mom_assemble")
                self._sweeps({e: int(c["nIter_" + "uvw"[e]]) for e in vel})
                self._step("rhie_chow")
                self._step("pcorr_coef")
                with self._on_stream():
                    for s in self.local:
                        self.slabs[s].zero("pc")
                self._sweeps({3: int(c["nIter_p"])})
                self._step("update")
            self.iterations += 1
        for s in self.local:
            self.slabs[s].sync()
        return {"outer_iterations": self.iterations, "exchanges": self.exchanges,
                "halo_bytes": self.halo.bytes if self.halo is not None else 0,
                "norm_mass": self.norm_mass() if self.iterations else 0.0}

    def solve(self, tol_mass: float = 1e-5, max_outer: int | None = None, check_every: int = 50) -> dict:
        """Outer iterations in blocks of check_every until the whole grid's
        mass imbalance falls below tol_mass times its largest value at the
        checks so far (the slab form's stopping rule: the reference's
        per-field rules need correction norms of every field over the whole
        grid), or until the handle has run max_outer outer iterations in all
        (default: the config's numOuterIter)."""
        limit = int(self.cfg["numOuterIter"] if max_outer is None else max_outer)
        st = {"outer_iterations": self.iterations, "converged": False}
        while self.iterations < limit:
            st = self.iterate(min(check_every, limit - self.iterations))
            self._peak_mass = max(self._peak_mass, st["norm_mass"])
            st["rel_mass"] = st["norm_mass"] / self._peak_mass if self._peak_mass > 0 else 0.0
            st["converged"] = st["rel_mass"] < tol_mass
            if st["converged"]:
                break
        return st

    # ---- whole-grid views
    def _owned(self, s: int, name: str) -> torch.Tensor:
        p = self.plan
        nx, ny, nz = self.layout.shape[s]
        row, _, planes = field_rows(name, self.dim, nx, ny, nz)
        if planes != 1:
            raise ValueError(f"{name}: coefficient planes are per slab")
        lo = p.halo_lo(s)
        r1 = lo + (p.own[s][1] - p.own[s][0])
        axis_face = (name == "vf" and self.dim == 2) or name == "wf"
        if axis_face and s == p.parts - 1:
            r1 += 1  # the grid's far boundary face
        return self.slabs[s].view(name)[lo * row:r1 * row]

    def norm_mass(self) -> float:
        """RMS over the whole grid of the p' source (mass imbalance) left by
        the last Rhie-Chow step, FP64 (src/Solver.cu:226-235)."""
        with self._on_stream():
            tot = sum(float(self._owned(s, "src_p").double().pow(2).sum()) for s in self.local)
            if self.group is not None:
                import torch.distributed as dist

                t = torch.tensor([tot], dtype=torch.float64, device=self.slabs[self.local[0]].view("p").device)
                dist.all_reduce(t, group=self.group)
                tot = float(t[0])
        nz = int(self.cfg.get("nz", 1)) if self.dim == 3 else 1
        return float(np.sqrt(tot / (int(self.cfg["nx"]) * int(self.cfg["ny"]) * nz)))

    def gather(self, name: str) -> np.ndarray:
        """The whole grid's field (reference layout) from the owned rows."""
        with self._on_stream():
            mine = {s: self._owned(s, name).cpu().numpy().copy() for s in self.local}
        if self.group is not None:
            import torch.distributed as dist

            got = [None] * self.plan.parts
            dist.all_gather_object(got, mine, group=self.group)
            for d in got:
                mine.update(d)
        return np.concatenate([mine[s] for s in range(self.plan.parts)])

    def write_vtk(self, path: str, binary: bool = False):
        """The whole grid's VTK file (ASCII RECTILINEAR_GRID as
        Solver::writeVTK writes it, src/Solver.cu:301-367, or binary=True for
        legacy VTK BINARY) from the gathered fields, byte for byte the file an
        undecomposed handle writes; in the distributed form rank 0 writes it
        (every rank takes part in the gathers)."""
        f = {n: self.gather(n) for n in ("u", "v", "w", "p", "T")}
        if self.group is not None:
            import torch.distributed as dist

            if dist.get_rank(self.group) != 0:
                return
        ifc.write_vtk_host(self.cfg, f["u"], f["v"], f["w"], f["p"], f["T"], path, binary)

    def load(self, name: str, values):
        """Set a field of the whole grid (reference layout) on every slab."""
        a = torch.as_tensor(np.ascontiguousarray(values).ravel())
        p = self.plan
        for s in self.local:
            nx, ny, nz = self.layout.shape[s]
            row, rows, planes = field_rows(name, self.dim, nx, ny, nz)
            if planes != 1:
                raise ValueError(f"{name}: coefficient planes are per slab")
            g0 = p.span[s][0]
            v = self.slabs[s].view(name)
            with self._on_stream():
                v.copy_(a[g0 * row:(g0 + rows) * row].to(device=v.device, dtype=v.dtype))
                if self.stream is not None:
                    self.stream.synchronize()
        self._faces_set = self._faces_set or name in _FACES[self.dim]

    def close(self):
        for s in self.local:
            self.slabs[s].close()
        self.slabs = {}

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

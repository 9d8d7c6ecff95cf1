"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle is a serial C restatement of the reference solver's kernels
(WanZijun271/IncompFlow-CUDA include/kernels.cuh:10-1005, driven in the order of
src/Solver.cu:153-299); see ifc_oracle.h.  Only tests/, the smoke check and the
cpu_baseline leg of bench.py import this module.  The product never does.

Configurations are plain dicts whose keys follow the reference's config.h names
(``nx``, ``density``, ``dynamicViscosity``, ``velBC_type``, ``nIter_u`` ...); the
same dicts drive the CUDA library's binding.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# IFC_ORACLE_LIB selects another build of the same restatement (the OpenMP one,
# _build/libifc_oracle_omp.so, times the all-cores CPU baseline).
LIB_PATH = os.environ.get("IFC_ORACLE_LIB") or os.path.join(HERE, "_build", "libifc_oracle.so")

GS_LEX, GS_REDBLACK, JACOBI = 0, 1, 2
CRIT_REFERENCE, CRIT_PER_FIELD, CRIT_RESIDUAL = 0, 1, 2
EQ_U, EQ_V, EQ_W, EQ_P = 0, 1, 2, 3
# Convection schemes (0 is the reference's first-order upwind; the others are
# applied by deferred correction).
CONV = {"upwind": 0, "central": 1, "sou": 2, "quick": 3, "minmod": 4, "van_leer": 5}
FIELDS = ["u", "v", "w", "p", "pc", "uf", "vf", "wf", "mcoef", "pcoef", "src_u", "src_v", "src_w", "src_p"]


class OrcConfig(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double), ("ymax", C.c_double),
        ("zmin", C.c_double), ("zmax", C.c_double),
        ("density", C.c_double), ("viscosity", C.c_double),
        ("bc_type", C.c_int * 6), ("bc_val", (C.c_double * 3) * 6),
        ("num_outer_iter", C.c_int), ("n_iter", C.c_int * 4),
        ("relax", C.c_double * 4), ("tol", C.c_double * 4), ("tol_mass", C.c_double),
        ("sweep_mode", C.c_int), ("check_every", C.c_int), ("criterion", C.c_int),
        ("pin_pressure", C.c_int), ("inlet_profile", C.POINTER(C.c_double)),
        ("convection", C.c_int), ("slab_axis_cells", C.c_int),
    ]


class OrcNorms(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("p", "u", "v", "w", "uf", "vf", "wf", "mass",
                                           "rel_p", "rel_u", "rel_v", "rel_w", "rel_uf", "rel_vf", "rel_wf",
                                           "res_u", "res_v", "res_w")] + [
        ("sweeps", C.c_int * 4), ("converged", C.c_int)]

    def as_dict(self):
        d = {n: getattr(self, n) for n, _ in self._fields_ if n != "sweeps"}
        d["sweeps"] = list(self.sweeps)
        return d


def build(force: bool = False) -> str:
    """Compile the oracle with gcc (make -C oracle); returns the library path."""
    if force or not os.path.exists(LIB_PATH) or _stale():
        target = "oracle_omp" if LIB_PATH.endswith("_omp.so") else "oracle"
        subprocess.run(["make", "-s", "-C", HERE, target], check=True)
    return LIB_PATH


def _stale() -> bool:
    t = os.path.getmtime(LIB_PATH)
    return any(os.path.getmtime(os.path.join(HERE, f)) > t
               for f in ("ifc_oracle.c", "ifc_oracle.h", "ifc_oracle_impl.h", "ifc_adjoint_impl.h"))


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        for s, T in (("f", C.c_float), ("d", C.c_double)):
            P = C.c_void_p
            sig = {
                "create": (P, [C.POINTER(OrcConfig)]), "destroy": (None, [P]),
                "field": (C.POINTER(T), [P, C.c_int]), "field_len": (C.c_size_t, [P, C.c_int]),
                "init_face_vel": (None, [P]), "bc_face_vel": (None, [P]), "mom_link_coef": (None, [P]),
                "mom_src": (None, [P]), "bc_mom": (None, [P]), "dc_source": (None, [P]), "sweep": (C.c_double, [P, C.c_int, C.c_int]),
                "linear_solve": (C.c_int, [P, C.c_int, C.POINTER(C.c_double)]),
                "rhie_chow": (None, [P]), "pcorr_link_coef": (None, [P]), "pcorr_src": (C.c_double, [P]),
                "pin_pcorr": (None, [P]), "update_field": (None, [P, C.POINTER(OrcNorms)]),
                "outer_iteration": (C.c_int, [P, C.POINTER(OrcNorms)]),
                "solve": (C.c_int, [P, C.c_int, C.POINTER(OrcNorms)]),
                "iteration_count": (C.c_int, [P]),
            }
            for name, (res, args) in sig.items():
                fn = getattr(_lib, f"orc_{name}_{s}")
                fn.restype = res
                fn.argtypes = args
        PD = C.POINTER(C.c_double)
        _lib.orc_adjoint_apply_d.restype = C.c_int
        _lib.orc_adjoint_apply_d.argtypes = [C.c_void_p] + [PD] * 12
        for s in ("f", "d"):
            fn = getattr(_lib, f"orc_set_iteration_count_{s}")
            fn.restype = None
            fn.argtypes = [C.c_void_p, C.c_int]
    return _lib


def make_struct(cfg: dict) -> tuple[OrcConfig, object]:
    """Fill an OrcConfig from a config dict; returns (struct, keep-alive)."""
    c = OrcConfig()
    c.dim = int(cfg["dim"])
    c.nx, c.ny = int(cfg["nx"]), int(cfg["ny"])
    c.nz = int(cfg.get("nz", 1)) if c.dim == 3 else 1
    for k in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax"):
        setattr(c, k, float(cfg[k]))
    c.density = float(cfg["density"])
    c.viscosity = float(cfg["dynamicViscosity"])
    for f in range(6):
        c.bc_type[f] = int(cfg["velBC_type"][f])
        for q in range(3):
            c.bc_val[f][q] = float(cfg["velBC_val"][f][q])
    c.num_outer_iter = int(cfg["numOuterIter"])
    for q, n in enumerate("uvwp"):
        c.n_iter[q] = int(cfg[f"nIter_{n}"])
        c.relax[q] = float(cfg[f"relax_{n}"])
        c.tol[q] = float(cfg[f"tol_{n}"])
    c.tol_mass = float(cfg["tol_mass"])
    c.sweep_mode = int(cfg.get("sweep_mode", GS_REDBLACK))
    c.check_every = int(cfg.get("check_every", 1))
    c.criterion = int(cfg.get("criterion", CRIT_PER_FIELD))
    c.pin_pressure = int(cfg.get("pin_pressure", 0))
    conv = cfg.get("convection_scheme", 0)
    c.convection = CONV[conv] if isinstance(conv, str) else int(conv)
    c.slab_axis_cells = int(cfg.get("slab_axis_cells", 0))
    keep = None
    prof = cfg.get("inlet_profile")
    if prof is not None:
        keep = np.ascontiguousarray(prof, dtype=np.float64)
        c.inlet_profile = keep.ctypes.data_as(C.POINTER(C.c_double))
    return c, keep


class Oracle:
    """One oracle state (fields, coefficients, running maxima) for one config."""

    def __init__(self, cfg: dict, precision: str = "f"):
        assert precision in ("f", "d")
        self.cfg = dict(cfg)
        self.s = precision
        self.dtype = np.float32 if precision == "f" else np.float64
        self._struct, self._keep = make_struct(cfg)
        self._h = self._fn("create")(C.byref(self._struct))
        if not self._h:
            raise MemoryError("oracle allocation failed")
        self.dim, self.nx, self.ny = self._struct.dim, self._struct.nx, self._struct.ny
        self.nz = self._struct.nz
        self.N = self.nx * self.ny * self.nz

    def _fn(self, name):
        return getattr(lib(), f"orc_{name}_{self.s}")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and lib is not None:  # module globals are gone at interpreter exit
            self._fn("destroy")(h)
            self._h = None

    def field(self, name: str) -> np.ndarray:
        """Writable numpy view of one oracle array (flat, reference layout)."""
        q = FIELDS.index(name)
        n = self._fn("field_len")(self._h, q)
        ptr = self._fn("field")(self._h, q)
        return np.ctypeslib.as_array(ptr, shape=(n,))

    def set_fields(self, **arrays):
        for k, a in arrays.items():
            dst = self.field(k)
            dst[:] = np.asarray(a, dtype=self.dtype).ravel()

    # single steps (names follow the reference's Solver methods)
    def init_face_vel(self): self._fn("init_face_vel")(self._h)
    def bc_face_vel(self): self._fn("bc_face_vel")(self._h)
    def mom_link_coef(self): self._fn("mom_link_coef")(self._h)
    def mom_src(self): self._fn("mom_src")(self._h)
    def bc_mom(self): self._fn("bc_mom")(self._h)
    def dc_source(self): self._fn("dc_source")(self._h)
    def rhie_chow(self): self._fn("rhie_chow")(self._h)
    def pcorr_link_coef(self): self._fn("pcorr_link_coef")(self._h)
    def pcorr_src(self) -> float: return self._fn("pcorr_src")(self._h)
    def pin_pcorr(self): self._fn("pin_pcorr")(self._h)

    def sweep(self, eq: int, mode: int = GS_REDBLACK) -> float:
        return self._fn("sweep")(self._h, eq, mode)

    def linear_solve(self, eq: int):
        norms = (C.c_double * 4096)()
        n = self._fn("linear_solve")(self._h, eq, norms)
        return n, np.array(norms[:n])

    def update_field(self) -> dict:
        nm = OrcNorms()
        self._fn("update_field")(self._h, C.byref(nm))
        return nm.as_dict()

    def outer_iteration(self) -> dict:
        nm = OrcNorms()
        self._fn("outer_iteration")(self._h, C.byref(nm))
        return nm.as_dict()

    def solve(self, max_outer: int = 0) -> tuple[int, dict]:
        nm = OrcNorms()
        n = self._fn("solve")(self._h, int(max_outer), C.byref(nm))
        return n, nm.as_dict()

    @property
    def iterations(self) -> int:
        return self._fn("iteration_count")(self._h)

    def set_iteration_count(self, it: int):
        """Continue from loaded fields: a count > 0 skips the face
        initialisation of the first outer iteration."""
        self._fn("set_iteration_count")(self._h, it)


def _ptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class AdjointOracle(Oracle):
    """FP64 oracle with the reverse pass of one outer iteration
    (orc_adjoint_apply_d) and the adjoint fixed-point solve built on it."""

    def __init__(self, cfg: dict):
        assert cfg.get("convection_scheme", 0) in (0, "upwind"), "the adjoint linearises upwind convection only"
        super().__init__(cfg, "d")

    def state_sizes(self):
        nx, ny = self.nx, self.ny
        return {"u": nx * ny, "v": nx * ny, "p": nx * ny, "uf": (nx + 1) * ny, "vf": nx * (ny + 1)}

    def apply_transpose(self, seed: dict):
        """G_x^T seed, G_theta^T seed, G_mu^T seed at the current (fixed-point) state."""
        sz = self.state_sizes()
        ins = {k: np.ascontiguousarray(seed[k], dtype=np.float64) for k in sz}
        outs = {k: np.zeros(n) for k, n in sz.items()}
        lth = np.zeros(self.ny)
        lmu = C.c_double()
        rc = lib().orc_adjoint_apply_d(self._h, *[_ptr(ins[k]) for k in ("u", "v", "p", "uf", "vf")],
                                       *[_ptr(outs[k]) for k in ("u", "v", "p", "uf", "vf")], _ptr(lth),
                                       C.byref(lmu))
        assert rc == 0
        return outs, lth, lmu.value

    def objective_seed(self):
        """dJ/dx of J = mean p over the first cell column - mean over the last."""
        nx, ny = self.nx, self.ny
        sz = self.state_sizes()
        seed = {k: np.zeros(n) for k, n in sz.items()}
        p = seed["p"].reshape(ny, nx)
        p[:, 0] = 1.0 / ny
        p[:, -1] = -1.0 / ny
        return seed

    def objective(self) -> float:
        p = self.field("p").reshape(self.ny, self.nx)
        return float(p[:, 0].mean() - p[:, -1].mean())

    def adjoint_gradient(self, max_iter: int = 100000, tol: float = 1e-12):
        """Fixed-point adjoint lambda = G_x^T lambda + dJ/dx; returns
        (dJ/dtheta, dJ/dmu, iterations)."""
        jx = self.objective_seed()
        lam = {k: v.copy() for k, v in jx.items()}
        for it in range(1, max_iter + 1):
            out, lth, lmu = self.apply_transpose(lam)
            new = {k: out[k] + jx[k] for k in lam}
            delta = max(np.abs(new[k] - lam[k]).max() for k in lam)
            scale = max(np.abs(new[k]).max() for k in lam)
            lam = new
            if delta <= tol * scale:
                break
        out, lth, lmu = self.apply_transpose(lam)
        return lth, lmu, it


# ---------------------------------------------------------------- energy
# The reference never solves its temperature; the library's energy equation
# (incompflow-cuda_b200/csrc/ifc_energy.cuh) discretises div(rho u T) =
# div(Gamma grad T), Gamma = k / cp, like the reference's momentum equations
# (include/kernels.cuh:97-134 with Gamma for mu, boundary fold-in of
# :252-334: wall form on Dirichlet faces, zero-gradient form on Neumann
# faces).  These functions restate it in numpy, operation by operation in the
# scalar type, as the checker of the device solve.

def _min0(x):
    return np.where(x < 0, x, x.dtype.type(0))


def energy_assemble(cfg: dict, uf, vf, wf, prec: str = "f"):
    """Coefficient planes (2*dim+1, slot-major as the library's) and source of
    the energy equation on the given face velocities."""
    T = np.float32 if prec == "f" else np.float64
    dim, nx, ny = cfg["dim"], cfg["nx"], cfg["ny"]
    nz = cfg.get("nz", 1) if dim == 3 else 1
    dx = (T(cfg["xmax"]) - T(cfg["xmin"])) / T(nx)
    dy = (T(cfg["ymax"]) - T(cfg["ymin"])) / T(ny)
    dz = (T(cfg["zmax"]) - T(cfg["zmin"])) / T(nz)
    Ax, Ay, Az = dy * dz, dz * dx, dx * dy
    rho = T(cfg["density"])
    gam = T(cfg.get("thermalConductivity", 1.0)) / T(cfg.get("specificHeatCapacity", 1.0))
    Dx, Dy, Dz = gam * Ax / dx, gam * Ay / dy, gam * Az / dz
    uf = np.asarray(uf, T).reshape(nz, ny, nx + 1)
    vf = np.asarray(vf, T).reshape(nz, ny + 1, nx)
    a = {}
    a["E"] = rho * _min0(uf[:, :, 1:]) * Ax - Dx
    a["W"] = rho * _min0(-uf[:, :, :-1]) * Ax - Dx
    a["N"] = rho * _min0(vf[:, 1:, :]) * Ay - Dy
    a["S"] = rho * _min0(-vf[:, :-1, :]) * Ay - Dy
    a["C"] = -(((a["E"] + a["W"]) + a["N"]) + a["S"])
    a["T"] = np.zeros_like(a["C"])
    a["B"] = np.zeros_like(a["C"])
    if dim == 3:
        wf = np.asarray(wf, T).reshape(nz + 1, ny, nx)
        a["T"] = rho * _min0(wf[1:]) * Az - Dz
        a["B"] = rho * _min0(-wf[:-1]) * Az - Dz
        a["C"] = a["C"] + (-(a["T"] + a["B"]))
    b = np.zeros_like(a["C"])
    c83 = T(8) / T(3)
    faces = [(0, "E", "W", (slice(None), slice(None), -1)), (1, "W", "E", (slice(None), slice(None), 0)),
             (2, "N", "S", (slice(None), -1, slice(None))), (3, "S", "N", (slice(None), 0, slice(None)))]
    if dim == 3:
        faces += [(4, "T", "B", (-1, slice(None), slice(None))), (5, "B", "T", (0, slice(None), slice(None)))]
    types = cfg.get("TempBC_type", [1, 1, 0, 0, 1, 1])
    vals = cfg.get("TempBC_val", [0.0, 0.0, 293.0, 373.0, 0.0, 0.0])
    for f, ex, inn, sl in faces:
        e = a[ex][sl].copy()
        if types[f] != 0:
            a["C"][sl] = a["C"][sl] + e
        else:
            a["C"][sl] = a["C"][sl] - T(2) * e
            a[inn][sl] = a[inn][sl] + e / T(3)
            b[sl] = b[sl] - c83 * e * T(vals[f])
        a[ex][sl] = T(0)
    order = ["C", "E", "W", "N", "S"] + (["T", "B"] if dim == 3 else [])
    return np.stack([a[k] for k in order]), b


def energy_sweeps(cfg: dict, coef, src, temp, n: int, prec: str = "f"):
    """n unrelaxed red-black Gauss-Seidel sweeps of the temperature (colour 0
    then colour 1, the library's point update); returns T and the FP64 sum of
    squared changes of each sweep."""
    Tt = np.float32 if prec == "f" else np.float64
    dim = cfg["dim"]
    nx, ny = cfg["nx"], cfg["ny"]
    nz = cfg.get("nz", 1) if dim == 3 else 1
    coef = np.asarray(coef, Tt)
    a = {k: coef[s].reshape(nz, ny, nx) for s, k in enumerate(["C", "E", "W", "N", "S", "T", "B"][: coef.shape[0]])}
    src = np.asarray(src, Tt).reshape(nz, ny, nx)
    t = np.asarray(temp, Tt).reshape(nz, ny, nx).copy()
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    colour = (i + j + k) & 1
    zero = Tt(0)
    sums = []
    for _ in range(n):
        sq = 0.0
        for c in (0, 1):
            pE = np.zeros_like(t); pE[:, :, :-1] = t[:, :, 1:]
            pW = np.zeros_like(t); pW[:, :, 1:] = t[:, :, :-1]
            pN = np.zeros_like(t); pN[:, :-1, :] = t[:, 1:, :]
            pS = np.zeros_like(t); pS[:, 1:, :] = t[:, :-1, :]
            npv = src - a["E"] * pE - a["W"] * pW - a["N"] * pN - a["S"] * pS
            if dim == 3:
                pT = np.zeros_like(t); pT[:-1] = t[1:]
                pB = np.zeros_like(t); pB[1:] = t[:-1]
                npv = npv - (a["T"] * pT + a["B"] * pB)
            npv = npv / a["C"]
            d = Tt(1) * (npv - t)
            new = t + d
            m = colour == c
            t = np.where(m, new, t)
            sq += float(np.sum(np.where(m, d, zero).astype(np.float64) ** 2))
        sums.append(sq)
    return t.ravel(), sums


def _dc_limit(scheme, du, dd, T):
    """Limited face increment L(du, dd) of the deferred-correction schemes
    (central, second-order upwind, QUICK, minmod, van Leer), element-wise in T."""
    s = CONV[scheme] if isinstance(scheme, str) else int(scheme)
    z = T(0)
    if s == 1:
        return dd
    if s == 2:
        return du
    if s == 3:
        return (T(3) * dd + du) / T(4)
    pos = du * dd > z
    with np.errstate(divide="ignore", invalid="ignore"):
        if s == 4:
            return np.where(pos, np.where(np.abs(du) < np.abs(dd), du, dd), z).astype(T)
        if s == 5:
            return np.where(pos, T(2) * du * dd / (du + dd), z).astype(T)
    return np.zeros_like(dd)


def energy_dc(cfg: dict, uf, vf, wf, temp, prec: str = "f"):
    """Deferred-correction source of the temperature (the momentum equations'
    formula, ifc_oracle_impl.h dc_source): per interior face whose far-upwind
    cell is inside the domain Q = (rho u_f A) (0.5 L), per cell
    (Q_w - Q_e) + (Q_s - Q_n) [+ (Q_b - Q_t)], every operation rounded in T."""
    T = np.float32 if prec == "f" else np.float64
    scheme = cfg.get("convection_scheme", 0)
    dim, nx, ny = cfg["dim"], cfg["nx"], cfg["ny"]
    nz = cfg.get("nz", 1) if dim == 3 else 1
    dx = (T(cfg["xmax"]) - T(cfg["xmin"])) / T(nx)
    dy = (T(cfg["ymax"]) - T(cfg["ymin"])) / T(ny)
    dz = (T(cfg["zmax"]) - T(cfg["zmin"])) / T(nz)
    Ax, Ay, Az = dy * dz, dz * dx, dx * dy
    rho = T(cfg["density"])
    t = np.asarray(temp, T).reshape(nz, ny, nx)

    def axis_q(phi, vel, A, n, ax):
        # faces 1..n-1 along axis ax (between cells f-1 and f); Q of each face
        phi = np.moveaxis(phi, ax, -1)
        vel = np.moveaxis(vel, ax, -1)[..., 1:n]
        F = rho * vel * A
        q = np.zeros(F.shape, T)
        for f in range(1, n):
            Fl = F[..., f - 1]
            pl, pr = phi[..., f - 1], phi[..., f]
            pll = phi[..., f - 2] if f >= 2 else np.zeros_like(pl)
            prr = phi[..., f + 1] if f + 1 < n else np.zeros_like(pr)
            fw = (Fl > T(0)) & (f >= 2)
            bw = (Fl < T(0)) & (f + 1 < n)
            U = np.where(Fl > T(0), pl, pr)
            D = np.where(Fl > T(0), pr, pl)
            UU = np.where(Fl > T(0), pll, prr)
            val = Fl * (T(0.5) * _dc_limit(scheme, (U - UU).astype(T), (D - U).astype(T), T))
            q[..., f - 1] = np.where(fw | bw, val, T(0))
        # per cell: Q of the face below minus Q of the face above (0 at the ends)
        lo = np.zeros(phi.shape, T)
        hi = np.zeros(phi.shape, T)
        lo[..., 1:] = q
        hi[..., :-1] = q
        return np.moveaxis(lo, -1, ax), np.moveaxis(hi, -1, ax)

    ufa = np.asarray(uf, T).reshape(nz, ny, nx + 1)
    vfa = np.asarray(vf, T).reshape(nz, ny + 1, nx)
    qw, qe = axis_q(t, ufa, Ax, nx, 2)
    qs, qn = axis_q(t, vfa, Ay, ny, 1)
    dc = (qw - qe) + (qs - qn)
    if dim == 3:
        wfa = np.asarray(wf, T).reshape(nz + 1, ny, nx)
        qb, qt = axis_q(t, wfa, Az, nz, 0)
        dc = dc + (qb - qt)
    return dc.ravel()


def energy_dc_sweeps(cfg: dict, coef, src, uf, vf, wf, temp, n: int, prec: str = "f", cycle: int = 25):
    """n sweeps in cycles of `cycle`, each cycle starting from src + the
    deferred-correction source of the current temperature (the library's
    ifc_solve_energy with a higher-order scheme and no early exit)."""
    T = np.float32 if prec == "f" else np.float64
    t = np.asarray(temp, T).copy()
    src = np.asarray(src, T).ravel()
    done = 0
    while done < n:
        k = min(cycle, n - done)
        eff = (src + energy_dc(cfg, uf, vf, wf, t, prec)).astype(T)
        t, _ = energy_sweeps(cfg, coef, eff, t, k, prec)
        done += k
    return t

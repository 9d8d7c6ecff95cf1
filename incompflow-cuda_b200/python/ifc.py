"""ctypes binding of libifc.so (the C ABI in include/ifc.h).

This is the Python face of the drop-in solver: tests and bench.py drive the
CUDA library through it.  It never falls back to anything: if the built
library is missing, ``load()`` raises.

Configurations are dicts keyed by the reference's config.h names
(include/config.h:6-81): ``dim, nx, ny, nz, xmin..zmax, density,
dynamicViscosity, velBC_type, velBC_val, numOuterIter, nIter_u/v/w/p,
relax_u/v/w/p, tol_u/v/w/p, tol_mass`` plus the additions ``precision``
("f"/"d"), ``linear_solver``, ``criterion``, ``pin_pressure``,
``sweeps_per_pass``, ``log_level``, ``inlet_profile`` and
``convection_scheme`` (a CONV_* value or its name: "upwind", "central",
"sou", "quick", "minmod", "van_leer").
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# IFC_LIB selects another build of the library, e.g. the bounds-checked
# lib/libifc_bc.so (make -C incompflow-cuda_b200 lib_bc).
LIB_PATH = os.environ.get("IFC_LIB") or os.path.join(PKG, "lib", "libifc.so")

OK, NOT_CONVERGED, DIVERGED, TIMEOUT, CUDA_ERROR, BAD_CONFIG, BAD_ARGUMENT, IO_ERROR, UNSUPPORTED = range(9)
EAST, WEST, NORTH, SOUTH, TOP, BOTTOM = range(6)
WALL, INLET, OUTLET = range(3)
GAUSS_SEIDEL, JACOBI = 0, 1
CRIT_REFERENCE, CRIT_PER_FIELD, CRIT_RESIDUAL = 0, 1, 2
CONV_UPWIND, CONV_CENTRAL, CONV_SOU, CONV_QUICK, CONV_MINMOD, CONV_VAN_LEER = range(6)
CONV_NAMES = {"upwind": CONV_UPWIND, "central": CONV_CENTRAL, "sou": CONV_SOU, "quick": CONV_QUICK,
              "minmod": CONV_MINMOD, "van_leer": CONV_VAN_LEER}
FIELDS = ["u", "v", "w", "p", "T", "pc", "uf", "vf", "wf", "ac", "mcoef", "pcoef",
          "src_u", "src_v", "src_w", "src_p"]
STAGES = ["face_bc", "mom_assemble", "mom_solve", "rhie_chow", "pcorr_coef", "pcorr_solve", "update"]


class IfcConfig(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double), ("ymax", C.c_double),
        ("zmin", C.c_double), ("zmax", C.c_double),
        ("thermal_conductivity", C.c_double), ("specific_heat_capacity", C.c_double),
        ("density", C.c_double), ("dynamic_viscosity", C.c_double),
        ("vel_bc_type", C.c_int * 6), ("vel_bc_val", (C.c_double * 3) * 6),
        ("temp_bc_type", C.c_int * 6), ("temp_bc_val", C.c_double * 6),
        ("num_outer_iter", C.c_int),
        ("n_iter_u", C.c_int), ("n_iter_v", C.c_int), ("n_iter_w", C.c_int), ("n_iter_p", C.c_int),
        ("relax_u", C.c_double), ("relax_v", C.c_double), ("relax_w", C.c_double), ("relax_p", C.c_double),
        ("tol_u", C.c_double), ("tol_v", C.c_double), ("tol_w", C.c_double), ("tol_p", C.c_double),
        ("tol_mass", C.c_double),
        ("precision", C.c_int), ("linear_solver", C.c_int), ("criterion", C.c_int),
        ("pin_pressure", C.c_int), ("sweeps_per_pass", C.c_int), ("log_level", C.c_int),
        ("inlet_profile", C.POINTER(C.c_double)), ("stream", C.c_void_p),
        ("convection_scheme", C.c_int), ("slab_axis_cells", C.c_int),
    ]


class IfcStats(C.Structure):
    _fields_ = [
        ("status", C.c_int), ("outer_iterations", C.c_int), ("converged", C.c_int),
        ("sweeps", C.c_int * 4), ("cell_updates", C.c_longlong),
    ] + [(n, C.c_double) for n in (
        "norm_p", "norm_u", "norm_v", "norm_w", "norm_uf", "norm_vf", "norm_wf", "norm_mass",
        "rel_p", "rel_u", "rel_v", "rel_w", "rel_uf", "rel_vf", "rel_wf", "device_ms")] + [
        ("kernel_launches", C.c_longlong)]

    def as_dict(self):
        d = {n: getattr(self, n) for n, _ in self._fields_ if n != "sweeps"}
        d["sweeps"] = list(self.sweeps)
        return d


class IfcBatchResult(C.Structure):
    _fields_ = [("status", C.c_int), ("outer_iterations", C.c_int), ("converged", C.c_int),
                ("sweeps", C.c_int * 4)] + [(n, C.c_double) for n in (
                    "rel_p", "rel_u", "rel_v", "rel_uf", "rel_vf", "norm_mass")] + [
                ("tile_x", C.c_int), ("tile_y", C.c_int), ("sweeps_per_pass", C.c_int)]

    def as_dict(self):
        d = {n: getattr(self, n) for n, _ in self._fields_ if n != "sweeps"}
        d["sweeps"] = list(self.sweeps)
        return d


class IfcAdjointResult(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("converged", C.c_int)] + [
        (n, C.c_double) for n in ("residual", "objective", "dJ_dmu", "device_ms")] + [
        ("kernel_launches", C.c_longlong)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class IfcEnergyResult(C.Structure):
    _fields_ = [("status", C.c_int), ("sweeps", C.c_int), ("converged", C.c_int), ("residual", C.c_double),
                ("device_ms", C.c_double)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


OBJ_PRESSURE_DROP, OBJ_CUSTOM = 0, 1
_DP = C.POINTER(C.c_double)

EXPORTS = {
    "ifc_abi_version": (C.c_int, []),
    "ifc_status_string": (C.c_char_p, [C.c_int]),
    "ifc_config_default": (C.c_int, [C.POINTER(IfcConfig)]),
    "ifc_config_check": (C.c_int, [C.POINTER(IfcConfig)]),
    "ifc_create": (C.c_int, [C.POINTER(IfcConfig), C.POINTER(C.c_void_p)]),
    "ifc_destroy": (C.c_int, [C.c_void_p]),
    "ifc_set_uniform": (C.c_int, [C.c_void_p] + [C.c_double] * 5),
    "ifc_set_field": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]),
    "ifc_get_field": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]),
    "ifc_field_size": (C.c_size_t, [C.c_void_p, C.c_int]),
    "ifc_device_ptr": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "ifc_solve": (C.c_int, [C.c_void_p, C.POINTER(IfcStats)]),
    "ifc_iterate": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(IfcStats)]),
    "ifc_write_vtk": (C.c_int, [C.c_void_p, C.c_char_p]),
    "ifc_write_vtk_host": (C.c_int, [C.POINTER(IfcConfig)] + [C.c_void_p] * 5 + [C.c_char_p]),
    "ifc_write_vtk_binary": (C.c_int, [C.c_void_p, C.c_char_p]),
    "ifc_write_vtk_binary_host": (C.c_int, [C.POINTER(IfcConfig)] + [C.c_void_p] * 5 + [C.c_char_p]),
    "ifc_run_stage": (C.c_int, [C.c_void_p, C.c_int]),
    "ifc_sweep": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double)]),
    "ifc_run_stage_async": (C.c_int, [C.c_void_p, C.c_int]),
    "ifc_sweep_async": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "ifc_sync": (C.c_int, [C.c_void_p]),
    "ifc_get_stats": (C.c_int, [C.c_void_p, C.POINTER(IfcStats)]),
    "ifc_time_stage": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    "ifc_last_error": (C.c_char_p, [C.c_void_p]),
    "ifc_batch_solve": (C.c_int, [C.POINTER(IfcConfig), C.c_int, C.POINTER(IfcBatchResult),
                                  C.POINTER(C.c_void_p), C.POINTER(C.c_double)]),
    "ifc_adjoint": (C.c_int, [C.c_void_p, C.c_int, _DP, _DP, _DP, C.c_int, C.c_double, _DP,
                              C.POINTER(IfcAdjointResult)]),
    "ifc_adjoint_apply": (C.c_int, [C.c_void_p] + [_DP] * 12),
    "ifc_set_inlet_profile": (C.c_int, [C.c_void_p, _DP]),
    "ifc_solve_energy": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.POINTER(IfcEnergyResult)]),
    "ifc_build_flags": (C.c_int, []),
}


def _dptr(a):
    return None if a is None else a.ctypes.data_as(_DP)

_lib = None


def load(path: str = LIB_PATH):
    """Load libifc.so; raises OSError when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise OSError(f"{path} is missing: build it with `make -C incompflow-cuda_b200` "
                          "or __graft_entry__.build()")
        lib = C.CDLL(path)
        for name, (res, args) in EXPORTS.items():
            fn = getattr(lib, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class IfcError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        self.status = status
        s = load().ifc_status_string(status).decode()
        super().__init__(f"{s} ({status}){': ' + msg if msg else ''}")


# ---------------------------------------------------------------- configs

def default_config() -> dict:
    """The reference's shipped include/config.h."""
    return dict(
        dim=2, nx=1024, ny=256, nz=1, xmin=-2.0, xmax=2.0, ymin=-0.5, ymax=0.5, zmin=0.0, zmax=1.0,
        thermalConductivity=1.0, specificHeatCapacity=1.0, density=50.0, dynamicViscosity=1.0,
        velBC_type=[OUTLET, INLET, WALL, WALL, WALL, WALL],
        velBC_val=[[0, 0, 0], [1, 0, 0], [0, 0, 0], [0, 0, 0], [0, 0, 0], [0, 0, 0]],
        TempBC_type=[1, 1, 0, 0, 1, 1], TempBC_val=[0.0, 0.0, 293.0, 373.0, 0.0, 0.0],
        numOuterIter=20000, nIter_u=10, nIter_v=10, nIter_w=10, nIter_p=20,
        relax_u=0.75, relax_v=0.75, relax_w=0.75, relax_p=0.25,
        tol_u=1e-5, tol_v=1e-5, tol_w=1e-5, tol_p=1e-3, tol_mass=1e-9,
    )


def cavity2d(n: int = 64, re: float = 100.0, **kw) -> dict:
    """Lid-driven cavity on the unit square: lid u=1 on the north wall,
    rho=1, mu=1/Re, SIMPLE alpha_u=0.7 alpha_p=0.3, GS 5/5/50, residual 1e-5."""
    c = default_config()
    c.update(dim=2, nx=n, ny=n, nz=1, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, zmin=0.0, zmax=1.0,
             density=1.0, dynamicViscosity=1.0 / re, velBC_type=[WALL] * 6,
             velBC_val=[[0, 0, 0], [0, 0, 0], [1, 0, 0], [0, 0, 0], [0, 0, 0], [0, 0, 0]],
             numOuterIter=20000, nIter_u=5, nIter_v=5, nIter_w=5, nIter_p=50,
             relax_u=0.7, relax_v=0.7, relax_w=0.7, relax_p=0.3,
             tol_u=1e-5, tol_v=1e-5, tol_w=1e-5, tol_p=1e-5, tol_mass=0.0)
    c.update(kw)
    return c


def channel2d(nx: int = 512, ny: int = 128, u_in: float = 0.001, **kw) -> dict:
    """The reference README's default case: water in a 0.125 x 0.025 m channel,
    west inlet, east outlet, no-slip north/south; alpha 0.75/0.25, GS 10/10/20."""
    c = default_config()
    c.update(dim=2, nx=nx, ny=ny, nz=1, xmin=-0.0625, xmax=0.0625, ymin=-0.0125, ymax=0.0125,
             zmin=0.0, zmax=1.0, density=998.2, dynamicViscosity=1.002e-3,
             velBC_type=[OUTLET, INLET, WALL, WALL, WALL, WALL],
             velBC_val=[[0, 0, 0], [u_in, 0, 0], [0, 0, 0], [0, 0, 0], [0, 0, 0], [0, 0, 0]],
             numOuterIter=100000, nIter_u=10, nIter_v=10, nIter_w=10, nIter_p=20,
             relax_u=0.75, relax_v=0.75, relax_w=0.75, relax_p=0.25,
             tol_u=1e-5, tol_v=1e-5, tol_w=1e-5, tol_p=1e-5, tol_mass=0.0)
    c.update(kw)
    return c


def cavity3d(n: int = 128, re: float = 400.0, **kw) -> dict:
    """Lid-driven cube: lid u=1 on the top (z-max) wall, rho=1, mu=1/Re;
    solver settings as the 2D cavity."""
    c = cavity2d(n, re)
    c.update(dim=3, nz=n, velBC_type=[WALL] * 6,
             velBC_val=[[0, 0, 0], [0, 0, 0], [0, 0, 0], [0, 0, 0], [1, 0, 0], [0, 0, 0]])
    c.update(kw)
    return c


def make_struct(cfg: dict) -> tuple[IfcConfig, object]:
    c = IfcConfig()
    load().ifc_config_default(C.byref(c))
    c.dim = int(cfg["dim"])
    c.nx, c.ny = int(cfg["nx"]), int(cfg["ny"])
    c.nz = int(cfg.get("nz", 1)) if c.dim == 3 else 1
    for k in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax"):
        setattr(c, k, float(cfg[k]))
    c.thermal_conductivity = float(cfg.get("thermalConductivity", 1.0))
    c.specific_heat_capacity = float(cfg.get("specificHeatCapacity", 1.0))
    if "TempBC_type" in cfg:
        for f in range(6):
            c.temp_bc_type[f] = int(cfg["TempBC_type"][f])
            c.temp_bc_val[f] = float(cfg["TempBC_val"][f])
    c.density = float(cfg["density"])
    c.dynamic_viscosity = float(cfg["dynamicViscosity"])
    for f in range(6):
        c.vel_bc_type[f] = int(cfg["velBC_type"][f])
        for q in range(3):
            c.vel_bc_val[f][q] = float(cfg["velBC_val"][f][q])
    c.num_outer_iter = int(cfg["numOuterIter"])
    for n in "uvwp":
        setattr(c, f"n_iter_{n}", int(cfg[f"nIter_{n}"]))
        setattr(c, f"relax_{n}", float(cfg[f"relax_{n}"]))
        setattr(c, f"tol_{n}", float(cfg[f"tol_{n}"]))
    c.tol_mass = float(cfg["tol_mass"])
    c.precision = 1 if cfg.get("precision", "f") in ("d", 1, "fp64", "double") else 0
    c.linear_solver = int(cfg.get("linear_solver", GAUSS_SEIDEL))
    c.criterion = int(cfg.get("criterion", CRIT_PER_FIELD))
    c.pin_pressure = int(cfg.get("pin_pressure", -1))
    c.sweeps_per_pass = int(cfg.get("sweeps_per_pass", 0))
    c.log_level = int(cfg.get("log_level", 0))
    conv = cfg.get("convection_scheme", CONV_UPWIND)
    c.convection_scheme = CONV_NAMES[conv] if isinstance(conv, str) else int(conv)
    if cfg.get("stream"):
        c.stream = C.c_void_p(int(cfg["stream"]))
    c.slab_axis_cells = int(cfg.get("slab_axis_cells", 0))
    keep = None
    if cfg.get("inlet_profile") is not None:
        keep = np.ascontiguousarray(cfg["inlet_profile"], dtype=np.float64)
        c.inlet_profile = keep.ctypes.data_as(C.POINTER(C.c_double))
    return c, keep


class Solver:
    """One solver handle (Solver::Solver ... Solver::~Solver of the reference)."""

    def __init__(self, cfg: dict, u=0.0, v=0.0, w=0.0, p=0.0, temp=273.0):
        lib = load()
        self.cfg = dict(cfg)
        self._struct, self._keep = make_struct(cfg)
        h = C.c_void_p()
        rc = lib.ifc_create(C.byref(self._struct), C.byref(h))
        if rc != OK:
            raise IfcError(rc, "ifc_create")
        self._h = h
        self.dtype = np.float64 if self._struct.precision == 1 else np.float32
        self.dim, self.nx, self.ny, self.nz = self._struct.dim, self._struct.nx, self._struct.ny, self._struct.nz
        self.N = self.nx * self.ny * self.nz
        if (u, v, w, p, temp) != (0.0, 0.0, 0.0, 0.0, 273.0):
            self.set_uniform(u, v, w, p, temp)

    def close(self):
        if getattr(self, "_h", None):
            load().ifc_destroy(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc, what, allow=(OK,)):
        if rc not in allow:
            msg = load().ifc_last_error(self._h)
            raise IfcError(rc, f"{what}: {msg.decode() if msg else ''}")
        return rc

    def set_uniform(self, u=0.0, v=0.0, w=0.0, p=0.0, temp=273.0):
        self._check(load().ifc_set_uniform(self._h, u, v, w, p, temp), "set_uniform")

    def field_size(self, name: str) -> int:
        return load().ifc_field_size(self._h, FIELDS.index(name))

    def get(self, name: str) -> np.ndarray:
        n = self.field_size(name)
        out = np.empty(n // np.dtype(self.dtype).itemsize, dtype=self.dtype)
        self._check(load().ifc_get_field(self._h, FIELDS.index(name), out.ctypes.data, n), f"get {name}")
        return out

    def set(self, name: str, arr):
        a = np.ascontiguousarray(arr, dtype=self.dtype).ravel()
        self._check(load().ifc_set_field(self._h, FIELDS.index(name), a.ctypes.data, a.nbytes), f"set {name}")

    def device_ptr(self, name: str) -> int:
        p = C.c_void_p()
        self._check(load().ifc_device_ptr(self._h, FIELDS.index(name), C.byref(p)), "device_ptr")
        return p.value

    def solve(self) -> dict:
        st = IfcStats()
        self._check(load().ifc_solve(self._h, C.byref(st)), "solve", allow=(OK, NOT_CONVERGED))
        return st.as_dict()

    def iterate(self, n: int) -> dict:
        st = IfcStats()
        self._check(load().ifc_iterate(self._h, int(n), C.byref(st)), "iterate")
        return st.as_dict()

    def stage(self, name: str, wait: bool = True):
        """One step of the outer iteration; wait=False enqueues its launches
        on the handle's stream and returns (outcome at the next sync())."""
        fn = load().ifc_run_stage if wait else load().ifc_run_stage_async
        self._check(fn(self._h, STAGES.index(name)), f"stage {name}")

    def sync(self):
        """Wait for the handle's stream; raises on a timed-out wait or an
        out-of-range index left by enqueued launches."""
        self._check(load().ifc_sync(self._h), "sync")

    def sweep(self, eq: int, n: int = 1, norms: bool = True, wait: bool = True) -> np.ndarray | None:
        """n sweeps of equation eq; with norms, sum (d phi)^2 of each sweep
        (the host then waits for every sweep); without, one cooperative
        launch where the handle has one, waited for once, or with wait=False
        only enqueued (outcome at the next sync())."""
        if not norms:
            if wait:
                self._check(load().ifc_sweep(self._h, eq, n, None), "sweep")
            else:
                self._check(load().ifc_sweep_async(self._h, eq, n), "sweep_async")
            return None
        sq = (C.c_double * max(n, 1))()
        self._check(load().ifc_sweep(self._h, eq, n, sq), "sweep")
        return np.array(sq[:n])

    def time_stage(self, name: str, reps: int = 10) -> tuple[float, int]:
        """Average device ms of one launch sequence of a stage, and its kernel count."""
        ms, nl = C.c_double(), C.c_int()
        self._check(load().ifc_time_stage(self._h, STAGES.index(name), reps, C.byref(ms), C.byref(nl)),
                    "time_stage")
        return ms.value, nl.value

    def stats(self) -> dict:
        st = IfcStats()
        self._check(load().ifc_get_stats(self._h, C.byref(st)), "stats")
        return st.as_dict()

    def write_vtk(self, path: str, binary: bool = False):
        """ASCII VTK as the reference writes it, or (binary=True) legacy VTK
        BINARY with the values of the handle's precision."""
        fn = load().ifc_write_vtk_binary if binary else load().ifc_write_vtk
        self._check(fn(self._h, path.encode()), "write_vtk")

    def solve_energy(self, max_sweeps: int = 20000, tol: float = 1e-6) -> dict:
        """Steady temperature on the current flow (ifc_solve_energy)."""
        r = IfcEnergyResult()
        self._check(load().ifc_solve_energy(self._h, int(max_sweeps), float(tol), C.byref(r)), "solve_energy",
                    allow=(OK, NOT_CONVERGED))
        return r.as_dict()

    def set_inlet_profile(self, profile):
        a = np.ascontiguousarray(profile, dtype=np.float64)
        if a.size != self.ny * self.nz:
            raise ValueError(f"inlet profile has {a.size} values, expected {self.ny * self.nz}")
        self._check(load().ifc_set_inlet_profile(self._h, _dptr(a)), "set_inlet_profile")

    def adjoint(self, objective: int = OBJ_PRESSURE_DROP, dJ_du=None, dJ_dv=None, dJ_dp=None,
                max_iter: int = 200000, tol: float = 1e-10) -> tuple[np.ndarray, dict]:
        """Discrete-adjoint gradient at the current state: (dJ/dtheta per inlet
        row, result dict with dJ_dmu, objective, iterations, device_ms)."""
        seeds = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (dJ_du, dJ_dv, dJ_dp)]
        dth = np.zeros(self.ny)
        r = IfcAdjointResult()
        self._check(load().ifc_adjoint(self._h, objective, *[_dptr(a) for a in seeds], int(max_iter), float(tol),
                                       _dptr(dth), C.byref(r)), "adjoint", allow=(OK, NOT_CONVERGED))
        return dth, r.as_dict()

    def adjoint_apply(self, lam: dict) -> tuple[dict, np.ndarray, float]:
        """One reverse pass: (G_x^T lam, G_theta^T lam, G_mu^T lam); lam and the
        result have keys u v p uf vf (FP64)."""
        nx, ny = self.nx, self.ny
        sizes = {"u": nx * ny, "v": nx * ny, "p": nx * ny, "uf": (nx + 1) * ny, "vf": nx * (ny + 1)}
        ins = {k: np.ascontiguousarray(lam[k], dtype=np.float64) for k in sizes}
        for k, n in sizes.items():
            if ins[k].size != n:
                raise ValueError(f"lam[{k}] has {ins[k].size} values, expected {n}")
        outs = {k: np.zeros(n) for k, n in sizes.items()}
        dth = np.zeros(ny)
        dmu = C.c_double()
        keys = ("u", "v", "p", "uf", "vf")
        self._check(load().ifc_adjoint_apply(self._h, *[_dptr(ins[k]) for k in keys],
                                             *[_dptr(outs[k]) for k in keys], _dptr(dth), C.byref(dmu)),
                    "adjoint_apply")
        return outs, dth, dmu.value


def write_vtk_host(cfg: dict, u, v, w, p, temp, path: str, binary: bool = False):
    """The VTK writer on host arrays (no GPU); binary=True writes legacy VTK
    BINARY."""
    s, keep = make_struct(cfg)
    dt = np.float64 if s.precision == 1 else np.float32
    arrs = [np.ascontiguousarray(a, dtype=dt).ravel() for a in (u, v, w, p, temp)]
    fn = load().ifc_write_vtk_binary_host if binary else load().ifc_write_vtk_host
    rc = fn(C.byref(s), *[a.ctypes.data for a in arrs], path.encode())
    if rc != OK:
        raise IfcError(rc, "write_vtk_host")


def batch_solve(cfgs: list, want_fields: bool = True):
    """Solve independent 2D cases in one persistent launch (ifc_batch_solve).
    Returns (results, fields, device_ms): per case a result dict and, when
    want_fields, a dict of u, v, p arrays."""
    n = len(cfgs)
    arr = (IfcConfig * n)()
    keep = []
    for k, c in enumerate(cfgs):
        st, kp = make_struct(c)
        arr[k] = st
        keep.append(kp)
    res = (IfcBatchResult * n)()
    outs = []
    ptrs = (C.c_void_p * n)()
    for k, c in enumerate(cfgs):
        dt = np.float64 if arr[k].precision == 1 else np.float32
        buf = np.empty(3 * c["nx"] * c["ny"], dtype=dt) if want_fields else None
        outs.append(buf)
        ptrs[k] = buf.ctypes.data if want_fields else None
    ms = C.c_double()
    rc = load().ifc_batch_solve(arr, n, res, ptrs, C.byref(ms))
    if rc != OK:
        raise IfcError(rc, "batch_solve")
    fields = []
    for k, c in enumerate(cfgs):
        if want_fields:
            m = c["nx"] * c["ny"]
            fields.append({"u": outs[k][:m], "v": outs[k][m:2 * m], "p": outs[k][2 * m:]})
        else:
            fields.append(None)
    return [r.as_dict() for r in res], fields, ms.value


def batch_cases(n: int = 256, seed: int = 0, sizes=(32, 64, 96, 128, 160, 192, 224, 256)) -> list:
    """The batched workload: n lid-driven cavities on the unit square, nx and ny
    drawn uniformly from `sizes`, Re log-uniform in [10, 1000] (mu = 1/Re,
    rho = 1, lid speed 1), solver settings of the 2D cavity."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nx, ny = int(rng.choice(sizes)), int(rng.choice(sizes))
        re = float(10 ** rng.uniform(1, 3))
        out.append(cavity2d(nx, re=re, ny=ny))
    return out


def case_weight(cfg: dict) -> float:
    """Weight of one batch case for sharding: its cells times cells^0.4, since
    larger cases also take more outer iterations to converge."""
    n = cfg["nx"] * cfg["ny"] * (cfg.get("nz", 1) if cfg["dim"] == 3 else 1)
    return n * n ** 0.4


def shard_cases(weights: list, rank: int, world: int) -> list:
    """Indices of the cases rank `rank` of `world` solves: a greedy
    longest-first split of the case weights (cells x expected iterations) over
    the ranks, identical on every rank, no communication needed."""
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    load_ = [0.0] * world
    mine = []
    for i in order:
        r = min(range(world), key=lambda q: (load_[q], q))
        load_[r] += weights[i]
        if r == rank:
            mine.append(i)
    return sorted(mine)

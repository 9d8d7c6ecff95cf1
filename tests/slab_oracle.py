"""The CPU oracle as one slab of ifc_slabs.SlabSolver (test infrastructure).

Each step calls the oracle functions that the device's ifc_run_stage step
matches bit for bit (tests/test_gpu_parity_steps.py), so a decomposition of
oracle slabs can be checked against the undecomposed oracle on the CPU, with
the same orchestration and halo exchange code the device slabs use.
"""
import numpy as np
import torch

import oracle as O
from helpers import assert_bitwise, to_oracle_cfg


class OracleSlab:
    def __init__(self, cfg: dict, precision: str = "f"):
        self.o = O.Oracle(to_oracle_cfg(cfg), precision)
        self.dim = cfg["dim"]
        self.N = len(self.o.field("u"))
        self.first = True
        self._views = {}

    def _assemble(self):
        o = self.o
        o.mom_link_coef()
        o.mom_src()
        o.bc_mom()
        o.dc_source()

    def stage(self, name: str):
        o = self.o
        if name == "face_bc":
            if self.first:
                o.init_face_vel()
            o.bc_face_vel()
        elif name == "mom_assemble":
            self._assemble()
        elif name == "mom_solve":
            self._assemble()
            for eq in range(self.dim):
                o.linear_solve(eq)
        elif name == "rhie_chow":
            o.rhie_chow()
            o.bc_face_vel()
            o.pcorr_src()
        elif name == "pcorr_coef":
            o.pcorr_link_coef()
        elif name == "pcorr_solve":
            o.pcorr_link_coef()
            o.field("pc")[:] = 0
            o.linear_solve(O.EQ_P)
        elif name == "update":
            o.update_field()
            o.bc_face_vel()
        else:
            raise ValueError(name)
        self.first = False

    def sweep(self, eq: int, n: int):
        mode = self.o.cfg["sweep_mode"]  # red-black Gauss-Seidel or Jacobi, as the config says
        for _ in range(n):
            self.o.sweep(eq, mode)

    def view(self, name: str) -> torch.Tensor:
        v = self._views.get(name)
        if v is None:
            if name == "ac":
                a = self.o.field("mcoef")[: self.N]
            elif name == "T":  # the oracle has no temperature: the handles' initial 273 K
                a = np.full(self.N, 273.0, dtype=self.o.field("u").dtype)
            else:
                a = self.o.field(name)
            v = torch.from_numpy(a)
            self._views[name] = v
        return v

    def sync(self):
        pass

    def zero(self, name: str):
        self.view(name).zero_()

    def close(self):
        self._views.clear()


def undecomposed(cfg: dict, iterations: int, precision: str = "f") -> O.Oracle:
    """The oracle's own outer iterations on the whole grid, every inner sweep
    run, no pinning (the slab solve's settings)."""
    c = dict(cfg, tol_u=0.0, tol_v=0.0, tol_w=0.0, tol_p=0.0, tol_mass=0.0, pin_pressure=0)
    o = O.Oracle(to_oracle_cfg(c), precision)
    for _ in range(iterations):
        o.outer_iteration()
    o.bc_face_vel()  # the device's update step writes the next iteration's boundary faces
    return o


def state_names(dim: int) -> list:
    return ["u", "v", "p", "uf", "vf"] + (["w", "wf"] if dim == 3 else [])


def assert_equal_fields(a: dict, b: dict, what: str):
    for k in a:
        assert_bitwise(np.asarray(a[k]), np.asarray(b[k]), f"{what} {k}")

"""The energy equation's restatement (oracle.energy_*) on its own, no GPU:
pure conduction between a hot south wall and a cold north wall with
adiabatic east/west walls and no flow has the linear profile as its exact
discrete solution (the boundary fold-in extrapolates quadratically through
the wall value, which a linear profile satisfies)."""
import numpy as np

import ifc
import oracle as O


def test_conduction_between_walls_is_linear():
    cfg = ifc.cavity2d(12, ny=10)  # TempBCs: E/W Neumann, N 293 K, S 373 K (the reference's config.h)
    nx, ny = cfg["nx"], cfg["ny"]
    uf = np.zeros((nx + 1) * ny)
    vf = np.zeros(nx * (ny + 1))
    coef, src = O.energy_assemble(cfg, uf, vf, None, "d")
    t, sums = O.energy_sweeps(cfg, coef, src, np.full(nx * ny, 273.0), 4000, "d")
    y = (np.arange(ny) + 0.5) / ny  # unit square
    expect = 373.0 - 80.0 * y
    assert np.abs(t.reshape(ny, nx) - expect[:, None]).max() < 1e-8
    assert sums[-1] < 1e-20 * sums[0]


def test_assembly_identities():
    cfg = ifc.channel2d(20, 8)
    rng = np.random.default_rng(0)
    nx, ny = 20, 8
    uf = rng.uniform(-1e-3, 2e-3, (nx + 1) * ny)
    vf = rng.uniform(-1e-3, 1e-3, nx * (ny + 1))
    coef, src = O.energy_assemble(cfg, uf, vf, None, "d")
    c = coef.reshape(5, ny, nx)
    # interior cells: aC = -sum of links, links <= 0, no source
    inner = (slice(1, -1), slice(1, -1))
    assert np.allclose(c[0][inner], -c[1:, 1:-1, 1:-1].sum(0), rtol=1e-13)
    assert (c[1:][(slice(None),) + inner] <= 0).all()
    assert np.all(src.reshape(ny, nx)[inner] == 0)
    # boundary links are folded away
    assert np.all(c[1][:, -1] == 0) and np.all(c[2][:, 0] == 0)
    assert np.all(c[3][-1, :] == 0) and np.all(c[4][0, :] == 0)

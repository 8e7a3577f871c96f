"""Wall distance on the device (cfd2d_sim_wall_distance) against the oracle (GPU).

The oracle restates cfd2d/turbulence.py:43-70, which takes scipy's exact Euclidean
distance transform of the wall cells. The device transform is separable and forms
the squared distance of the nearest wall cell from integer offsets in scipy's
order, so the fields must be equal bit for bit: no-slip boxes, inflow/outflow
channels with obstacles, periodic channels (with and without walls), unequal
spacings and seeded random scatters of solid cells (many equidistant walls).
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu]


def _sim(nx, ny, lx, ly, sides, mask=None):
    from cfd2d_b200.boundary import BoundaryCondition as BC
    from cfd2d_b200.grid import Grid
    from cfd2d_b200.solver import Simulation

    grid = Grid(nx, ny, lx, ly)
    if mask is not None:
        grid.add_obstacle(mask)
    kinds = dict(zip(("left", "right", "bottom", "top"), sides))
    bcs = {}
    for side, kind in kinds.items():
        if kind == "inflow":
            bcs[side] = BC("inflow", velocity=1.0)
        elif kind == "noslip" and side == "top":
            bcs[side] = BC("noslip", velocity=1.0)
        else:
            bcs[side] = BC(kind)
    return Simulation(grid, bcs, nu=0.01, pressure_solver="cg")


def _circle(nx, ny, lx, ly, xc, yc, r):
    x = (np.arange(nx) + 0.5) * lx / nx
    y = (np.arange(ny) + 0.5) * ly / ny
    X, Y = np.meshgrid(x, y, indexing="ij")
    return (X - xc) ** 2 + (Y - yc) ** 2 <= r * r


def _check(sim):
    import oracle as O
    from cfd2d_b200 import turbulence

    got = turbulence.wall_distance(sim)
    want = O.wall_distance(sim)
    assert got.shape == want.shape
    bad = np.argwhere(got != want)
    assert bad.size == 0, (len(bad), bad[:5].tolist(), got[tuple(bad[0])], want[tuple(bad[0])])
    return got


CASES = {
    "cavity32": (32, 32, 1.0, 1.0, ("noslip",) * 4, None),
    "cylinder440x82": (440, 82, 2.2, 0.41, ("inflow", "outflow", "noslip", "noslip"),
                       ("circle", 0.2, 0.2, 0.05)),
    "sst_channel_128x192": (128, 192, 2 * np.pi, 2.0, ("periodic", "periodic", "noslip", "noslip"), None),
    "periodic_cylinder": (64, 48, 1.0, 0.75, ("periodic", "periodic", "noslip", "slip"), ("circle", 0.3, 0.4, 0.12)),
    "slip_box_obstacle": (200, 90, 2.0, 1.0, ("inflow", "outflow", "slip", "slip"), ("circle", 0.7, 0.5, 0.1)),
    "obstacles1024x512": (1024, 512, 2.0, 1.0, ("inflow", "outflow", "slip", "slip"), ("circle", 0.5, 0.45, 0.06)),
}


@pytest.mark.parametrize("name", list(CASES))
def test_wall_distance_matches_oracle(cuda_lib, name):
    nx, ny, lx, ly, sides, shape = CASES[name]
    mask = _circle(nx, ny, lx, ly, *shape[1:]) if shape else None
    d = _check(_sim(nx, ny, lx, ly, sides, mask))
    assert d.max() < 1e6


def test_wall_distance_without_walls_is_1e6(cuda_lib):
    d = _check(_sim(40, 20, 2.0, 1.0, ("periodic", "periodic", "slip", "slip")))
    assert (d == 1e6).all()


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_wall_distance_random_solids(cuda_lib, seed):
    rng = np.random.default_rng(seed)
    nx, ny = int(rng.integers(40, 200)), int(rng.integers(40, 200))
    lx, ly = float(rng.uniform(0.5, 3.0)), float(rng.uniform(0.5, 3.0))
    mask = rng.random((nx, ny)) < 0.01
    sides = [("noslip", "noslip", "noslip", "noslip"), ("inflow", "outflow", "slip", "noslip"),
             ("periodic", "periodic", "slip", "slip")][seed]
    _check(_sim(nx, ny, lx, ly, sides, mask))

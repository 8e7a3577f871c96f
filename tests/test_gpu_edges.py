"""Tile edges, tiny and odd grids, and repeatability (GPU).

The smallest grid the reference accepts (4 x 4, cfd2d/grid.py:30-31) and odd sizes
that leave partial 32 x 8 tiles, partial cell pairs and partial cluster slabs, run
against the oracle for 20 steps; a run repeated on the device is bit-identical.
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle as O

pytestmark = [pytest.mark.gpu, pytest.mark.filterwarnings("ignore::RuntimeWarning")]


def rel(a, b):
    s = np.abs(b).max()
    return np.abs(a - b).max() / s if s > 0 else np.abs(a - b).max()


def _pair(nx, ny, periodic):
    from cfd2d_b200 import geometry
    from cfd2d_b200.boundary import BoundaryCondition as BC
    from cfd2d_b200.grid import Grid
    from cfd2d_b200.solver import Simulation

    lx, ly = 1.0, ny / nx
    g, og = Grid(nx, ny, lx, ly), O.OGrid(nx, ny, lx, ly)
    if periodic:
        sides = dict(left="periodic", right="periodic", bottom="noslip", top="slip")
        g.add_obstacle(geometry.circle(g, 0.5, 0.5 * ly, 0.2 * ly))
        og.add_obstacle(O.circle_mask(og, 0.5, 0.5 * ly, 0.2 * ly))
        kw = dict(nu=0.05, flow_rate=1.0)
    else:
        sides = dict(left="noslip", right="noslip", bottom="noslip", top="noslip")
        kw = dict(nu=0.05)
    bcs = {s: BC(k, velocity=1.0 if s == "top" and not periodic else 0.0) for s, k in sides.items()}
    obcs = {s: O.OBC(k, velocity=1.0 if s == "top" and not periodic else 0.0) for s, k in sides.items()}
    sim = Simulation(g, bcs, pressure_solver="cg", **kw)
    sim.pressure.tol = 1e-10
    osim = O.OSimulation(og, obcs, pressure_solver="cg", tol=1e-10, **kw)
    return sim, osim


@pytest.mark.parametrize("nx,ny,periodic", [(4, 4, False), (5, 7, False), (33, 17, False), (7, 33, False),
                                            (33, 17, True), (40, 9, True)])
def test_small_and_odd_grids_match_the_oracle(cuda_lib, nx, ny, periodic):
    sim, osim = _pair(nx, ny, periodic)
    for _ in range(20):
        sim.step()
        osim.step()
    for f in "uvp":
        assert rel(getattr(sim, f), getattr(osim, f)) < 1e-9, (f, nx, ny, periodic)


def test_repeated_run_is_bit_identical(cuda_lib):
    from cfd2d_b200 import cases

    runs = []
    for _ in range(2):
        case = cases.build_case({"fall": "cylinder", "parameter": {"re": 100, "nx": 110, "ny": 21},
                                 "numerik": {"pressure_solver": "cg"},
                                 "skalar": {"name": "c", "diffusivity": 1e-3, "inflow_band": [0.15, 0.25]}})
        case.sim.pressure.tol = 1e-8
        case.sim.advance(30)
        runs.append((case.sim.u.copy(), case.sim.p.copy(), case.sim.scalars["c"].phi.copy(),
                     list(case.sim.history.fx)))
    for a, b in zip(*runs):
        assert np.array_equal(np.asarray(a), np.asarray(b))

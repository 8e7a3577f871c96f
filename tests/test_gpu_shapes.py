"""Polygon, NACA and image obstacles on the device (GPU).

Masks bit-identical to the oracle's crossings test (cell centres on an edge
included) and to the reference's image masks; the reference's own obstacle test with
a NACA 2412 at 10 degrees (tests/test_cfd2d.py:29-41) on the device, and that case
against the oracle step by step.
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from conftest import golden

pytestmark = [pytest.mark.gpu, pytest.mark.filterwarnings("ignore::RuntimeWarning")]


def _polygons(rng):
    polys = []
    for n in (3, 6, 11, 40):
        ang = np.sort(rng.uniform(0, 2 * np.pi, n))
        r = rng.uniform(0.1, 0.4, n)
        polys.append(np.column_stack([0.55 + r * np.cos(ang), 0.45 + r * np.sin(ang)]))
    polys.append(rng.uniform(0.05, 0.95, (9, 2)))  # self-intersecting
    # vertices on cell centres and edges through them (ties of the crossings test)
    c = (np.arange(64) + 0.5) / 64
    polys.append(np.array([[c[10], c[12]], [c[40], c[12]], [c[40], c[30]], [c[25], c[50]], [c[10], c[30]]]))
    polys.append(np.array([[c[5], c[5]], [c[20], c[20]], [c[35], c[5]], [c[35], c[35]], [c[5], c[35]]]))
    return polys


def test_polygon_masks_bitwise(cuda_lib):
    from cfd2d_b200 import geometry
    from cfd2d_b200.grid import Grid

    rng = np.random.default_rng(17)
    for nx, ny in ((64, 64), (97, 53), (300, 200)):
        g, og = Grid(nx, ny, 1.0, 1.0), O.OGrid(nx, ny, 1.0, 1.0)
        for P in _polygons(rng):
            assert np.array_equal(geometry.polygon(g, P), O.polygon_mask(og, P)), (nx, ny, len(P))


@pytest.mark.parametrize("code,angle", [("0012", 0.0), ("2412", 10.0), ("4415", -7.5), ("6409", 23.0)])
def test_naca_masks_bitwise(cuda_lib, code, angle):
    from cfd2d_b200 import geometry
    from cfd2d_b200.grid import Grid

    for nx, ny, lx, ly in ((200, 100, 2.0, 1.0), (80, 20, 4.0, 1.0), (513, 257, 3.0, 1.5)):
        g, og = Grid(nx, ny, lx, ly), O.OGrid(nx, ny, lx, ly)
        m = geometry.naca4(g, code, 0.4 * lx / 2, 0.5 * ly, 0.6 * lx / 2, angle)
        assert m.any()
        assert np.array_equal(m, O.naca4_mask(og, code, 0.4 * lx / 2, 0.5 * ly, 0.6 * lx / 2, angle))


def test_reference_naca_area(cuda_lib):
    from cfd2d_b200 import geometry
    from cfd2d_b200.grid import Grid

    g = Grid(200, 100, 2.0, 1.0)
    m = geometry.naca4(g, "0012", 0.5, 0.5, 1.0, 0.0)
    assert m.sum() * g.dx * g.dy == pytest.approx(0.0822, rel=0.05)


def test_image_masks_bitwise(cuda_lib, tmp_path):
    from PIL import Image

    from cfd2d_b200 import geometry
    from cfd2d_b200.grid import Grid

    g = golden("golden_shapes")
    for k in range(int(g["n_img"])):
        name = str(g[f"img{k}_name"])
        path = tmp_path / f"{name}_{k}.png"
        Image.fromarray(g[f"pixels_{name}"]).save(path)
        kw = {}
        for item in g[f"img{k}_kw"]:
            a, b = str(item).split("=")
            kw[a] = b == "True" if b in ("True", "False") else float(b)
        nx, ny, lx, ly = g[f"img{k}_grid"]
        m = geometry.from_image(Grid(int(nx), int(ny), lx, ly), path, **kw)
        assert np.array_equal(m, g[f"img{k}_mask"]), k


def test_reference_obstacles_with_naca(cuda_lib):
    """tests/test_cfd2d.py:29-41: a cylinder and a NACA 2412 at 10 degrees in a
    channel with outflow stay divergence-free and conserve mass over 100 steps."""
    from cfd2d_b200 import cases

    obst = [{"typ": "kreis", "x": 1.0, "y": 0.5, "r": 0.15},
            {"typ": "naca", "code": "2412", "x": 2.0, "y": 0.4, "sehne": 0.6, "winkel": 10}]
    case = cases.custom_obstacles(obst, lx=4, ly=1, nx=80, ny=20, re=100)
    for _ in range(100):
        case.sim.step()
    assert case.sim.max_divergence() < 1e-10
    g = case.sim.grid
    u = case.sim.u
    q_in = u[0, 1:-1].sum() * g.dy
    q_out = u[g.nx, 1:-1].sum() * g.dy
    assert q_out == pytest.approx(q_in, rel=1e-8)


def test_naca_case_matches_the_oracle(cuda_lib):
    from cfd2d_b200 import cases

    obst = [{"typ": "naca", "code": "2412", "x": 1.0, "y": 0.45, "sehne": 1.2, "winkel": 8},
            {"typ": "polygon", "punkte": [(2.6, 0.2), (3.0, 0.35), (2.7, 0.7)]}]
    case = cases.custom_obstacles(obst, lx=4, ly=1, nx=160, ny=40, re=200, pressure_solver="cg")
    case.sim.pressure.tol = 1e-10
    osim = O.custom_obstacles(obst, lx=4, ly=1, nx=160, ny=40, re=200, pressure_solver="cg", tol=1e-10)
    assert np.array_equal(case.sim.grid.fluid, osim.grid.fluid)
    for _ in range(30):
        case.sim.step()
        osim.step()
    for f in "uvp":
        a, b = getattr(case.sim, f), getattr(osim, f)
        assert np.abs(a - b).max() / np.abs(b).max() < 1e-9, f

"""Host side of the polygon and NACA obstacles (CPU): the package's NACA outline is
the reference's bit for bit, and bad shape descriptions are refused as the
reference refuses them (cfd2d/geometry.py:43-102)."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden


def test_naca_outline_bitwise():
    from cfd2d_b200 import geometry

    g = golden("golden_shapes")
    for k in range(int(g["n_naca"])):
        code, chord, n, closed = g[f"naca{k}_spec"]
        pts = geometry.naca4_coordinates(str(code), float(chord), int(n), bool(int(closed)))
        assert np.array_equal(pts, g[f"naca{k}_pts"]), k


def test_bad_shapes_raise():
    from cfd2d_b200 import geometry
    from cfd2d_b200.grid import Grid

    g = Grid(8, 8, 1.0, 1.0)
    with pytest.raises(ValueError):
        geometry.naca4_coordinates("12")
    with pytest.raises(ValueError):
        geometry.naca4_coordinates("2400")
    with pytest.raises(ValueError):
        geometry.polygon(g, [(0.1, 0.1), (0.5, 0.5)])
    with pytest.raises(FileNotFoundError):
        geometry.from_image(g, "/nonexistent/obstacle.png")
    with pytest.raises(ValueError):
        geometry.build_obstacle(g, {"typ": "stern"})
    assert geometry.describe_obstacle({"typ": "polygon", "punkte": [(0, 0), (1, 0), (0, 1)]}) == \
        "Polygon mit 3 Punkten"

"""Obstacle masks, voxelised on the GPU (cell centres inside the shape).

Drop-in for cfd2d/geometry.py: every function returns a host bool array of shape
(nx, ny), True where the cell centre lies in the solid. The three analytic shapes
are computed by the CUDA kernels behind ``cfd2d_mask_*`` with the reference's
float64 expressions (no fused multiply-add), so the masks are bit-identical.
Polygon, NACA and image obstacles are not part of this path.
"""

from __future__ import annotations

import numpy as np

from . import _lib
from .grid import Grid


def _run_mask(grid: Grid, fn, *args) -> np.ndarray:
    t = _lib.torch()
    out = t.empty((grid.nx, grid.ny), dtype=t.uint8, device=_lib.device())
    L = _lib.lib()
    rc = getattr(L, fn)(grid.nx, grid.ny, grid.dx, grid.dy, *[float(a) for a in args],
                        _lib.ptr(out), _lib.stream_ptr())
    _lib.check(rc, fn)
    return out.cpu().numpy().astype(bool)


def circle(grid: Grid, xc: float, yc: float, radius: float) -> np.ndarray:
    """Circle (cfd2d/geometry.py:17-22)."""
    if radius <= 0:
        raise ValueError("Radius muss positiv sein.")
    return _run_mask(grid, "cfd2d_mask_circle", xc, yc, radius)


def ellipse(grid: Grid, xc: float, yc: float, a: float, b: float, angle_deg: float = 0.0) -> np.ndarray:
    """Ellipse with half axes a (x), b (y), rotated by angle_deg (cfd2d/geometry.py:25-32).

    cos and sin of the angle are evaluated with numpy, exactly as the reference does,
    and passed to the kernel.
    """
    phi = np.deg2rad(angle_deg)
    return _run_mask(grid, "cfd2d_mask_ellipse", xc, yc, a, b, float(np.cos(phi)), float(np.sin(phi)))


def rectangle(grid: Grid, x0: float, y0: float, x1: float, y1: float) -> np.ndarray:
    """Axis-parallel rectangle with corners (x0, y0), (x1, y1) (cfd2d/geometry.py:35-40)."""
    xa, xb = sorted((x0, x1))
    ya, yb = sorted((y0, y1))
    return _run_mask(grid, "cfd2d_mask_rectangle", xa, ya, xb, yb)


def build_obstacle(grid: Grid, spec: dict) -> np.ndarray:
    """Mask from a description dict (cfd2d/geometry.py:166-195): kreis, ellipse, rechteck."""
    typ = spec.get("typ", "").lower()
    if typ == "kreis":
        return circle(grid, spec["x"], spec["y"], spec["r"])
    if typ == "ellipse":
        return ellipse(grid, spec["x"], spec["y"], spec["a"], spec["b"], spec.get("winkel", 0.0))
    if typ == "rechteck":
        return rectangle(grid, spec["x0"], spec["y0"], spec["x1"], spec["y1"])
    if typ in ("naca", "polygon", "bild"):
        raise NotImplementedError(f"Hindernistyp {typ!r} ist nicht Teil des B200-Pfads "
                                  "(nur kreis, ellipse, rechteck)")
    raise ValueError(f"Unbekannter Hindernistyp: {typ!r}")


def describe_obstacle(spec: dict) -> str:
    typ = spec.get("typ", "?")
    if typ == "kreis":
        return f"Kreis: Mittelpunkt ({spec['x']}, {spec['y']}), r={spec['r']}"
    if typ == "ellipse":
        return (f"Ellipse: Mittelpunkt ({spec['x']}, {spec['y']}), a={spec['a']}, b={spec['b']}, "
                f"Winkel={spec.get('winkel', 0)}°")
    if typ == "rechteck":
        return f"Rechteck: ({spec['x0']}, {spec['y0']}) bis ({spec['x1']}, {spec['y1']})"
    return str(spec)

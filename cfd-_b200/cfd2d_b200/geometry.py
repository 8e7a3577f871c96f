"""Obstacle masks, voxelised on the GPU (cell centres inside the shape).

Drop-in for cfd2d/geometry.py: every function returns a host bool array of shape
(nx, ny), True where the cell centre lies in the solid. Every mask is computed
by a CUDA kernel behind ``cfd2d_mask_*`` with the reference's float64 expressions
(no fused multiply-add): the analytic shapes directly, polygons and NACA profiles by
the crossing test over their outline, images by the pixel under each cell centre
(the file is decoded and thresholded on the host).
"""

from __future__ import annotations

from pathlib import Path

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


def polygon(grid: Grid, points) -> np.ndarray:
    """Closed polygon through the (x, y) points (cfd2d/geometry.py:43-51).

    The reference asks matplotlib's ``Path.contains_points``; the kernel runs the same
    crossings test (E. Haines, Graphics Gems IV, 1994) with the same comparisons, so
    cell centres on an edge fall on the same side."""
    pts = np.asarray(points, dtype=float)
    if pts.ndim != 2 or pts.shape[1] != 2 or len(pts) < 3:
        raise ValueError("Ein Polygon braucht mindestens 3 Punkte (x, y).")
    t = _lib.torch()
    px = _lib.to_dev(np.ascontiguousarray(pts[:, 0]), t.float64)
    py = _lib.to_dev(np.ascontiguousarray(pts[:, 1]), t.float64)
    out = t.empty((grid.nx, grid.ny), dtype=t.uint8, device=_lib.device())
    rc = _lib.lib().cfd2d_mask_polygon(grid.nx, grid.ny, grid.dx, grid.dy, _lib.ptr(px), _lib.ptr(py), len(pts),
                                       _lib.ptr(out), _lib.stream_ptr())
    _lib.check(rc, "cfd2d_mask_polygon")
    return out.cpu().numpy().astype(bool)


def naca4_coordinates(code: str, chord: float = 1.0, n: int = 200, closed_te: bool = True) -> np.ndarray:
    """Outline of a NACA 4-digit section, leading edge at the origin (cfd2d/geometry.py:54-102).

    The published section formulas (Abbott and von Doenhoff): thickness
    5 t (0.2969 sqrt(x) - 0.1260 x - 0.3516 x^2 + 0.2843 x^3 + a4 x^4) with a4 = -0.1036
    (closed trailing edge) or -0.1015, laid off normal to the two-arc camber line;
    n cosine-spaced stations per side, from the trailing edge over the upper side to
    the nose and back along the lower side. A few hundred points, set up on the host."""
    code = str(code).strip()
    if len(code) != 4 or not code.isdigit():
        raise ValueError("NACA-Code muss aus genau 4 Ziffern bestehen, z. B. '0012'.")
    m, p, t = int(code[0]) / 100.0, int(code[1]) / 10.0, int(code[2:]) / 100.0
    if t <= 0:
        raise ValueError("Die Profildicke muss größer als 0 sein.")
    x = 0.5 * (1.0 - np.cos(np.linspace(0.0, np.pi, n)))
    a4 = -0.1036 if closed_te else -0.1015
    half = 5 * t * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x**2 + 0.2843 * x**3 + a4 * x**4)
    camber, slope = np.zeros_like(x), np.zeros_like(x)
    if m > 0 and p > 0:
        ahead = x < p
        aft = ~ahead
        camber[ahead] = m / p**2 * (2 * p * x[ahead] - x[ahead] ** 2)
        slope[ahead] = 2 * m / p**2 * (p - x[ahead])
        camber[aft] = m / (1 - p) ** 2 * ((1 - 2 * p) + 2 * p * x[aft] - x[aft] ** 2)
        slope[aft] = 2 * m / (1 - p) ** 2 * (p - x[aft])
    th = np.arctan(slope)
    upper = (x - half * np.sin(th), camber + half * np.cos(th))
    lower = (x + half * np.sin(th), camber - half * np.cos(th))
    xs = np.concatenate([upper[0][::-1], lower[0][1:]]) * chord
    ys = np.concatenate([upper[1][::-1], lower[1][1:]]) * chord
    return np.column_stack([xs, ys])


def naca4(grid: Grid, code: str, x_le: float, y_le: float, chord: float,
          angle_of_attack_deg: float = 0.0) -> np.ndarray:
    """NACA 4-digit profile with its leading edge at (x_le, y_le); a positive angle of
    attack raises the nose (clockwise about the leading edge) (cfd2d/geometry.py:105-116)."""
    pts = naca4_coordinates(code, chord)
    a = np.deg2rad(angle_of_attack_deg)
    xr = pts[:, 0] * np.cos(a) + pts[:, 1] * np.sin(a)
    yr = -pts[:, 0] * np.sin(a) + pts[:, 1] * np.cos(a)
    return polygon(grid, np.column_stack([xr + x_le, yr + y_le]))


def _solid_pixels(path: Path, threshold: float, invert: bool) -> np.ndarray:
    """Decode and threshold an image file (cfd2d/geometry.py:136-149): dark pixels are
    solid; with an alpha channel the opaque ones (the dark opaque ones where every
    pixel is opaque)."""
    from PIL import Image

    img = Image.open(path)
    if img.mode in ("RGBA", "LA") or (img.mode == "P" and "transparency" in img.info):
        rgba = np.asarray(img.convert("RGBA"), dtype=float) / 255.0
        grey, alpha = rgba[..., :3].mean(axis=2), rgba[..., 3]
        solid = (alpha > 0.5) & (grey < threshold) if alpha.min() > 0.5 else alpha > 0.5
    else:
        solid = np.asarray(img.convert("L"), dtype=float) / 255.0 < threshold
    return ~solid if invert else solid


def from_image(grid: Grid, path, x0: float = 0.0, y0: float = 0.0, width: float | None = None,
               height: float | None = None, threshold: float = 0.5, invert: bool = False) -> np.ndarray:
    """Obstacle from an image file laid on [x0, x0 + width] x [y0, y0 + height]
    (cfd2d/geometry.py:119-163): the whole domain without width, the aspect ratio kept
    without height. Each cell centre takes the pixel under it on the device."""
    path = Path(path)
    if not path.exists():
        raise FileNotFoundError(f"Bilddatei nicht gefunden: {path}")
    solid = np.ascontiguousarray(_solid_pixels(path, threshold, invert), dtype=np.uint8)
    h, w = solid.shape
    if width is None:
        x0, y0, width, height = 0.0, 0.0, grid.lx, grid.ly
    if height is None:
        height = width * h / w
    t = _lib.torch()
    sd = _lib.to_dev(solid)
    out = t.empty((grid.nx, grid.ny), dtype=t.uint8, device=_lib.device())
    rc = _lib.lib().cfd2d_mask_image(grid.nx, grid.ny, grid.dx, grid.dy, _lib.ptr(sd), h, w, float(x0), float(y0),
                                     float(width), float(height), _lib.ptr(out), _lib.stream_ptr())
    _lib.check(rc, "cfd2d_mask_image")
    return out.cpu().numpy().astype(bool)


def build_obstacle(grid: Grid, spec: dict) -> np.ndarray:
    """Mask from a description dict (cfd2d/geometry.py:166-195): kreis, ellipse,
    rechteck, naca, polygon, bild."""
    typ = spec.get("typ", "").lower()
    if typ == "kreis":
        return circle(grid, spec["x"], spec["y"], spec["r"])
    if typ == "ellipse":
        return ellipse(grid, spec["x"], spec["y"], spec["a"], spec["b"], spec.get("winkel", 0.0))
    if typ == "rechteck":
        return rectangle(grid, spec["x0"], spec["y0"], spec["x1"], spec["y1"])
    if typ == "naca":
        return naca4(grid, spec.get("code", "0012"), spec["x"], spec["y"], spec["sehne"], spec.get("winkel", 0.0))
    if typ == "polygon":
        return polygon(grid, spec["punkte"])
    if typ == "bild":
        return from_image(grid, spec["pfad"], spec.get("x", 0.0), spec.get("y", 0.0), spec.get("breite"),
                          spec.get("hoehe"), spec.get("schwelle", 0.5), spec.get("invertieren", False))
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
    if typ == "naca":
        return (f"NACA {spec.get('code', '0012')}: Vorderkante ({spec['x']}, {spec['y']}), "
                f"Sehne={spec['sehne']}, Anstellwinkel={spec.get('winkel', 0)}°")
    if typ == "polygon":
        return f"Polygon mit {len(spec['punkte'])} Punkten"
    if typ == "bild":
        return f"Bild: {spec['pfad']}"
    return str(spec)

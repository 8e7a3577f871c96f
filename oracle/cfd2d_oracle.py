"""NumPy restatement of cfd2d's projection step (oracle; test infrastructure only).

Every function names the reference file:line it restates. The arithmetic is kept
in the reference's operation order (IEEE double, no fused multiply-add), so the
stencil results are bit-identical to the reference's Numba kernels and the CG
reproduces scipy's iteration trajectory.

Array conventions follow the reference (cfd2d/grid.py:1-18): cell (i, j) with one
ghost layer, C order, j contiguous; p-like fields (nx+2, ny+2), u (nx+1, ny+2),
v (nx+2, ny+1); ``fluid`` is a bool (nx+2, ny+2) mask.
"""

from __future__ import annotations

import math
import warnings

import numpy as np
from scipy import ndimage
from scipy.sparse import csr_matrix
from scipy.sparse.csgraph import connected_components

__all__ = [
    "SIDES", "LIMITERS", "OGrid", "circle_mask", "ellipse_mask", "rectangle_mask",
    "obstacle_mask", "OBC", "OBoundary", "momentum_tendencies", "obstacle_bc",
    "scalar_transport", "OPressure", "pcg_scipy_trajectory", "OScalarBC", "OScalarField",
    "OPassiveScalar", "OBoussinesq", "OSmagorinsky", "OKOmegaSST", "OSimulation", "cavity", "cylinder",
    "custom_obstacles", "heated_cavity", "sst_channel", "add_scalar", "wall_distance",
    "wall_adjacent_cells", "strain_rate_squared", "KAPPA", "cell_velocity", "cell_pressure",
    "cell_vorticity", "streamfunction", "available_fields", "field_data", "sample_u", "sample_v",
    "sample_field", "line_points", "OFieldAverage", "write_vtk_bytes",
    "vof_advect", "OVOF", "dam_break", "polygon_mask", "naca4_coordinates", "naca4_mask",
    "image_solid_pixels", "image_mask",
]

SIDES = ("left", "right", "bottom", "top")
# von Karman constant of the Smagorinsky wall damping, cfd2d/turbulence.py:21
KAPPA = 0.41
# limiter codes, cfd2d/kernels.py:33
LIMITERS = {"upwind": 0, "vanleer": 1, "minmod": 2, "superbee": 3, "linear": 4, "mc": 5}


# --------------------------------------------------------------------------- #
# Grid and geometry (cfd2d/grid.py:26-148, cfd2d/geometry.py:17-40)
# --------------------------------------------------------------------------- #
class OGrid:
    """Uniform MAC grid with ghost layer and fluid mask (cfd2d/grid.py:29-42)."""

    def __init__(self, nx, ny, lx, ly):
        if nx < 4 or ny < 4:
            raise ValueError("grid needs at least 4 cells per direction")
        self.nx, self.ny = int(nx), int(ny)
        self.lx, self.ly = float(lx), float(ly)
        self.dx = self.lx / self.nx
        self.dy = self.ly / self.ny
        self.fluid = np.zeros((self.nx + 2, self.ny + 2), dtype=bool)
        self.fluid[1:-1, 1:-1] = True
        self.periodic_x = False

    def centres(self):
        # cfd2d/grid.py:47-55, 67-69: (arange + 0.5) * d, meshgrid 'ij'
        xc = (np.arange(self.nx) + 0.5) * self.dx
        yc = (np.arange(self.ny) + 0.5) * self.dy
        return np.meshgrid(xc, yc, indexing="ij")

    @property
    def xc(self):
        return (np.arange(self.nx) + 0.5) * self.dx

    @property
    def yc(self):
        return (np.arange(self.ny) + 0.5) * self.dy

    def add_obstacle(self, mask):
        # cfd2d/grid.py:91-98
        self.fluid[1:-1, 1:-1] &= ~np.asarray(mask, dtype=bool)

    def finalize(self):
        """Turn fluid regions without contact to the domain border into solid.

        cfd2d/grid.py:100-125: 4-connected labelling of the interior fluid; if there
        is at most one region nothing changes; otherwise every region that has no
        cell on the outermost interior ring is removed.
        """
        inner = self.fluid[1:-1, 1:-1]
        lab, n = ndimage.label(inner)
        if n <= 1:
            return 0
        ring = np.zeros_like(inner)
        ring[0, :] = ring[-1, :] = ring[:, 0] = ring[:, -1] = True
        keep = np.unique(lab[ring & inner])
        keep = keep[keep > 0]
        enclosed = inner & ~np.isin(lab, keep)
        k = int(enclosed.sum())
        if k:
            self.fluid[1:-1, 1:-1] &= ~enclosed
        return k

    def set_periodic_x(self):
        # cfd2d/grid.py:127-133
        self.periodic_x = True
        self.fluid[0, :] = self.fluid[self.nx, :]
        self.fluid[self.nx + 1, :] = self.fluid[1, :]
        self.fluid[:, 0] = False
        self.fluid[:, -1] = False

    def interior_solid_padded(self):
        # cfd2d/grid.py:74-78
        s = ~self.fluid
        s[0, :] = s[-1, :] = s[:, 0] = s[:, -1] = False
        return s

    def u_fluid_faces(self):
        # cfd2d/grid.py:138-142
        return self.fluid[:-1, :] & self.fluid[1:, :]

    def v_fluid_faces(self):
        # cfd2d/grid.py:144-148
        return self.fluid[:, :-1] & self.fluid[:, 1:]


def circle_mask(g, xc, yc, r):
    # cfd2d/geometry.py:17-22: (X-xc)**2 + (Y-yc)**2 <= r**2
    if r <= 0:
        raise ValueError("radius must be positive")
    X, Y = g.centres()
    return (X - xc) ** 2 + (Y - yc) ** 2 <= r ** 2


def ellipse_mask(g, xc, yc, a, b, angle_deg=0.0):
    # cfd2d/geometry.py:25-32
    X, Y = g.centres()
    phi = np.deg2rad(angle_deg)
    c, s = np.cos(phi), np.sin(phi)
    xr = (X - xc) * c + (Y - yc) * s
    yr = -(X - xc) * s + (Y - yc) * c
    return (xr / a) ** 2 + (yr / b) ** 2 <= 1.0


def rectangle_mask(g, x0, y0, x1, y1):
    # cfd2d/geometry.py:35-40
    xa, xb = sorted((x0, x1))
    ya, yb = sorted((y0, y1))
    X, Y = g.centres()
    return (X >= xa) & (X <= xb) & (Y >= ya) & (Y <= yb)


def polygon_mask(g, points):
    """cfd2d/geometry.py:43-51: cell centres inside a closed polygon.

    The reference asks matplotlib (>= 3.7, not installed here) for
    ``Path(points).contains_points(centres)`` with radius 0. That is the crossings
    test of E. Haines, "Point in Polygon Strategies" (Graphics Gems IV, 1994): a ray
    from the point towards +x, an edge counted when its end points lie on opposite
    sides (y >= Y against y < Y) and the sign test
    ``(y1 - Y) (x0 - x1) >= (x1 - X) (y0 - y1)`` equals the side of the second end
    point; the polygon is closed from the last point back to the first. Restated
    here edge by edge over all centres at once."""
    pts = np.asarray(points, dtype=float)
    if pts.ndim != 2 or pts.shape[1] != 2 or len(pts) < 3:
        raise ValueError("a polygon needs at least 3 points (x, y)")
    X, Y = g.centres()
    inside = np.zeros(X.shape, dtype=bool)
    x0, y0 = pts[-1]
    for x1, y1 in pts:
        f0, f1 = y0 >= Y, y1 >= Y
        hit = (f0 != f1) & (((y1 - Y) * (x0 - x1) >= (x1 - X) * (y0 - y1)) == f1)
        inside ^= hit
        x0, y0 = x1, y1
    return inside


def naca4_coordinates(code, chord=1.0, n=200, closed_te=True):
    """cfd2d/geometry.py:54-102: outline of a NACA 4-digit section from the published
    formulas (Abbott and von Doenhoff, Theory of Wing Sections, 1959): thickness
    5 t (0.2969 sqrt(x) - 0.1260 x - 0.3516 x^2 + 0.2843 x^3 + a4 x^4), a4 = -0.1036
    for a closed trailing edge, else -0.1015; camber line m/p^2 (2 p x - x^2) ahead of
    p, m/(1-p)^2 ((1 - 2p) + 2 p x - x^2) behind it; the thickness is laid off normal
    to the camber line. n cosine-spaced stations per side; the outline runs from the
    trailing edge over the upper side to the nose and back along the lower side."""
    code = str(code).strip()
    if len(code) != 4 or not code.isdigit():
        raise ValueError("a NACA code has exactly 4 digits")
    m, p, t = int(code[0]) / 100.0, int(code[1]) / 10.0, int(code[2:]) / 100.0
    if t <= 0:
        raise ValueError("the thickness must be positive")
    beta = np.linspace(0.0, np.pi, n)
    x = 0.5 * (1.0 - np.cos(beta))
    a4 = -0.1036 if closed_te else -0.1015
    yt = 5 * t * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x**2 + 0.2843 * x**3 + a4 * x**4)
    yc, dyc = np.zeros_like(x), np.zeros_like(x)
    if m > 0 and p > 0:
        f = x < p
        b = ~f
        yc[f] = m / p**2 * (2 * p * x[f] - x[f] ** 2)
        dyc[f] = 2 * m / p**2 * (p - x[f])
        yc[b] = m / (1 - p) ** 2 * ((1 - 2 * p) + 2 * p * x[b] - x[b] ** 2)
        dyc[b] = 2 * m / (1 - p) ** 2 * (p - x[b])
    th = np.arctan(dyc)
    xu, yu = x - yt * np.sin(th), yc + yt * np.cos(th)
    xl, yl = x + yt * np.sin(th), yc - yt * np.cos(th)
    return np.column_stack([np.concatenate([xu[::-1], xl[1:]]) * chord,
                            np.concatenate([yu[::-1], yl[1:]]) * chord])


def naca4_mask(g, code, x_le, y_le, chord, angle_of_attack_deg=0.0):
    # cfd2d/geometry.py:105-116: outline turned clockwise about the leading edge
    pts = naca4_coordinates(code, chord)
    a = np.deg2rad(angle_of_attack_deg)
    xr = pts[:, 0] * np.cos(a) + pts[:, 1] * np.sin(a)
    yr = -pts[:, 0] * np.sin(a) + pts[:, 1] * np.cos(a)
    return polygon_mask(g, np.column_stack([xr + x_le, yr + y_le]))


def image_solid_pixels(path, threshold=0.5, invert=False):
    """cfd2d/geometry.py:136-149: solid pixels of an image file (PIL). Dark pixels
    (mean grey < threshold) are solid; with an alpha channel opaque pixels are, and
    where every pixel is opaque the dark opaque ones."""
    from PIL import Image

    img = Image.open(path)
    if img.mode in ("RGBA", "LA") or (img.mode == "P" and "transparency" in img.info):
        rgba = np.asarray(img.convert("RGBA"), dtype=float) / 255.0
        grey = rgba[..., :3].mean(axis=2)
        a = rgba[..., 3]
        solid = (a > 0.5) & (grey < threshold) if a.min() > 0.5 else a > 0.5
    else:
        solid = np.asarray(img.convert("L"), dtype=float) / 255.0 < threshold
    return ~solid if invert else solid


def image_mask(g, path, x0=0.0, y0=0.0, width=None, height=None, threshold=0.5, invert=False):
    """cfd2d/geometry.py:119-163: the bitmap laid on [x0, x0 + width] x
    [y0, y0 + height] (the whole domain without width; the aspect ratio kept without
    height); a centre inside takes the pixel at column floor(sx w), row
    floor((1 - sy) h), clamped (row 0 is the top of the image)."""
    from pathlib import Path as _P

    if not _P(path).exists():
        raise FileNotFoundError(path)
    solid = image_solid_pixels(path, threshold, invert)
    h, w = solid.shape
    if width is None:
        x0, y0, width, height = 0.0, 0.0, g.lx, g.ly
    if height is None:
        height = width * h / w
    X, Y = g.centres()
    sx, sy = (X - x0) / width, (Y - y0) / height
    inside = (sx >= 0) & (sx < 1) & (sy >= 0) & (sy < 1)
    col = np.clip((sx * w).astype(int), 0, w - 1)
    row = np.clip(((1.0 - sy) * h).astype(int), 0, h - 1)
    out = np.zeros(X.shape, dtype=bool)
    out[inside] = solid[row[inside], col[inside]]
    return out


def obstacle_mask(g, spec):
    # cfd2d/geometry.py:166-195
    typ = spec.get("typ", "").lower()
    if typ == "kreis":
        return circle_mask(g, spec["x"], spec["y"], spec["r"])
    if typ == "ellipse":
        return ellipse_mask(g, spec["x"], spec["y"], spec["a"], spec["b"], spec.get("winkel", 0.0))
    if typ == "rechteck":
        return rectangle_mask(g, spec["x0"], spec["y0"], spec["x1"], spec["y1"])
    if typ == "naca":
        return naca4_mask(g, spec.get("code", "0012"), spec["x"], spec["y"], spec["sehne"],
                          spec.get("winkel", 0.0))
    if typ == "polygon":
        return polygon_mask(g, spec["punkte"])
    if typ == "bild":
        return image_mask(g, spec["pfad"], spec.get("x", 0.0), spec.get("y", 0.0), spec.get("breite"),
                          spec.get("hoehe"), spec.get("schwelle", 0.5), spec.get("invertieren", False))
    raise ValueError(f"unknown obstacle type {typ!r}")


# --------------------------------------------------------------------------- #
# Domain boundary (cfd2d/boundary.py:41-245)
# --------------------------------------------------------------------------- #
class OBC:
    """Side condition (cfd2d/boundary.py:41-51)."""

    def __init__(self, kind="noslip", velocity=0.0, profile="uniform"):
        if kind not in ("noslip", "slip", "inflow", "outflow", "periodic"):
            raise ValueError(kind)
        self.kind, self.velocity, self.profile = kind, float(velocity), profile


def _inflow_profile(coords, open_mask, h, mean, profile):
    # cfd2d/boundary.py:63-89: one profile per contiguous open run of the side
    out = np.zeros_like(coords)
    n = len(open_mask)
    j = 0
    while j < n:
        if not open_mask[j]:
            j += 1
            continue
        k = j
        while k + 1 < n and open_mask[k + 1]:
            k += 1
        a = coords[j] - 0.5 * h
        b = coords[k] + 0.5 * h
        s = coords[j:k + 1]
        if profile == "parabolic":
            out[j:k + 1] = 6.0 * mean * (s - a) * (b - s) / (b - a) ** 2
        else:
            out[j:k + 1] = mean
        j = k + 1
    return out


class OBoundary:
    """Ghost/face boundary values on u and v (cfd2d/boundary.py:92-245)."""

    def __init__(self, g, bcs):
        self.g, self.bcs = g, bcs
        pl = bcs["left"].kind == "periodic"
        if pl != (bcs["right"].kind == "periodic"):
            raise ValueError("periodic needs left and right")
        self.periodic = pl
        if pl:
            g.set_periodic_x()
        fl, nx, ny = g.fluid, g.nx, g.ny
        self.open = {"left": fl[1, 1:ny + 1].copy(), "right": fl[nx, 1:ny + 1].copy(),
                     "bottom": fl[1:nx + 1, 1].copy(), "top": fl[1:nx + 1, ny].copy()}
        self.inflow = {}
        for side, bc in bcs.items():
            if bc.kind != "inflow":
                continue
            if side in ("left", "right"):
                vals = _inflow_profile(g.yc, self.open[side], g.dy, bc.velocity, bc.profile)
            else:
                vals = _inflow_profile(g.xc, self.open[side], g.dx, bc.velocity, bc.profile)
            self.inflow[side] = (1.0 if side in ("left", "bottom") else -1.0) * vals

    def outflow_mask(self, side):
        # cfd2d/boundary.py:137-141
        if self.bcs[side].kind != "outflow":
            return np.zeros_like(self.open[side])
        return self.open[side]

    def apply(self, u, v):
        # cfd2d/boundary.py:143-223, same statement order
        g, nx, ny = self.g, self.g.nx, self.g.ny
        if self.periodic:
            u[0, :] = u[nx, :]
            v[0, :] = v[nx, :]
            v[nx + 1, :] = v[1, :]
        for side, inner, ghost, nrm in (("left", 1, 0, 0), ("right", nx, nx + 1, nx)):
            bc, op = self.bcs[side], self.open[side]
            if bc.kind == "noslip":
                u[nrm, 1:ny + 1] = 0.0
                v[ghost, :] = 2.0 * bc.velocity - v[inner, :]
            elif bc.kind == "slip":
                u[nrm, 1:ny + 1] = 0.0
                v[ghost, :] = v[inner, :]
            elif bc.kind == "inflow":
                u[nrm, 1:ny + 1] = self.inflow[side]
                v[ghost, :] = -v[inner, :]
            elif bc.kind == "outflow":
                u[nrm, 1:ny + 1] = np.where(op, u[nrm, 1:ny + 1], 0.0)
                v[ghost, :] = v[inner, :]
        for side, inner, ghost, nrm in (("bottom", 1, 0, 0), ("top", ny, ny + 1, ny)):
            bc, op = self.bcs[side], self.open[side]
            if bc.kind == "noslip":
                v[1:nx + 1, nrm] = 0.0
                u[:, ghost] = 2.0 * bc.velocity - u[:, inner]
            elif bc.kind == "slip":
                v[1:nx + 1, nrm] = 0.0
                u[:, ghost] = u[:, inner]
            elif bc.kind == "inflow":
                v[1:nx + 1, nrm] = self.inflow[side]
                u[:, ghost] = -u[:, inner]
            elif bc.kind == "outflow":
                v[1:nx + 1, nrm] = np.where(op, v[1:nx + 1, nrm], 0.0)
                u[:, ghost] = u[:, inner]
        if not self.periodic:
            u[0, 1:ny + 1][~self.open["left"]] = 0.0
            u[nx, 1:ny + 1][~self.open["right"]] = 0.0
        v[1:nx + 1, 0][~self.open["bottom"]] = 0.0
        v[1:nx + 1, ny][~self.open["top"]] = 0.0

    def extrapolate_outflow_predictor(self, F, G):
        # cfd2d/boundary.py:225-245
        nx, ny = self.g.nx, self.g.ny
        if self.periodic:
            F[0, :] = F[nx, :]
        if self.bcs["left"].kind == "outflow":
            m = self.open["left"]
            F[0, 1:ny + 1][m] = F[1, 1:ny + 1][m]
        if self.bcs["right"].kind == "outflow":
            m = self.open["right"]
            F[nx, 1:ny + 1][m] = F[nx - 1, 1:ny + 1][m]
        if self.bcs["bottom"].kind == "outflow":
            m = self.open["bottom"]
            G[1:nx + 1, 0][m] = G[1:nx + 1, 1][m]
        if self.bcs["top"].kind == "outflow":
            m = self.open["top"]
            G[1:nx + 1, ny][m] = G[1:nx + 1, ny - 1][m]


# --------------------------------------------------------------------------- #
# Stencils (cfd2d/kernels.py:44-391), vectorised with the same per-element order
# --------------------------------------------------------------------------- #
def momentum_tendencies(u, v, fluid, nx, ny, dx, dy, nu, variable, gamma, periodic, hu, hv,
                        rho, var_density):
    """hu, hv = diffusion - convection on fluid faces (cfd2d/kernels.py:44-155)."""
    idx2 = 1.0 / (dx * dx)
    idy2 = 1.0 / (dy * dy)
    idx = 1.0 / dx
    idy = 1.0 / dy
    hu[:] = 0.0
    hv[:] = 0.0
    imax = nx if periodic else nx - 1
    nu0 = nu[1, 1]
    gx = gamma * idx
    gy = gamma * idy

    # u momentum on faces i = 1..imax, j = 1..ny (kernels.py:85-119)
    I = np.arange(1, imax + 1)
    ip = np.where(I < nx, I + 1, 1)
    J = slice(1, ny + 1)
    Jn = slice(2, ny + 2)
    Js = slice(0, ny)
    m = fluid[1:imax + 1, J] & fluid[2:imax + 2, J]
    uc = u[1:imax + 1, J]
    ue = u[ip, J]
    uw = u[0:imax, J]
    un = u[1:imax + 1, Jn]
    us = u[1:imax + 1, Js]
    if variable:
        nu_e = nu[2:imax + 2, J]
        nu_w = nu[1:imax + 1, J]
        nu_n = 0.25 * (nu[1:imax + 1, J] + nu[2:imax + 2, J] + nu[1:imax + 1, Jn] + nu[2:imax + 2, Jn])
        nu_s = 0.25 * (nu[1:imax + 1, J] + nu[2:imax + 2, J] + nu[1:imax + 1, Js] + nu[2:imax + 2, Js])
        diff = (2.0 * nu_e * (ue - uc) - 2.0 * nu_w * (uc - uw)) * idx2 + idy * (
            nu_n * ((un - uc) * idy + (v[2:imax + 2, J] - v[1:imax + 1, J]) * idx)
            - nu_s * ((uc - us) * idy + (v[2:imax + 2, 0:ny] - v[1:imax + 1, 0:ny]) * idx))
    else:
        diff = nu0 * ((ue - 2.0 * uc + uw) * idx2 + (un - 2.0 * uc + us) * idy2)
    if var_density:
        diff = diff / (0.5 * (rho[1:imax + 1, J] + rho[2:imax + 2, J]))
    a_e = 0.5 * (uc + ue)
    a_w = 0.5 * (uw + uc)
    du2dx = idx * (a_e * a_e - a_w * a_w) + gx * (
        np.abs(a_e) * 0.5 * (uc - ue) - np.abs(a_w) * 0.5 * (uw - uc))
    v_n = 0.5 * (v[1:imax + 1, J] + v[2:imax + 2, J])
    v_s = 0.5 * (v[1:imax + 1, 0:ny] + v[2:imax + 2, 0:ny])
    duvdy = idy * (v_n * 0.5 * (uc + un) - v_s * 0.5 * (us + uc)) + gy * (
        np.abs(v_n) * 0.5 * (uc - un) - np.abs(v_s) * 0.5 * (us - uc))
    hu[1:imax + 1, J] = np.where(m, diff - du2dx - duvdy, 0.0)

    # v momentum on faces i = 1..nx, j = 1..ny-1 (kernels.py:122-155)
    Ii = slice(1, nx + 1)
    Ie = slice(2, nx + 2)
    Iw = slice(0, nx)
    Jc = slice(1, ny)
    Jn = slice(2, ny + 1)
    Js = slice(0, ny - 1)
    m = fluid[Ii, 1:ny] & fluid[Ii, 2:ny + 1]
    vc = v[Ii, Jc]
    ve = v[Ie, Jc]
    vw = v[Iw, Jc]
    vn = v[Ii, Jn]
    vs = v[Ii, Js]
    if variable:
        nu_n = nu[Ii, 2:ny + 1]
        nu_s = nu[Ii, 1:ny]
        nu_e = 0.25 * (nu[Ii, 1:ny] + nu[Ie, 1:ny] + nu[Ii, 2:ny + 1] + nu[Ie, 2:ny + 1])
        nu_w = 0.25 * (nu[Ii, 1:ny] + nu[Iw, 1:ny] + nu[Ii, 2:ny + 1] + nu[Iw, 2:ny + 1])
        diff = (2.0 * nu_n * (vn - vc) - 2.0 * nu_s * (vc - vs)) * idy2 + idx * (
            nu_e * ((ve - vc) * idx + (u[1:nx + 1, 2:ny + 1] - u[1:nx + 1, 1:ny]) * idy)
            - nu_w * ((vc - vw) * idx + (u[0:nx, 2:ny + 1] - u[0:nx, 1:ny]) * idy))
    else:
        diff = nu0 * ((ve - 2.0 * vc + vw) * idx2 + (vn - 2.0 * vc + vs) * idy2)
    if var_density:
        diff = diff / (0.5 * (rho[Ii, 1:ny] + rho[Ii, 2:ny + 1]))
    b_n = 0.5 * (vc + vn)
    b_s = 0.5 * (vs + vc)
    dv2dy = idy * (b_n * b_n - b_s * b_s) + gy * (
        np.abs(b_n) * 0.5 * (vc - vn) - np.abs(b_s) * 0.5 * (vs - vc))
    u_e = 0.5 * (u[1:nx + 1, 1:ny] + u[1:nx + 1, 2:ny + 1])
    u_w = 0.5 * (u[0:nx, 1:ny] + u[0:nx, 2:ny + 1])
    duvdx = idx * (u_e * 0.5 * (vc + ve) - u_w * 0.5 * (vw + vc)) + gx * (
        np.abs(u_e) * 0.5 * (vc - ve) - np.abs(u_w) * 0.5 * (vw - vc))
    hv[Ii, Jc] = np.where(m, diff - duvdx - dv2dy, 0.0)


def obstacle_bc(u, v, fluid, nx, ny, periodic):
    """Solid-face velocities (cfd2d/kernels.py:158-209).

    Faces with exactly one fluid cell get 0; faces inside a solid get minus the mean of
    the adjacent both-fluid tangential neighbours. The neighbours read are never
    written by this function, so a vectorised update equals the reference loop.
    """
    imax = nx if periodic else nx - 1
    fl = fluid[1:imax + 1, 1:ny + 1]
    fr = fluid[2:imax + 2, 1:ny + 1]
    one = fl ^ fr
    none = ~fl & ~fr
    top = fluid[1:imax + 1, 2:ny + 2] & fluid[2:imax + 2, 2:ny + 2]
    bot = fluid[1:imax + 1, 0:ny] & fluid[2:imax + 2, 0:ny]
    # the reference adds into s = 0.0 in the order top, bottom
    s = np.where(top, u[1:imax + 1, 2:ny + 2], 0.0) + np.where(bot, u[1:imax + 1, 0:ny], 0.0)
    c = top.astype(np.int64) + bot.astype(np.int64)
    with np.errstate(invalid="ignore", divide="ignore"):
        val = np.where(c > 0, -s / np.maximum(c, 1), 0.0)
    blk = u[1:imax + 1, 1:ny + 1]
    blk[one] = 0.0
    blk[none] = val[none]
    if periodic:
        u[0, :] = u[nx, :]

    fb = fluid[1:nx + 1, 1:ny]
    ft = fluid[1:nx + 1, 2:ny + 1]
    one = fb ^ ft
    none = ~fb & ~ft
    east = fluid[2:nx + 2, 1:ny] & fluid[2:nx + 2, 2:ny + 1]
    west = fluid[0:nx, 1:ny] & fluid[0:nx, 2:ny + 1]
    s = np.where(east, v[2:nx + 2, 1:ny], 0.0) + np.where(west, v[0:nx, 1:ny], 0.0)
    c = east.astype(np.int64) + west.astype(np.int64)
    with np.errstate(invalid="ignore", divide="ignore"):
        val = np.where(c > 0, -s / np.maximum(c, 1), 0.0)
    blk = v[1:nx + 1, 1:ny]
    blk[one] = 0.0
    blk[none] = val[none]


def _limiter(r, kind):
    # cfd2d/kernels.py:215-235 (r is an array; non-positive r gives 0 except linear)
    pos = r > 0.0
    with np.errstate(all="ignore"):
        if kind == 0:
            return np.zeros_like(r)
        if kind == 1:
            return np.where(pos, 2.0 * r / (1.0 + r), 0.0)
        if kind == 2:
            return np.where(pos, np.minimum(r, 1.0), 0.0)
        if kind == 3:
            return np.where(pos, np.maximum(np.minimum(2.0 * r, 1.0), np.minimum(r, 2.0)), 0.0)
        if kind == 5:
            return np.where(pos, np.minimum(2.0 * r, np.minimum(0.5 * (1.0 + r), 2.0)), 0.0)
    return np.ones_like(r)


def _face_value(phu, phc, phd, has_u, kind):
    # cfd2d/kernels.py:238-251
    if kind == 0:
        return phc.copy()
    if kind == 4:
        return 0.5 * (phc + phd)
    den = phd - phc
    tiny = np.abs(den) < 1e-300
    with np.errstate(all="ignore"):
        r = (phc - phu) / np.where(tiny, 1.0, den)
        out = phc + 0.5 * _limiter(r, kind) * den
    return np.where(~has_u | tiny, phc, out)


def _harm(a, b):
    # harmonic face diffusivity, cfd2d/kernels.py:325-327
    s = a + b
    with np.errstate(all="ignore"):
        return np.where(s > 0.0, 2.0 * a * b / np.where(s > 0.0, s, 1.0), 0.0)


def scalar_transport(phi, u, v, fluid, nx, ny, dx, dy, diff, limiter, periodic,
                     bt_l, bv_l, bt_r, bv_r, bt_b, bv_b, bt_t, bv_t, obs_t, obs_v, out):
    """out = -div(u phi) + div(D grad phi) on fluid cells (cfd2d/kernels.py:254-391).

    The reference accumulates into ``out`` face by face (x faces by increasing i, then
    y faces by increasing j). For a cell the two x contributions are added first
    (their order is immaterial: the first addition is onto 0), then the south and
    the north y contributions; this function sums the per-face terms in that order.
    """
    fl = fluid
    P = (slice(1, nx + 1), slice(1, ny + 1))
    # ---- x faces: term entering cell (i, j) from its west face (xw) and east face (xe)
    xw = np.zeros((nx, ny))
    xe = np.zeros((nx, ny))
    # interior faces i = 1..nx-1 (+ face nx when periodic, joining cell nx and cell 1)
    nfx = nx if periodic else nx - 1
    I = np.arange(1, nfx + 1)
    L = I
    R = np.where(I < nx, I + 1, 1)
    J = np.arange(1, ny + 1)
    LL, JJ = np.meshgrid(L, J, indexing="ij")
    RR, _ = np.meshgrid(R, J, indexing="ij")
    fL = fl[LL, JJ]
    fR = fl[RR, JJ]
    uf = u[I, 1:ny + 1]
    pos = uf >= 0.0
    C = np.where(pos, LL, RR)
    D = np.where(pos, RR, LL)
    Ui = np.where(pos, LL - 1, RR + 1)
    if periodic:
        Ui = np.where(Ui < 1, nx, np.where(Ui > nx, 1, Ui))
    else:
        Ui = np.where((Ui < 1) | (Ui > nx), -1, Ui)
    has_u = (Ui >= 1) & fl[np.clip(Ui, 0, nx + 1), JJ]
    phu = np.where(has_u, phi[np.clip(Ui, 0, nx + 1), JJ], 0.0)
    phf = _face_value(phu, phi[C, JJ], phi[D, JJ], has_u, limiter)
    df = _harm(diff[LL, JJ], diff[RR, JJ])
    F = uf * phf - df * (phi[RR, JJ] - phi[LL, JJ]) / dx
    both = fL & fR
    tL = np.where(both, -(F / dx), 0.0)
    tR = np.where(both, F / dx, 0.0)
    if obs_t == 1:
        one = fL ^ fR
        Pc = np.where(fL, LL, RR)
        tob = diff[Pc, JJ] * (obs_v - phi[Pc, JJ]) / (0.5 * dx) / dx
        tL = np.where(one & fL, tob, tL)
        tR = np.where(one & fR, tob, tR)
    # face k joins cells L=k (its east face) and R (its west face)
    xe[L - 1, :] = tL
    xw[R - 1, :] = tR
    if not periodic:
        for side, face, cell, sgn, bt, bv in (("l", 0, 1, 1.0, bt_l, bv_l),
                                              ("r", nx, nx, -1.0, bt_r, bv_r)):
            un = sgn * u[face, 1:ny + 1]
            ph = phi[cell, 1:ny + 1]
            bt = np.asarray(bt)
            bv = np.asarray(bv, dtype=float)
            phb = np.where((bt == 1) & (un > 0.0), bv, ph)
            flux = un * phb
            flux = np.where(bt == 1, flux + diff[cell, 1:ny + 1] * (bv - ph) / (0.5 * dx),
                            np.where(bt == 2, flux + bv, flux))
            t = np.where(fl[cell, 1:ny + 1], flux / dx, 0.0)
            if side == "l":
                xw[0, :] = t
            else:
                xe[nx - 1, :] = t
    # ---- y faces: south (ys) and north (yn) terms
    ys = np.zeros((nx, ny))
    yn = np.zeros((nx, ny))
    Ii = np.arange(1, nx + 1)
    Jf = np.arange(1, ny)
    II, BB = np.meshgrid(Ii, Jf, indexing="ij")
    TT = BB + 1
    fB = fl[II, BB]
    fT = fl[II, TT]
    vf = v[1:nx + 1, 1:ny]
    pos = vf >= 0.0
    C = np.where(pos, BB, TT)
    D = np.where(pos, TT, BB)
    Uj = np.where(pos, BB - 1, TT + 1)
    has_u = (Uj >= 1) & (Uj <= ny) & fl[II, np.clip(Uj, 0, ny + 1)]
    phu = np.where(has_u, phi[II, np.clip(Uj, 0, ny + 1)], 0.0)
    phf = _face_value(phu, phi[II, C], phi[II, D], has_u, limiter)
    df = _harm(diff[II, BB], diff[II, TT])
    F = vf * phf - df * (phi[II, TT] - phi[II, BB]) / dy
    both = fB & fT
    tB = np.where(both, -(F / dy), 0.0)
    tT = np.where(both, F / dy, 0.0)
    if obs_t == 1:
        one = fB ^ fT
        Pc = np.where(fB, BB, TT)
        tob = diff[II, Pc] * (obs_v - phi[II, Pc]) / (0.5 * dy) / dy
        tB = np.where(one & fB, tob, tB)
        tT = np.where(one & fT, tob, tT)
    yn[:, 0:ny - 1] = tB
    ys[:, 1:ny] = tT
    for side, face, cell, sgn, bt, bv in (("b", 0, 1, 1.0, bt_b, bv_b),
                                          ("t", ny, ny, -1.0, bt_t, bv_t)):
        vn = sgn * v[1:nx + 1, face]
        ph = phi[1:nx + 1, cell]
        bt = np.asarray(bt)
        bv = np.asarray(bv, dtype=float)
        phb = np.where((bt == 1) & (vn > 0.0), bv, ph)
        flux = vn * phb
        flux = np.where(bt == 1, flux + diff[1:nx + 1, cell] * (bv - ph) / (0.5 * dy),
                        np.where(bt == 2, flux + bv, flux))
        t = np.where(fl[1:nx + 1, cell], flux / dy, 0.0)
        if side == "b":
            ys[:, 0] = t
        else:
            yn[:, ny - 1] = t
    total = ((xw + xe) + ys) + yn
    out[:] = 0.0
    out[P] = np.where(fl[P], total, 0.0)


# --------------------------------------------------------------------------- #
# Pressure Poisson (cfd2d/pressure.py:29-185) and scipy's CG trajectory
# --------------------------------------------------------------------------- #
def pcg_scipy_trajectory(matvec, b, x0, rtol, maxiter, dinv, callback=None):
    """Jacobi-preconditioned CG in the exact form of scipy.sparse.linalg.cg.

    scipy 1.18.1 ``scipy/sparse/linalg/_isolve/iterative.py:311-431`` (installed
    third-party code called by cfd2d/pressure.py:171): atol = rtol*||b||; if ||b|| == 0
    return b; r = b - A x0 only if x0 has a nonzero; the test ||r|| < atol is made at
    the top of every iteration; p = z on the first spin, then p = beta*p + z.
    Returns (x, info, iterations).
    """
    bnrm2 = math.sqrt(np.dot(b, b))
    atol = max(0.0, rtol * bnrm2)
    if bnrm2 == 0:
        return b, 0, 0
    x = x0.copy()
    r = b - matvec(x) if x.any() else b.copy()
    rho_prev = None
    p = None
    for it in range(maxiter):
        if math.sqrt(np.dot(r, r)) < atol:
            return x, 0, it
        z = dinv * r
        rho = np.dot(r, z)
        if it > 0:
            beta = rho / rho_prev
            p *= beta
            p += z
        else:
            p = z.copy()
        q = matvec(p)
        alpha = rho / np.dot(p, q)
        x += alpha * p
        r -= alpha * q
        rho_prev = rho
        if callback is not None:
            callback(x)
    return x, maxiter, maxiter


class OPressure:
    """5-point operator A = -Lap over the fluid cells (cfd2d/pressure.py:32-140)."""

    # scipy cg's maxiter in cfd2d/pressure.py:171; the CPU timing arm lowers it to
    # time a bounded sample of a solve
    maxiter = 5000
    # "numpy": pcg_scipy_trajectory on the stencil matvec (the parity form);
    # "scipy": scipy.sparse.linalg.cg on the assembled matrix with the Jacobi
    # preconditioner, the call cfd2d/pressure.py:171 makes (the timing form).
    # Set on the class to reach the solve a simulation makes while it is built.
    engine = "numpy"

    def __init__(self, g, boundary, method="cg", tol=1e-10):
        if method == "lu":
            method = "direct"
        if method not in ("direct", "cg"):
            raise ValueError(method)
        self.g, self.method, self.tol = g, method, tol
        nx, ny = g.nx, g.ny
        self.dx2 = dx2 = 1.0 / g.dx ** 2
        self.dy2 = dy2 = 1.0 / g.dy ** 2
        f = g.fluid[1:-1, 1:-1].copy()
        self.fluid = f
        n = int(f.sum())
        if n == 0:
            raise ValueError("no fluid cells")
        self.n = n
        idx = -np.ones((nx, ny), dtype=np.int64)
        idx[f] = np.arange(n)
        self.idx = idx
        bx = f[:-1, :] & f[1:, :]
        by = f[:, :-1] & f[:, 1:]
        self.both_x, self.both_y = bx, by
        self.periodic = boundary.periodic
        bp = (f[-1, :] & f[0, :]) if self.periodic else np.zeros(ny, dtype=bool)
        self.both_p = bp
        # diagonal in the reference's accumulation order (pressure.py:64-125)
        diag = np.zeros((nx, ny))
        diag[:-1, :][bx] += dx2
        diag[1:, :][bx] += dx2
        diag[:, :-1][by] += dy2
        diag[:, 1:][by] += dy2
        if self.periodic:
            diag[-1, :][bp] += dx2
            diag[0, :][bp] += dx2
        self.dirichlet = {s: boundary.outflow_mask(s) for s in SIDES}
        diag[0, :][self.dirichlet["left"]] += 2 * dx2
        diag[-1, :][self.dirichlet["right"]] += 2 * dx2
        diag[:, 0][self.dirichlet["bottom"]] += 2 * dy2
        diag[:, -1][self.dirichlet["top"]] += 2 * dy2
        has_dir = np.zeros((nx, ny), dtype=bool)
        has_dir[0, :] |= self.dirichlet["left"]
        has_dir[-1, :] |= self.dirichlet["right"]
        has_dir[:, 0] |= self.dirichlet["bottom"]
        has_dir[:, -1] |= self.dirichlet["top"]
        # components of the coupling graph; each Neumann-only component pins its first
        # cell in C order (pressure.py:105-125)
        a = np.concatenate([idx[:-1, :][bx], idx[:, :-1][by], idx[-1, :][bp]])
        b = np.concatenate([idx[1:, :][bx], idx[:, 1:][by], idx[0, :][bp]])
        adj = csr_matrix((np.ones(a.size), (a, b)), shape=(n, n))
        ncomp, comp = connected_components(adj, directed=False)
        labels = np.zeros((nx, ny), dtype=np.int64)
        labels[f] = comp + 1
        self.labels = labels
        dir_comps = set(np.unique(labels[has_dir & f]).tolist())
        self.neumann_components = []
        self.pinned = []
        for c in range(1, ncomp + 1):
            if c not in dir_comps:
                first = int(np.argmax(comp == c - 1))
                fi, fj = np.argwhere(idx == first)[0]
                diag[fi, fj] += dx2
                self.neumann_components.append(c)
                self.pinned.append((int(fi), int(fj)))
        self.diag = diag
        self.dinv = 1.0 / diag[f]
        self.x0 = np.zeros(n)
        self.last_iterations = 0
        self.last_info = 0
        self._A = None
        if method == "direct":
            from scipy.sparse import csc_matrix
            from scipy.sparse.linalg import splu
            self._lu = splu(csc_matrix(self._assemble()), permc_spec="COLAMD")

    def _assemble(self):
        nx, ny, f, idx = self.g.nx, self.g.ny, self.fluid, self.idx
        bx, by, bp = self.both_x, self.both_y, self.both_p
        rows = [idx[:-1, :][bx], idx[1:, :][bx], idx[:, :-1][by], idx[:, 1:][by],
                idx[-1, :][bp], idx[0, :][bp], np.arange(self.n)]
        cols = [idx[1:, :][bx], idx[:-1, :][bx], idx[:, 1:][by], idx[:, :-1][by],
                idx[0, :][bp], idx[-1, :][bp], np.arange(self.n)]
        vals = [np.full(bx.sum(), -self.dx2)] * 2 + [np.full(by.sum(), -self.dy2)] * 2 + \
               [np.full(bp.sum(), -self.dx2)] * 2 + [self.diag[f]]
        return csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                          shape=(self.n, self.n))

    def _scipy_cg(self, b):
        """scipy's cg with the Jacobi preconditioner, as cfd2d/pressure.py:165-172."""
        from scipy.sparse.linalg import LinearOperator, cg

        if self._A is None:
            self._A = self._assemble().tocsc()
            dinv = self.dinv
            self._M = LinearOperator((self.n, self.n), matvec=lambda r: dinv * r)
        it = [0]

        def cb(_):
            it[0] += 1

        x, info = cg(self._A, b, x0=self.x0, rtol=self.tol, maxiter=self.maxiter, M=self._M, callback=cb)
        return x, info, it[0]

    def matvec(self, xc):
        """y = A x summed per row in increasing column order, as scipy's csc_matvec.

        Column order of a row's entries: west, south, centre, north, east; with
        periodic x the wrapped west neighbour of the first row comes last and the
        wrapped east neighbour of the last row comes first.
        """
        nx, ny, f = self.g.nx, self.g.ny, self.fluid
        X = np.zeros((nx + 2, ny + 2))
        X[1:-1, 1:-1][f] = xc
        if self.periodic:
            X[0, 1:-1] = X[nx, 1:-1]
            X[nx + 1, 1:-1] = X[1, 1:-1]
        fp = np.zeros((nx + 2, ny + 2), dtype=bool)
        fp[1:-1, 1:-1] = f
        if self.periodic:
            fp[0, 1:-1] = f[-1, :]
            fp[nx + 1, 1:-1] = f[0, :]
        c = (slice(1, nx + 1), slice(1, ny + 1))
        tW = np.where(fp[0:nx, 1:ny + 1], -self.dx2 * X[0:nx, 1:ny + 1], 0.0)
        tE = np.where(fp[2:nx + 2, 1:ny + 1], -self.dx2 * X[2:nx + 2, 1:ny + 1], 0.0)
        tS = np.where(fp[1:nx + 1, 0:ny], -self.dy2 * X[1:nx + 1, 0:ny], 0.0)
        tN = np.where(fp[1:nx + 1, 2:ny + 2], -self.dy2 * X[1:nx + 1, 2:ny + 2], 0.0)
        tC = self.diag * X[c]
        y = (((tW + tS) + tC) + tN) + tE
        if self.periodic:
            y[0, :] = (((tS[0] + tC[0]) + tN[0]) + tE[0]) + tW[0]
            y[-1, :] = (((tE[-1] + tW[-1]) + tS[-1]) + tC[-1]) + tN[-1]
        return y[f]

    def solve(self, rhs):
        """Lap(p) = rhs on the fluid cells (cfd2d/pressure.py:143-185)."""
        b = rhs[self.fluid].astype(float)
        if self.neumann_components:
            lab = self.labels[self.fluid]
            for c in self.neumann_components:
                m = lab == c
                b[m] -= b[m].mean()
        b = -b
        if self.method == "direct":
            x = self._lu.solve(b)
            self.last_iterations = 1
        else:
            if self.engine == "scipy":
                x, info, it = self._scipy_cg(b)
            else:
                x, info, it = pcg_scipy_trajectory(self.matvec, b, self.x0, self.tol, self.maxiter, self.dinv)
            self.last_iterations = it
            self.last_info = info
            if info > 0:
                warnings.warn(f"CG pressure solver did not converge ({info} iterations)")
            self.x0 = x
        p = np.zeros(self.fluid.shape)
        p[self.fluid] = x
        if self.neumann_components:
            for c in self.neumann_components:
                m = self.labels == c
                p[m] -= p[m].mean()
        return p


    def solve_variable(self, rhs, bx, by):
        """div(b grad p) = rhs with face coefficients b = 1/rho, bx (nx+1, ny), by
        (nx, ny+1); the matrix is rebuilt and solved directly on every call
        (cfd2d/pressure.py:187-244)."""
        from scipy.sparse import csc_matrix
        from scipy.sparse.linalg import spsolve

        g, f, idx = self.g, self.fluid, self.idx
        nx, ny = g.nx, g.ny
        dx2, dy2 = self.dx2, self.dy2
        bxm, bym, bp = self.both_x, self.both_y, self.both_p
        diag = np.zeros((nx, ny))
        cxi = (bx[1:nx, :] * dx2)[bxm]
        diag[:-1, :][bxm] += cxi
        diag[1:, :][bxm] += cxi
        cyi = (by[:, 1:ny] * dy2)[bym]
        diag[:, :-1][bym] += cyi
        diag[:, 1:][bym] += cyi
        cpi = np.zeros(0)
        if self.periodic:
            cpi = (bx[nx, :] * dx2)[bp]
            diag[-1, :][bp] += cpi
            diag[0, :][bp] += cpi
        d = self.dirichlet
        diag[0, :][d["left"]] += 2 * dx2 * bx[0, :][d["left"]]
        diag[-1, :][d["right"]] += 2 * dx2 * bx[nx, :][d["right"]]
        diag[:, 0][d["bottom"]] += 2 * dy2 * by[:, 0][d["bottom"]]
        diag[:, -1][d["top"]] += 2 * dy2 * by[:, ny][d["top"]]
        for fi, fj in self.pinned:
            diag[fi, fj] += dx2 * max(float(bx.max()), 1e-30)
        rows = [idx[:-1, :][bxm], idx[1:, :][bxm], idx[:, :-1][bym], idx[:, 1:][bym],
                idx[-1, :][bp], idx[0, :][bp], np.arange(self.n)]
        cols = [idx[1:, :][bxm], idx[:-1, :][bxm], idx[:, 1:][bym], idx[:, :-1][bym],
                idx[0, :][bp], idx[-1, :][bp], np.arange(self.n)]
        vals = [-cxi, -cxi, -cyi, -cyi, -cpi, -cpi, diag[f]]
        A = csc_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                       shape=(self.n, self.n))
        b = rhs[f].astype(float)
        if self.neumann_components:
            lab = self.labels[f]
            for c in self.neumann_components:
                m = lab == c
                b[m] -= b[m].mean()
        x = spsolve(A, -b)
        p = np.zeros(f.shape)
        p[f] = x
        if self.neumann_components:
            for c in self.neumann_components:
                m = self.labels == c
                p[m] -= p[m].mean()
        return p


# --------------------------------------------------------------------------- #
# Scalars and models (cfd2d/models.py:28-426, cfd2d/turbulence.py:28-325)
# --------------------------------------------------------------------------- #
class OScalarBC:
    CODES = {"zerogradient": 0, "fixed": 1, "flux": 2}

    def __init__(self, kind="zerogradient", value=0.0):
        if kind not in self.CODES:
            raise ValueError(kind)
        self.kind, self.value = kind, value

    @property
    def code(self):
        return self.CODES[self.kind]


def default_scalar_bcs(sim, inflow_value=0.0):
    # cfd2d/models.py:61-70
    return {s: (OScalarBC("fixed", inflow_value) if sim.bcs[s].kind == "inflow"
                else OScalarBC("zerogradient")) for s in SIDES}


class OScalarField:
    """Explicit TVD transport of one cell field (cfd2d/models.py:73-250)."""

    def __init__(self, name, diffusivity, bcs=None, obstacle=None, limiter="vanleer",
                 initial=0.0, source=None, lower=None, upper=None):
        self.name, self.D0 = name, float(diffusivity)
        self.bcs_in, self.obstacle = bcs, obstacle or OScalarBC("zerogradient")
        self.limiter, self.initial, self.source = limiter, initial, source
        self.lower, self.upper = lower, upper

    def attach(self, sim):
        # cfd2d/models.py:102-136
        self.sim = sim
        g = sim.grid
        nx, ny = g.nx, g.ny
        self.phi = np.zeros((nx + 2, ny + 2))
        if np.isscalar(self.initial):
            self.phi[:] = float(self.initial)
        else:
            init = np.asarray(self.initial, dtype=float)
            if init.shape == (nx, ny):
                self.phi[1:-1, 1:-1] = init
            else:
                self.phi[:] = init
        self.diff = np.full((nx + 2, ny + 2), self.D0)
        self.rhs = np.zeros_like(self.phi)
        bcs = default_scalar_bcs(sim)
        bcs.update(self.bcs_in or {})
        self.bcs = bcs
        coords = {"left": g.yc, "right": g.yc, "bottom": g.xc, "top": g.xc}
        self.bt, self.bv = {}, {}
        for side in SIDES:
            s = coords[side]
            bc = bcs[side]
            self.bt[side] = np.full(len(s), bc.code, dtype=np.int64)
            val = bc.value
            if callable(val):
                self.bv[side] = np.asarray(val(s), dtype=float)
            else:
                self.bv[side] = np.broadcast_to(np.asarray(val, dtype=float), s.shape).copy()
        self.fill_ghosts()

    def fill_ghosts(self):
        # cfd2d/models.py:139-183
        phi, sim = self.phi, self.sim
        g = sim.grid
        nx, ny = g.nx, g.ny
        D = np.maximum(self.diff, 1e-300)

        def ghost(inner, code, val, h, Dl):
            out = inner.copy()
            m1 = code == 1
            out[m1] = 2 * val[m1] - inner[m1]
            m2 = code == 2
            out[m2] = inner[m2] + val[m2] * h / Dl[m2]
            return out

        if sim.periodic:
            phi[0, :] = phi[nx, :]
            phi[nx + 1, :] = phi[1, :]
        else:
            phi[0, 1:-1] = ghost(phi[1, 1:-1], self.bt["left"], self.bv["left"], g.dx, D[1, 1:-1])
            phi[nx + 1, 1:-1] = ghost(phi[nx, 1:-1], self.bt["right"], self.bv["right"], g.dx,
                                      D[nx, 1:-1])
        phi[1:-1, 0] = ghost(phi[1:-1, 1], self.bt["bottom"], self.bv["bottom"], g.dy, D[1:-1, 1])
        phi[1:-1, ny + 1] = ghost(phi[1:-1, ny], self.bt["top"], self.bv["top"], g.dy, D[1:-1, ny])
        solid = g.interior_solid_padded()
        if solid.any():
            fl = g.fluid.astype(float)
            pf = np.where(g.fluid, phi, 0.0)
            s = np.zeros_like(phi)
            c = np.zeros_like(phi)
            s[1:-1, 1:-1] = pf[2:, 1:-1] + pf[:-2, 1:-1] + pf[1:-1, 2:] + pf[1:-1, :-2]
            c[1:-1, 1:-1] = fl[2:, 1:-1] + fl[:-2, 1:-1] + fl[1:-1, 2:] + fl[1:-1, :-2]
            near = solid & (c > 0)
            avg = np.where(c > 0, s / np.maximum(c, 1), 0.0)
            if self.obstacle.kind == "fixed":
                phi[near] = 2 * float(self.obstacle.value) - avg[near]
                phi[solid & ~near] = float(self.obstacle.value)
            else:
                phi[near] = avg[near]

    def step(self, dt):
        # cfd2d/models.py:186-208
        sim = self.sim
        g = sim.grid
        scalar_transport(self.phi, sim.u, sim.v, g.fluid, g.nx, g.ny, g.dx, g.dy, self.diff,
                         LIMITERS[self.limiter], sim.periodic,
                         self.bt["left"], self.bv["left"], self.bt["right"], self.bv["right"],
                         self.bt["bottom"], self.bv["bottom"], self.bt["top"], self.bv["top"],
                         self.obstacle.code,
                         float(self.obstacle.value) if self.obstacle.kind == "fixed" else 0.0,
                         self.rhs)
        fl = g.fluid[1:-1, 1:-1]
        phi_i = self.phi[1:-1, 1:-1]
        new = phi_i + dt * self.rhs[1:-1, 1:-1]
        if self.source is not None:
            s_exp, s_imp = self.source(sim, self)
            new = (new + dt * s_exp) / (1.0 + dt * np.maximum(s_imp, 0.0))
        if self.lower is not None:
            new = np.maximum(new, self.lower)
        if self.upper is not None:
            new = np.minimum(new, self.upper)
        self.phi[1:-1, 1:-1] = np.where(fl, new, phi_i)
        self.fill_ghosts()

    def dt_limit(self):
        # cfd2d/models.py:210-215
        g = self.sim.grid
        dmax = float(self.diff[g.fluid].max()) if g.fluid.any() else self.D0
        if dmax <= 0:
            return np.inf
        return 0.5 / (dmax * (1.0 / g.dx ** 2 + 1.0 / g.dy ** 2))

    def total(self):
        g = self.sim.grid
        c = np.where(~g.fluid[1:-1, 1:-1], np.nan, self.phi[1:-1, 1:-1])
        return float(np.nansum(c) * g.dx * g.dy)


class OModel:
    kind = "model"

    def attach(self, sim):
        self.sim = sim

    def pre_momentum(self, sim):
        pass

    def momentum_source(self, sim, hu, hv):
        pass

    def post_step(self, sim, dt):
        pass

    def dt_limit(self, sim):
        return None


class OPassiveScalar(OModel):
    """cfd2d/models.py:296-333"""
    kind = "scalar"

    def __init__(self, name="c", diffusivity=1e-3, bcs=None, obstacle=None, limiter="vanleer",
                 initial=0.0, turbulent_schmidt=0.7):
        self.field = OScalarField(name, diffusivity, bcs, obstacle, limiter, initial)
        self.sct, self.name = turbulent_schmidt, name

    def attach(self, sim):
        super().attach(sim)
        self.field.attach(sim)
        sim.scalars[self.name] = self.field

    def post_step(self, sim, dt):
        if sim.variable_viscosity:
            self.field.diff[:] = self.field.D0 + sim.nu_t / self.sct
        self.field.step(dt)

    def dt_limit(self, sim):
        lim = self.field.dt_limit()
        return lim if np.isfinite(lim) else None

    def fields(self, sim):
        # cfd2d/models.py:332-333 with ScalarField.cell (models.py:217-219)
        return {self.name: ("Skalar " + self.name,
                            np.where(~sim.grid.fluid[1:-1, 1:-1], np.nan, self.field.phi[1:-1, 1:-1]))}


class OBoussinesq(OModel):
    """cfd2d/models.py:339-426"""
    kind = "thermal"

    def __init__(self, alpha, bcs=None, gravity=(0.0, -1.0), T_ref=0.0, initial=0.0,
                 obstacle=None, limiter="vanleer", prandtl_turbulent=0.85, buoyancy=True):
        self.field = OScalarField("T", alpha, bcs, obstacle, limiter, initial)
        self.alpha = float(alpha)
        self.gravity = (float(gravity[0]), float(gravity[1]))
        self.T_ref, self.prt, self.buoyancy = float(T_ref), prandtl_turbulent, buoyancy

    def attach(self, sim):
        super().attach(sim)
        self.field.attach(sim)
        sim.scalars["T"] = self.field

    def momentum_source(self, sim, hu, hv):
        # cfd2d/models.py:386-396
        if not self.buoyancy:
            return
        T = self.field.phi
        gx, gy = self.gravity
        if gx:
            Tf = 0.5 * (T[:-1, :] + T[1:, :]) - self.T_ref
            hu[sim.u_fluid] += -gx * Tf[sim.u_fluid]
        if gy:
            Tf = 0.5 * (T[:, :-1] + T[:, 1:]) - self.T_ref
            hv[sim.v_fluid] += -gy * Tf[sim.v_fluid]

    def post_step(self, sim, dt):
        if sim.variable_viscosity:
            self.field.diff[:] = self.alpha + sim.nu_t / self.prt
        self.field.step(dt)

    def dt_limit(self, sim):
        lim = self.field.dt_limit()
        return lim if np.isfinite(lim) else None

    def nusselt(self, side, L=1.0, dT=1.0):
        f = self.field
        g = self.sim.grid
        code, val = f.bt[side], f.bv[side]
        if not np.any(code == 1):
            return None
        if side == "left":
            inner, D, h = f.phi[1, 1:-1], f.diff[1, 1:-1], g.dx
        elif side == "right":
            inner, D, h = f.phi[g.nx, 1:-1], f.diff[g.nx, 1:-1], g.dx
        elif side == "bottom":
            inner, D, h = f.phi[1:-1, 1], f.diff[1:-1, 1], g.dy
        else:
            inner, D, h = f.phi[1:-1, g.ny], f.diff[1:-1, g.ny], g.dy
        q = np.zeros_like(inner)
        m = code == 1
        q[m] = -D[m] * (val[m] - inner[m]) / (0.5 * h)
        m2 = code == 2
        q[m2] = -val[m2]
        return abs(float(np.mean(q))) * L / (self.alpha * dT)


def _wall_mask(sim):
    # cfd2d/turbulence.py:28-40
    wall = sim.grid.interior_solid_padded()
    if sim.bcs["left"].kind == "noslip":
        wall[0, :] = True
    if sim.bcs["right"].kind == "noslip":
        wall[-1, :] = True
    if sim.bcs["bottom"].kind == "noslip":
        wall[:, 0] = True
    if sim.bcs["top"].kind == "noslip":
        wall[:, -1] = True
    return wall


def wall_distance(sim):
    # cfd2d/turbulence.py:43-70 (exact Euclidean distance transform, scipy.ndimage)
    g = sim.grid
    wall = _wall_mask(sim)
    if not wall.any():
        return np.full(wall.shape, 1e6)
    if sim.periodic:
        core = wall[1:-1, :]
        tiled = np.concatenate([core, core, core], axis=0)
        d = ndimage.distance_transform_edt(~tiled, sampling=(g.dx, g.dy))
        n = core.shape[0]
        dc = d[n:2 * n, :]
        dist = np.empty(wall.shape)
        dist[1:-1, :] = dc
        dist[0, :] = dc[-1, :]
        dist[-1, :] = dc[0, :]
    else:
        dist = ndimage.distance_transform_edt(~wall, sampling=(g.dx, g.dy))
    half = 0.5 * min(g.dx, g.dy)
    dist = np.maximum(dist - half, 0.5 * min(g.dx, g.dy))
    dist[~g.fluid] = 0.0
    return dist


def wall_adjacent_cells(sim):
    # cfd2d/turbulence.py:73-86
    g = sim.grid
    wall = _wall_mask(sim)
    fl = g.fluid
    adj = np.zeros_like(fl)
    dist = np.full(fl.shape, np.inf)
    inner = (slice(1, -1), slice(1, -1))
    for sl, h in (((slice(2, None), slice(1, -1)), g.dx), ((slice(0, -2), slice(1, -1)), g.dx),
                  ((slice(1, -1), slice(2, None)), g.dy), ((slice(1, -1), slice(0, -2)), g.dy)):
        nb = wall[sl] & fl[inner]
        adj[inner] |= nb
        dist[inner] = np.where(nb, np.minimum(dist[inner], 0.5 * h), dist[inner])
    return adj, dist


def strain_rate_squared(sim):
    # cfd2d/turbulence.py:89-100
    g = sim.grid
    u, v = sim.u, sim.v
    dudx = (u[1:, 1:-1] - u[:-1, 1:-1]) / g.dx
    dvdy = (v[1:-1, 1:] - v[1:-1, :-1]) / g.dy
    dudy = (u[:, 1:] - u[:, :-1]) / g.dy
    dvdx = (v[1:, :] - v[:-1, :]) / g.dx
    sh = dudy + dvdx
    sh2 = 0.25 * (sh[:-1, :-1] ** 2 + sh[1:, :-1] ** 2 + sh[:-1, 1:] ** 2 + sh[1:, 1:] ** 2)
    return 2.0 * (dudx ** 2 + dvdy ** 2) + sh2


def _grad(phi, dx, dy):
    # cfd2d/turbulence.py:103-107
    return ((phi[2:, 1:-1] - phi[:-2, 1:-1]) / (2 * dx),
            (phi[1:-1, 2:] - phi[1:-1, :-2]) / (2 * dy))


def _set_nut_ghosts(sim, nut):
    # cfd2d/turbulence.py:110-124
    g = sim.grid
    nx, ny = g.nx, g.ny
    nut[~g.fluid] = 0.0
    if sim.periodic:
        nut[0, :] = nut[nx, :]
        nut[nx + 1, :] = nut[1, :]
    else:
        nut[0, :] = 0.0 if sim.bcs["left"].kind == "noslip" else nut[1, :]
        nut[nx + 1, :] = 0.0 if sim.bcs["right"].kind == "noslip" else nut[nx, :]
    nut[:, 0] = 0.0 if sim.bcs["bottom"].kind == "noslip" else nut[:, 1]
    nut[:, ny + 1] = 0.0 if sim.bcs["top"].kind == "noslip" else nut[:, ny]
    nut[g.interior_solid_padded()] = 0.0


class OSmagorinsky(OModel):
    """LES Smagorinsky, nu_t = l^2 |S| with l = min(C_s sqrt(dx dy), kappa d)
    (cfd2d/turbulence.py:130-160)."""
    kind = "turbulence"

    def __init__(self, cs=0.17, wall_damping=True):
        self.cs, self.wall_damping = float(cs), wall_damping

    def attach(self, sim):
        # cfd2d/turbulence.py:137-147: the squared length is fixed at attach time
        super().attach(sim)
        sim.variable_viscosity = True
        g = sim.grid
        length = np.full((g.nx, g.ny), self.cs * np.sqrt(g.dx * g.dy))
        if self.wall_damping:
            length = np.minimum(length, KAPPA * wall_distance(sim)[1:-1, 1:-1])
        self.l2 = length ** 2
        self.pre_momentum(sim)

    def pre_momentum(self, sim):
        # cfd2d/turbulence.py:149-152
        rate = np.sqrt(strain_rate_squared(sim))
        sim.nu_t[1:-1, 1:-1] = np.where(sim.grid.fluid[1:-1, 1:-1], self.l2 * rate, 0.0)
        _set_nut_ghosts(sim, sim.nu_t)


class OKOmegaSST(OModel):
    """k-omega SST, low-Re form (cfd2d/turbulence.py:166-325)."""
    kind = "turbulence"
    a1, beta_star = 0.31, 0.09
    sk1, so1, beta1, gamma1 = 0.85, 0.5, 0.075, 5.0 / 9.0
    sk2, so2, beta2, gamma2 = 1.0, 0.856, 0.0828, 0.44

    def __init__(self, intensity=0.05, viscosity_ratio=10.0, U_ref=1.0, limiter="upwind"):
        self.I, self.ratio, self.U_ref, self.limiter = float(intensity), float(viscosity_ratio), \
            float(U_ref), limiter

    def attach(self, sim):
        super().attach(sim)
        sim.variable_viscosity = True
        nu = sim.nu
        k0 = 1.5 * (self.I * self.U_ref) ** 2
        w0 = k0 / (nu * self.ratio)
        kb, wb = {}, {}
        for side in SIDES:
            kind = sim.bcs[side].kind
            if kind == "inflow":
                kb[side], wb[side] = OScalarBC("fixed", k0), OScalarBC("fixed", w0)
            elif kind == "noslip":
                kb[side], wb[side] = OScalarBC("fixed", 0.0), OScalarBC("zerogradient")
            else:
                kb[side], wb[side] = OScalarBC("zerogradient"), OScalarBC("zerogradient")
        self.k = OScalarField("k", nu, kb, OScalarBC("fixed", 0.0), self.limiter, k0,
                              source=self._k_source, lower=1e-14)
        self.w = OScalarField("omega", nu, wb, OScalarBC("zerogradient"), self.limiter, w0,
                              source=self._w_source, lower=1e-8)
        self.k.attach(sim)
        self.w.attach(sim)
        sim.scalars["k"] = self.k
        sim.scalars["omega"] = self.w
        self.d = np.maximum(wall_distance(sim)[1:-1, 1:-1], 1e-12)
        adj, dist = wall_adjacent_cells(sim)
        self.wall_adj = adj[1:-1, 1:-1]
        self.w_wall = np.where(self.wall_adj, 6.0 * nu / (self.beta1 * np.where(
            np.isfinite(dist[1:-1, 1:-1]), dist[1:-1, 1:-1], 1.0) ** 2), 0.0)
        self.apply_wall_omega()
        self.F1 = np.ones((sim.grid.nx, sim.grid.ny))
        self.pre_momentum(sim)

    def apply_wall_omega(self):
        w = self.w.phi[1:-1, 1:-1]
        w[self.wall_adj] = self.w_wall[self.wall_adj]
        self.w.fill_ghosts()

    def _blending(self, sim):
        # cfd2d/turbulence.py:244-260
        g = sim.grid
        nu = sim.nu
        k = np.maximum(self.k.phi[1:-1, 1:-1], 0.0)
        w = np.maximum(self.w.phi[1:-1, 1:-1], 1e-12)
        d = self.d
        dkx, dky = _grad(self.k.phi, g.dx, g.dy)
        dwx, dwy = _grad(self.w.phi, g.dx, g.dy)
        cross = dkx * dwx + dky * dwy
        CD = np.maximum(2.0 * self.so2 / w * cross, 1e-10)
        sk = np.sqrt(k)
        arg1 = np.minimum(np.maximum(sk / (self.beta_star * w * d), 500 * nu / (d ** 2 * w)),
                          4 * self.so2 * k / (CD * d ** 2))
        F1 = np.tanh(arg1 ** 4)
        arg2 = np.maximum(2 * sk / (self.beta_star * w * d), 500 * nu / (d ** 2 * w))
        F2 = np.tanh(arg2 ** 2)
        return F1, F2, cross

    def pre_momentum(self, sim):
        # cfd2d/turbulence.py:262-282
        k = np.maximum(self.k.phi[1:-1, 1:-1], 0.0)
        w = np.maximum(self.w.phi[1:-1, 1:-1], 1e-12)
        S2 = strain_rate_squared(sim)
        self.S2 = S2
        F1, F2, cross = self._blending(sim)
        self.F1, self.F2, self.cross = F1, F2, cross
        nut = self.a1 * k / np.maximum(self.a1 * w, np.sqrt(S2) * F2)
        sim.nu_t[1:-1, 1:-1] = np.where(sim.grid.fluid[1:-1, 1:-1], nut, 0.0)
        _set_nut_ghosts(sim, sim.nu_t)
        sk = F1 * self.sk1 + (1 - F1) * self.sk2
        so = F1 * self.so1 + (1 - F1) * self.so2
        self.k.diff[1:-1, 1:-1] = sim.nu + sk * nut
        self.w.diff[1:-1, 1:-1] = sim.nu + so * nut
        for f in (self.k, self.w):
            f.diff[0, :] = f.diff[1, :]
            f.diff[-1, :] = f.diff[-2, :]
            f.diff[:, 0] = f.diff[:, 1]
            f.diff[:, -1] = f.diff[:, -2]

    def _k_source(self, sim, field):
        # cfd2d/turbulence.py:285-291
        k = np.maximum(self.k.phi[1:-1, 1:-1], 0.0)
        w = np.maximum(self.w.phi[1:-1, 1:-1], 1e-12)
        nut = sim.nu_t[1:-1, 1:-1]
        Pk = np.minimum(nut * self.S2, 10.0 * self.beta_star * k * w)
        self._Pk = Pk
        return Pk, self.beta_star * w

    def _w_source(self, sim, field):
        # cfd2d/turbulence.py:293-304
        F1 = self.F1
        w = np.maximum(self.w.phi[1:-1, 1:-1], 1e-12)
        gamma = F1 * self.gamma1 + (1 - F1) * self.gamma2
        beta = F1 * self.beta1 + (1 - F1) * self.beta2
        nut = np.maximum(sim.nu_t[1:-1, 1:-1], 1e-14)
        Pw = gamma * self._Pk / nut
        Pw = np.where(sim.nu_t[1:-1, 1:-1] > 1e-14, Pw, gamma * self.S2)
        CDw = 2.0 * (1 - F1) * self.so2 / w * self.cross
        return Pw + np.maximum(CDw, 0.0), beta * w + np.maximum(-CDw, 0.0) / w

    def post_step(self, sim, dt):
        # cfd2d/turbulence.py:306-311
        self.S2 = strain_rate_squared(sim)
        self.k.step(dt)
        self.w.step(dt)
        self.apply_wall_omega()

    def dt_limit(self, sim):
        return min(self.k.dt_limit(), self.w.dt_limit())


# --------------------------------------------------------------------------- #
# Time integrator (cfd2d/solver.py:95-567)
# --------------------------------------------------------------------------- #
class OSimulation:
    """Chorin projection step on the MAC grid (cfd2d/solver.py:58-567)."""

    def __init__(self, grid, bcs, nu, scheme="ab2", gamma="auto", tau=0.5, dt=None,
                 pressure_solver="direct", compute_forces=False, initial_velocity=(0.0, 0.0),
                 models=None, body_force=(0.0, 0.0), flow_rate=None, tol=None):
        if nu <= 0:
            raise ValueError("viscosity must be positive")
        self.removed_cells = grid.finalize()
        self.grid = g = grid
        self.nu, self.scheme, self.gamma_setting = float(nu), scheme, gamma
        self.tau, self.dt_fixed, self.compute_forces = float(tau), dt, compute_forces
        nx, ny = g.nx, g.ny
        self.boundary = OBoundary(g, bcs)
        self.bcs = bcs
        self.pressure = OPressure(g, self.boundary, pressure_solver)
        self.u = np.zeros((nx + 1, ny + 2))
        self.v = np.zeros((nx + 2, ny + 1))
        self.p = np.zeros((nx + 2, ny + 2))
        self.F = np.zeros_like(self.u)
        self.G = np.zeros_like(self.v)
        self.hu = np.zeros_like(self.u)
        self.hv = np.zeros_like(self.v)
        self.hu_old = self.hv_old = self.dt_old = None
        self.u_fluid = g.u_fluid_faces()
        self.v_fluid = g.v_fluid_faces()
        self.periodic = self.boundary.periodic
        if self.periodic:
            self.u_fluid[0, :] = False
        self.nu_t = np.zeros((nx + 2, ny + 2))
        self.nu_eff = np.full((nx + 2, ny + 2), self.nu)
        self.variable_viscosity = False
        self.variable_density = False
        self.rho = np.ones((nx + 2, ny + 2))
        self.body_force = (float(body_force[0]), float(body_force[1]))
        self.flow_rate = flow_rate
        self.flow_force = 0.0
        self.scalars = {}
        self.models = []
        for m in models or []:
            self.add_model(m)
        u0, v0 = initial_velocity
        if u0:
            self.u[self.u_fluid] = u0
        if v0:
            self.v[self.v_fluid] = v0
        self.t, self.n, self.dt = 0.0, 0, 0.0
        self.gamma = 0.0 if gamma == "auto" else float(gamma)
        self.residual = np.inf
        self.iterations = []
        self.hist = {"dt": [], "residual": [], "divergence": [], "kinetic_energy": [],
                     "fx": [], "fy": [], "flow_force": []}
        self.apply_bc()
        self.project_initial()
        # the reference's Simulation takes no tolerance: callers set sim.pressure.tol after
        # construction, so the initial projection above runs at the default 1e-10
        if tol is not None:
            self.pressure.tol = tol
        self.iterations = []  # CG iterations per step (the initial projection not counted)

    def add_model(self, m):
        m.attach(self)
        self.models.append(m)

    def model(self, kind):
        for m in self.models:
            if getattr(m, "kind", None) == kind:
                return m
        return None

    def apply_bc(self):
        # cfd2d/solver.py:189-193
        self.boundary.apply(self.u, self.v)
        obstacle_bc(self.u, self.v, self.grid.fluid, self.grid.nx, self.grid.ny, self.periodic)

    def project_initial(self):
        # cfd2d/solver.py:195-204
        if not (np.any(self.u) or np.any(self.v)):
            return
        self.F[:] = self.u
        self.G[:] = self.v
        self.boundary.extrapolate_outflow_predictor(self.F, self.G)
        self.solve_pressure_and_correct(1.0)
        self.p[:] = 0.0
        self.apply_bc()

    def compute_dt(self):
        # cfd2d/solver.py:209-231
        if self.dt_fixed:
            return float(self.dt_fixed)
        g = self.grid
        umax = max(np.abs(self.u).max(), 1e-12)
        vmax = max(np.abs(self.v).max(), 1e-12)
        if self.variable_density:
            nu_max = float((self.nu_eff / self.rho)[g.fluid].max())
        else:
            nu_max = float(self.nu_eff.max()) if self.variable_viscosity else self.nu
        dt_visc = 0.5 / (nu_max * (1.0 / g.dx ** 2 + 1.0 / g.dy ** 2))
        dt_conv = min(g.dx / umax, g.dy / vmax)
        if self.scheme == "ab2":
            dt_visc *= 0.5
            dt_conv *= 0.8
        dt = self.tau * min(dt_visc, dt_conv)
        for m in self.models:
            lim = m.dt_limit(self)
            if lim is not None:
                dt = min(dt, self.tau * lim)
        return dt

    def auto_gamma(self, dt):
        # cfd2d/solver.py:233-253
        g = self.grid
        umax = np.abs(self.u).max()
        vmax = np.abs(self.v).max()
        if self.scheme == "euler":
            cfl = max(umax * dt / g.dx, vmax * dt / g.dy)
            return float(min(1.0, max(0.05, 1.2 * cfl)))
        if self.variable_density:
            nu_ref = float((self.nu_eff / self.rho)[g.fluid].min())
        else:
            nu_ref = float(self.nu_eff[g.fluid].min()) if self.variable_viscosity else self.nu
        re_cell = max(umax * g.dx, vmax * g.dy) / nu_ref
        return float(min(1.0, max(0.05, 0.015 * re_cell)))

    def solve_pressure_and_correct(self, dt):
        # cfd2d/solver.py:258-321; with variable density the face coefficients
        # b = 2 / (rho_L + rho_R) scale the operator and the correction
        g = self.grid
        nx, ny, dx, dy = g.nx, g.ny, g.dx, g.dy
        F, G = self.F, self.G
        if self.periodic:
            F[0, :] = F[nx, :]
        div = (F[1:, 1:-1] - F[:-1, 1:-1]) / dx + (G[1:-1, 1:] - G[1:-1, :-1]) / dy
        if self.variable_density:
            bx = 2.0 / (self.rho[:-1, :] + self.rho[1:, :])
            by = 2.0 / (self.rho[:, :-1] + self.rho[:, 1:])
            if self.periodic:
                bx[nx, :] = 2.0 / (self.rho[nx, :] + self.rho[1, :])
            p_int = self.pressure.solve_variable(div / dt, bx[:, 1:-1], by[1:-1, :])
            self._solve_correct_variable(dt, p_int, bx, by)
            return
        p_int = self.pressure.solve(div / dt)
        self.iterations.append(self.pressure.last_iterations)
        p = self.p
        p[:] = 0.0
        p[1:-1, 1:-1] = p_int
        if self.periodic:
            p[0, :] = p[nx, :]
            p[nx + 1, :] = p[1, :]
        uf = self.u_fluid[1:nx, 1:ny + 1]
        corr = F[1:nx, 1:ny + 1] - dt * 1.0 * (p[2:nx + 1, 1:ny + 1] - p[1:nx, 1:ny + 1]) / dx
        self.u[1:nx, 1:ny + 1] = np.where(uf, corr, F[1:nx, 1:ny + 1])
        vf = self.v_fluid[1:nx + 1, 1:ny]
        corr = G[1:nx + 1, 1:ny] - dt * 1.0 * (p[1:nx + 1, 2:ny + 1] - p[1:nx + 1, 1:ny]) / dy
        self.v[1:nx + 1, 1:ny] = np.where(vf, corr, G[1:nx + 1, 1:ny])
        if self.periodic:
            uf = self.u_fluid[nx, 1:ny + 1]
            corr = F[nx, 1:ny + 1] - dt * 1.0 * (p[1, 1:ny + 1] - p[nx, 1:ny + 1]) / dx
            self.u[nx, 1:ny + 1] = np.where(uf, corr, F[nx, 1:ny + 1])
            self.u[0, :] = self.u[nx, :]
            return
        d = self.pressure.dirichlet
        self.u[0, 1:ny + 1] = np.where(d["left"], F[0, 1:ny + 1] - 2 * dt * 1.0 * p[1, 1:ny + 1] / dx,
                                       F[0, 1:ny + 1])
        self.u[nx, 1:ny + 1] = np.where(d["right"], F[nx, 1:ny + 1] + 2 * dt * 1.0 * p[nx, 1:ny + 1] / dx,
                                        F[nx, 1:ny + 1])
        self.v[1:nx + 1, 0] = np.where(d["bottom"], G[1:nx + 1, 0] - 2 * dt * 1.0 * p[1:nx + 1, 1] / dy,
                                       G[1:nx + 1, 0])
        self.v[1:nx + 1, ny] = np.where(d["top"], G[1:nx + 1, ny] + 2 * dt * 1.0 * p[1:nx + 1, ny] / dy,
                                        G[1:nx + 1, ny])

    def _solve_correct_variable(self, dt, p_int, bx, by):
        # cfd2d/solver.py:274-321 with cx = bx, cy = by
        g = self.grid
        nx, ny, dx, dy = g.nx, g.ny, g.dx, g.dy
        F, G = self.F, self.G
        self.iterations.append(1)
        p = self.p
        p[:] = 0.0
        p[1:-1, 1:-1] = p_int
        if self.periodic:
            p[0, :] = p[nx, :]
            p[nx + 1, :] = p[1, :]
        uf = self.u_fluid[1:nx, 1:ny + 1]
        corr = F[1:nx, 1:ny + 1] - dt * bx[1:nx, 1:ny + 1] * (p[2:nx + 1, 1:ny + 1] - p[1:nx, 1:ny + 1]) / dx
        self.u[1:nx, 1:ny + 1] = np.where(uf, corr, F[1:nx, 1:ny + 1])
        vf = self.v_fluid[1:nx + 1, 1:ny]
        corr = G[1:nx + 1, 1:ny] - dt * by[1:nx + 1, 1:ny] * (p[1:nx + 1, 2:ny + 1] - p[1:nx + 1, 1:ny]) / dy
        self.v[1:nx + 1, 1:ny] = np.where(vf, corr, G[1:nx + 1, 1:ny])
        if self.periodic:
            uf = self.u_fluid[nx, 1:ny + 1]
            corr = F[nx, 1:ny + 1] - dt * bx[nx, 1:ny + 1] * (p[1, 1:ny + 1] - p[nx, 1:ny + 1]) / dx
            self.u[nx, 1:ny + 1] = np.where(uf, corr, F[nx, 1:ny + 1])
            self.u[0, :] = self.u[nx, :]
            return
        d = self.pressure.dirichlet
        self.u[0, 1:ny + 1] = np.where(d["left"], F[0, 1:ny + 1] - 2 * dt * bx[0, 1:ny + 1] * p[1, 1:ny + 1] / dx,
                                       F[0, 1:ny + 1])
        self.u[nx, 1:ny + 1] = np.where(d["right"],
                                        F[nx, 1:ny + 1] + 2 * dt * bx[nx, 1:ny + 1] * p[nx, 1:ny + 1] / dx,
                                        F[nx, 1:ny + 1])
        self.v[1:nx + 1, 0] = np.where(d["bottom"], G[1:nx + 1, 0] - 2 * dt * by[1:nx + 1, 0] * p[1:nx + 1, 1] / dy,
                                       G[1:nx + 1, 0])
        self.v[1:nx + 1, ny] = np.where(d["top"],
                                        G[1:nx + 1, ny] + 2 * dt * by[1:nx + 1, ny] * p[1:nx + 1, ny] / dy,
                                        G[1:nx + 1, ny])

    def step(self):
        # cfd2d/solver.py:326-403
        g = self.grid
        self.apply_bc()
        for m in self.models:
            m.pre_momentum(self)
        if self.variable_viscosity and not self.variable_density:
            np.add(self.nu, self.nu_t, out=self.nu_eff)
        dt = self.compute_dt()
        self.gamma = self.auto_gamma(dt) if self.gamma_setting == "auto" else float(self.gamma_setting)
        momentum_tendencies(self.u, self.v, g.fluid, g.nx, g.ny, g.dx, g.dy, self.nu_eff,
                            self.variable_viscosity, self.gamma, self.periodic, self.hu, self.hv,
                            self.rho, self.variable_density)
        for m in self.models:
            m.momentum_source(self, self.hu, self.hv)
        if self.scheme == "ab2" and self.hu_old is not None:
            r = dt / self.dt_old
            a, b = 1.0 + 0.5 * r, -0.5 * r
            Hu = a * self.hu + b * self.hu_old
            Hv = a * self.hv + b * self.hv_old
        else:
            Hu, Hv = self.hu, self.hv
        u_prev = self.u.copy()
        v_prev = self.v.copy()
        self.F[:] = self.u
        self.G[:] = self.v
        self.F[self.u_fluid] += dt * Hu[self.u_fluid]
        self.G[self.v_fluid] += dt * Hv[self.v_fluid]
        fx = self.body_force[0] + self.flow_force
        fy = self.body_force[1]
        if fx:
            self.F[self.u_fluid] += dt * fx
        if fy:
            self.G[self.v_fluid] += dt * fy
        self.boundary.extrapolate_outflow_predictor(self.F, self.G)
        self.solve_pressure_and_correct(dt)
        self.apply_bc()
        if self.flow_rate is not None:
            self.control_flow_rate(dt)
        for m in self.models:
            m.post_step(self, dt)
        if self.scheme == "ab2":
            self.hu_old = self.hu.copy()
            self.hv_old = self.hv.copy()
        self.dt_old = dt
        self.t += dt
        self.n += 1
        self.dt = dt
        du = np.abs(self.u[self.u_fluid] - u_prev[self.u_fluid]).max(initial=0.0)
        dv = np.abs(self.v[self.v_fluid] - v_prev[self.v_fluid]).max(initial=0.0)
        self.residual = max(du, dv) / dt
        if not np.isfinite(self.residual) or self.residual > 1e8:
            raise FloatingPointError(f"unstable at step {self.n}")
        h = self.hist
        h["dt"].append(dt)
        h["residual"].append(self.residual)
        h["divergence"].append(self.max_divergence())
        h["kinetic_energy"].append(self.kinetic_energy())
        if self.compute_forces:
            fxo, fyo = self.obstacle_forces()
            h["fx"].append(fxo)
            h["fy"].append(fyo)
        if self.flow_rate is not None:
            h["flow_force"].append(self.flow_force)

    def bulk_velocity(self):
        m = self.u_fluid[1:self.grid.nx + 1, 1:-1]
        return float(self.u[1:self.grid.nx + 1, 1:-1][m].mean())

    def control_flow_rate(self, dt):
        # cfd2d/solver.py:410-425
        du = self.flow_rate - self.bulk_velocity()
        self.u[self.u_fluid] += du
        if self.periodic:
            self.u[0, :] = self.u[self.grid.nx, :]
        self.flow_force += du / dt
        if (~self.grid.fluid[1:-1, 1:-1]).any():
            self.F[:] = self.u
            self.G[:] = self.v
            self.boundary.extrapolate_outflow_predictor(self.F, self.G)
            p_save = self.p.copy()
            self.solve_pressure_and_correct(1.0)
            self.p[:] = p_save
        self.apply_bc()

    def divergence(self):
        g = self.grid
        div = ((self.u[1:, 1:-1] - self.u[:-1, 1:-1]) / g.dx
               + (self.v[1:-1, 1:] - self.v[1:-1, :-1]) / g.dy)
        return np.where(g.fluid[1:-1, 1:-1], div, 0.0)

    def max_divergence(self):
        return float(np.abs(self.divergence()).max())

    def kinetic_energy(self):
        # cfd2d/solver.py:522-536
        uc = 0.5 * (self.u[:-1, 1:-1] + self.u[1:, 1:-1])
        vc = 0.5 * (self.v[1:-1, :-1] + self.v[1:-1, 1:])
        solid = ~self.grid.fluid[1:-1, 1:-1]
        uc = np.where(solid, np.nan, uc)
        vc = np.where(solid, np.nan, vc)
        return float(0.5 * np.nansum(uc ** 2 + vc ** 2) * self.grid.dx * self.grid.dy)

    def obstacle_forces(self):
        # cfd2d/solver.py:542-567
        g = self.grid
        solid = g.interior_solid_padded()
        f = g.fluid[1:-1, 1:-1]
        east = f & solid[2:, 1:-1]
        west = f & solid[:-2, 1:-1]
        north = f & solid[1:-1, 2:]
        south = f & solid[1:-1, :-2]
        p = self.p[1:-1, 1:-1]
        uc = 0.5 * (self.u[:-1, 1:-1] + self.u[1:, 1:-1])
        vc = 0.5 * (self.v[1:-1, :-1] + self.v[1:-1, 1:])
        mu = self.nu
        fx = (p[east].sum() - p[west].sum()) * g.dy
        fy = (p[north].sum() - p[south].sum()) * g.dx
        fx += mu * (uc[north].sum() + uc[south].sum()) / (0.5 * g.dy) * g.dx
        fy += mu * (vc[east].sum() + vc[west].sum()) / (0.5 * g.dx) * g.dy
        return float(fx), float(fy)


# --------------------------------------------------------------------------- #
# Case builders for the measured configurations (cfd2d/cases.py:60-379)
# --------------------------------------------------------------------------- #
def cavity(re=100.0, n=64, scheme="ab2", gamma="auto", tau=0.5, pressure_solver="cg", tol=1e-8):
    # cfd2d/cases.py:60-70
    g = OGrid(n, n, 1.0, 1.0)
    bcs = {"left": OBC("noslip"), "right": OBC("noslip"), "bottom": OBC("noslip"),
           "top": OBC("noslip", velocity=1.0)}
    return OSimulation(g, bcs, nu=1.0 / re, scheme=scheme, gamma=gamma, tau=tau,
                       pressure_solver=pressure_solver, tol=tol)


def cylinder(re=100.0, nx=440, ny=82, profile="parabolic", length=2.2, pressure_solver="cg",
             tol=1e-8, **num):
    # cfd2d/cases.py:84-104
    H, D, xc, yc = 0.41, 0.1, 0.2, 0.2
    g = OGrid(nx, ny, length, H)
    g.add_obstacle(circle_mask(g, xc, yc, D / 2))
    bcs = {"left": OBC("inflow", 1.0, profile), "right": OBC("outflow"),
           "bottom": OBC("noslip"), "top": OBC("noslip")}
    return OSimulation(g, bcs, nu=1.0 * D / re, compute_forces=True, pressure_solver=pressure_solver,
                       tol=tol, **num)


def add_scalar(sim, name="c", diffusivity=1e-3, inflow_value=1.0, inflow_band=None,
               obstacle_value=None, limiter="vanleer"):
    # cfd2d/cases.py:359-379
    bcs = default_scalar_bcs(sim, 0.0)
    for side, bc in bcs.items():
        if bc.kind == "fixed":
            if inflow_band is None:
                bc.value = inflow_value
            else:
                a, b = inflow_band
                bc.value = (lambda s, a=a, b=b: np.where((s >= a) & (s <= b), inflow_value, 0.0))
    obs = OScalarBC("fixed", obstacle_value) if obstacle_value is not None else None
    m = OPassiveScalar(name, diffusivity, bcs, obs, limiter)
    sim.add_model(m)
    return m


def custom_obstacles(obstacles, lx=4.0, ly=1.0, nx=320, ny=80, re=100.0, U=1.0, L_ref=None,
                     inflow_profile="uniform", walls="slip", flow_rate=None, pressure_solver="cg",
                     tol=1e-8, **num):
    # cfd2d/cases.py:161-201
    g = OGrid(nx, ny, lx, ly)
    for spec in obstacles:
        g.add_obstacle(obstacle_mask(g, spec))
    if L_ref is None:
        solid = ~g.fluid[1:-1, 1:-1]
        L_ref = solid.any(axis=0).sum() * g.dy if solid.any() else ly
    bcs = {"left": OBC("inflow", U, inflow_profile), "right": OBC("outflow"),
           "bottom": OBC(walls), "top": OBC(walls)}
    return OSimulation(g, bcs, nu=U * L_ref / re, compute_forces=bool(obstacles),
                       flow_rate=flow_rate,
                       initial_velocity=(U, 0.0) if flow_rate is not None else (0.0, 0.0),
                       pressure_solver=pressure_solver, tol=tol, **num)


def heated_cavity(ra=1e4, pr=0.71, n=48, limiter="vanleer", pressure_solver="cg", tol=1e-8, **num):
    # cfd2d/cases.py:207-223
    g = OGrid(n, n, 1.0, 1.0)
    bcs = {s: OBC("noslip") for s in SIDES}
    th = OBoussinesq(alpha=1.0 / np.sqrt(ra * pr), limiter=limiter,
                     bcs={"left": OScalarBC("fixed", 0.5), "right": OScalarBC("fixed", -0.5),
                          "bottom": OScalarBC("zerogradient"), "top": OScalarBC("zerogradient")})
    return OSimulation(g, bcs, nu=np.sqrt(pr / ra), models=[th], pressure_solver=pressure_solver,
                       tol=tol, **num)


def sst_channel(nx=128, ny=192, lx=2 * np.pi, ly=2.0, re_b=1e4, seed=0, noise=0.05,
                pressure_solver="cg", tol=1e-8, **num):
    """Periodic channel with k-omega SST held at bulk velocity 1 (volume-flow forcing).

    Laminar parabola u = 1.5 y (2 - y) plus seeded uniform +-noise, re-projected by
    the reference's initial projection; k = 1e-3 and omega = 10 through
    intensity = sqrt(1e-3 / 1.5), viscosity_ratio = k0 / (nu omega0).
    """
    g = OGrid(nx, ny, lx, ly)
    bcs = {"left": OBC("periodic"), "right": OBC("periodic"), "bottom": OBC("noslip"),
           "top": OBC("noslip")}
    nu = 2.0 / re_b
    k0, w0 = 1e-3, 10.0
    sst = OKOmegaSST(intensity=np.sqrt(k0 / 1.5), viscosity_ratio=k0 / (nu * w0), U_ref=1.0)
    sim = OSimulation(g, bcs, nu=nu, flow_rate=1.0, models=[sst], pressure_solver=pressure_solver,
                      tol=tol, **num)
    rng = np.random.default_rng(seed)
    y = (np.arange(g.ny) + 0.5) * g.dy
    prof = 1.5 * y * (2.0 - y)
    u = sim.u
    u[1:g.nx + 1, 1:g.ny + 1] = prof[None, :] * (1.0 + noise * rng.uniform(-1.0, 1.0, (g.nx, g.ny)))
    v = sim.v
    v[1:g.nx + 1, 1:g.ny] = noise * rng.uniform(-1.0, 1.0, (g.nx, g.ny - 1))
    u[~sim.u_fluid] = 0.0
    v[~sim.v_fluid] = 0.0
    sim.apply_bc()
    sim.project_initial()
    return sim


# --------------------------------------------------------------------------- #
# Function objects, VTK export and derived fields (cfd2d/functions.py:24-287,
# cfd2d/solver.py:526-615, cfd2d/visualization.py:41-89). They take any object
# with the reference's Simulation attributes (u, v, p, grid, models, t, dt,
# nu_t, variable_viscosity).
# --------------------------------------------------------------------------- #
BASE_FIELDS = {"speed": "Geschwindigkeitsbetrag |u|", "vorticity": "Wirbelstärke ω", "pressure": "Druck p",
               "u": "Geschwindigkeit u (x-Richtung)", "v": "Geschwindigkeit v (y-Richtung)",
               "streamfunction": "Stromfunktion ψ"}


def _solid(sim):
    return ~sim.grid.fluid[1:-1, 1:-1]


def cell_velocity(sim):
    # cfd2d/solver.py:526-533
    uc = 0.5 * (sim.u[:-1, 1:-1] + sim.u[1:, 1:-1])
    vc = 0.5 * (sim.v[1:-1, :-1] + sim.v[1:-1, 1:])
    return np.where(_solid(sim), np.nan, uc), np.where(_solid(sim), np.nan, vc)


def cell_pressure(sim):
    # cfd2d/solver.py:535-536
    return np.where(_solid(sim), np.nan, sim.p[1:-1, 1:-1])


def cell_vorticity(sim):
    # cfd2d/solver.py:569-578
    g = sim.grid
    w = (sim.v[1:, :] - sim.v[:-1, :]) / g.dx - (sim.u[:, 1:] - sim.u[:, :-1]) / g.dy
    wc = 0.25 * (w[:-1, :-1] + w[1:, :-1] + w[:-1, 1:] + w[1:, 1:])
    return np.where(_solid(sim), np.nan, wc)


def streamfunction(sim):
    # cfd2d/solver.py:580-596
    g = sim.grid
    fl = g.fluid
    u_open = fl[:-1, 1:-1] | fl[1:, 1:-1]
    v_open = fl[1:-1, 0] | fl[1:-1, 1]
    u = np.where(u_open, sim.u[:, 1:-1], 0.0)
    v0 = np.where(v_open, sim.v[1:-1, 0], 0.0)
    psi = np.zeros((g.nx + 1, g.ny + 1))
    psi[1:, 0] = -np.cumsum(v0) * g.dx
    psi[:, 1:] = psi[:, :1] + np.cumsum(u, axis=1) * g.dy
    return psi


def _model_fields(sim):
    out = {}
    for m in getattr(sim, "models", []):
        if hasattr(m, "fields"):
            out.update(m.fields(sim))
    return out


def available_fields(sim):
    # cfd2d/visualization.py:80-89
    out = dict(BASE_FIELDS)
    for k, (label, _) in _model_fields(sim).items():
        out[k] = label
    if (getattr(sim, "variable_viscosity", False) and not getattr(sim, "variable_density", False)
            and "nu_t" not in out):
        out["nu_t"] = "Turbulente Viskosität ν_t"
    return out


def field_data(sim, field):
    # cfd2d/visualization.py:50-73
    if field == "speed":
        uc, vc = cell_velocity(sim)
        return np.sqrt(uc ** 2 + vc ** 2)
    if field == "vorticity":
        return cell_vorticity(sim)
    if field == "pressure":
        return cell_pressure(sim)
    if field == "u":
        return cell_velocity(sim)[0]
    if field == "v":
        return cell_velocity(sim)[1]
    if field == "streamfunction":
        psi = streamfunction(sim)
        pc = 0.25 * (psi[:-1, :-1] + psi[1:, :-1] + psi[:-1, 1:] + psi[1:, 1:])
        return np.where(_solid(sim), np.nan, pc)
    mf = _model_fields(sim)
    if field in mf:
        return mf[field][1]
    if field == "nu_t" and getattr(sim, "variable_viscosity", False):
        return np.where(_solid(sim), np.nan, sim.nu_t[1:-1, 1:-1])
    raise ValueError(field)


def _rgi(xs, ys, values, x, y):
    from scipy.interpolate import RegularGridInterpolator

    f = RegularGridInterpolator((xs, ys), values, bounds_error=False, fill_value=None)
    return f(np.column_stack([np.ravel(x), np.ravel(y)]))


def sample_u(sim, x, y):
    # cfd2d/solver.py:598-606
    g = sim.grid
    return _rgi(np.arange(g.nx + 1) * g.dx, (np.arange(g.ny + 2) - 0.5) * g.dy, sim.u, x, y)


def sample_v(sim, x, y):
    # cfd2d/solver.py:608-615
    g = sim.grid
    return _rgi((np.arange(g.nx + 2) - 0.5) * g.dx, np.arange(g.ny + 1) * g.dy, sim.v, x, y)


def sample_field(sim, field, x, y):
    # cfd2d/functions.py:24-39
    x = np.atleast_1d(np.asarray(x, dtype=float))
    y = np.atleast_1d(np.asarray(y, dtype=float))
    if field == "u":
        return sample_u(sim, x, y)
    if field == "v":
        return sample_v(sim, x, y)
    g = sim.grid
    xc = (np.arange(g.nx) + 0.5) * g.dx
    yc = (np.arange(g.ny) + 0.5) * g.dy
    return _rgi(xc, yc, field_data(sim, field), np.clip(x, xc[0], xc[-1]), np.clip(y, yc[0], yc[-1]))


def line_points(p0, p1, n):
    # cfd2d/functions.py:133-137
    s = np.linspace(0, 1, n)
    x = p0[0] + s * (p1[0] - p0[0])
    y = p0[1] + s * (p1[1] - p0[1])
    return s * np.hypot(p1[0] - p0[0], p1[1] - p0[1]), x, y


class OFieldAverage:
    """cfd2d/functions.py:180-224"""

    def __init__(self, t_start=0.0):
        self.t_start, self.T, self.sum, self.sum2 = float(t_start), 0.0, None, None

    def execute(self, sim):
        if sim.t < self.t_start:
            return
        uc, vc = cell_velocity(sim)
        vals = {"u": uc, "v": vc, "p": cell_pressure(sim)}
        if self.sum is None:
            self.sum = {k: np.zeros_like(a) for k, a in vals.items()}
            self.sum2 = {k: np.zeros_like(a) for k, a in vals.items()}
        for k, a in vals.items():
            self.sum[k] += a * sim.dt
            self.sum2[k] += a * a * sim.dt
        self.T += sim.dt

    def mean(self, k):
        return self.sum[k] / max(self.T, 1e-300)

    def rms(self, k):
        m = self.mean(k)
        return np.sqrt(np.maximum(self.sum2[k] / max(self.T, 1e-300) - m * m, 0.0))


def write_vtk_bytes(sim):
    """The bytes of cfd2d/functions.py:244-287 write_vtk (legacy binary RECTILINEAR_GRID)."""
    g = sim.grid
    nx, ny = g.nx, g.ny
    out = bytearray()

    def line(s):
        out.extend((s + "\n").encode("ascii"))

    line("# vtk DataFile Version 3.0")
    line(f"cfd2d t={sim.t:.8g}")
    line("BINARY")
    line("DATASET RECTILINEAR_GRID")
    line(f"DIMENSIONS {nx + 1} {ny + 1} 1")
    line(f"X_COORDINATES {nx + 1} float")
    out.extend((np.arange(nx + 1) * g.dx).astype(">f4").tobytes())
    line("")
    line(f"Y_COORDINATES {ny + 1} float")
    out.extend((np.arange(ny + 1) * g.dy).astype(">f4").tobytes())
    line("")
    line("Z_COORDINATES 1 float")
    out.extend(np.zeros(1, ">f4").tobytes())
    line("")
    line(f"CELL_DATA {nx * ny}")
    uc, vc = cell_velocity(sim)
    vec = np.stack([np.nan_to_num(uc).T.ravel(), np.nan_to_num(vc).T.ravel(), np.zeros(nx * ny)], axis=1)
    line("VECTORS U float")
    out.extend(vec.astype(">f4").tobytes())
    line("")
    names = [k for k in available_fields(sim) if k not in ("u", "v")]
    for k in names + ["fluid"]:
        d = g.fluid[1:-1, 1:-1].astype(float) if k == "fluid" else field_data(sim, k)
        line(f"SCALARS {k.replace(' ', '_')} float 1")
        line("LOOKUP_TABLE default")
        out.extend(np.nan_to_num(d, nan=0.0).T.astype(">f4").ravel().tobytes())
        line("")
    return bytes(out)


# --------------------------------------------------------------------------- #
# Two-phase VOF (cfd2d/vof.py) and the dam break (cfd2d/cases.py:294-320).
# The advection is restated face by face in the reference's loop order (small
# grids only): every cell receives its west, east, south and north face terms in
# that order, and with periodic x the wrapped face nx reaches cell 1 last.
# --------------------------------------------------------------------------- #
def _vof_face_value(a_up, a_c, a_d, has_up):
    # cfd2d/vof.py:23-33: van Leer face value, first order without an upwind cell
    if not has_up:
        return a_c
    den = a_d - a_c
    if abs(den) < 1e-300:
        return a_c
    r = (a_c - a_up) / den
    lim = 0.0 if r <= 0.0 else 2.0 * r / (1.0 + r)
    return a_c + 0.5 * lim * den


def _vof_face_flux(vel, a_lo, a_hi, a_up, has_up, g_n, g_t, c_alpha):
    """Flux through one face from its low to its high cell: upwind-bounded
    advection plus the compression term (cfd2d/vof.py:72-88, 113-124)."""
    if vel >= 0.0:
        af = _vof_face_value(a_up, a_lo, a_hi, has_up)
    else:
        af = _vof_face_value(a_up, a_hi, a_lo, has_up)
    flux = vel * af
    gm = np.sqrt(g_n * g_n + g_t * g_t)
    if gm > 1e-12 and c_alpha > 0.0:
        ur = c_alpha * abs(vel) * g_n / gm
        ac, ad = (a_lo, a_hi) if ur >= 0.0 else (a_hi, a_lo)
        flux += ur * ac * (1.0 - ad)
    return flux


def vof_advect(a, u, v, fluid, nx, ny, dx, dy, dt, c_alpha, periodic, a_in, out):
    """One explicit conservative alpha transport step (cfd2d/vof.py:36-137)."""
    out[:, :] = a
    for i in range(0, nx + 1):
        for j in range(1, ny + 1):
            uf = u[i, j]
            if i == 0 and periodic:
                continue
            if i == 0 or (i == nx and not periodic):
                P = 1 if i == 0 else nx
                if fluid[P, j]:
                    into = uf if i == 0 else -uf
                    ab = a_in if into > 0 else a[P, j]
                    out[P, j] += dt * into * ab / dx
                continue
            L, R = i, (i + 1 if i < nx else 1)
            if not (fluid[L, j] and fluid[R, j]):
                continue
            if uf >= 0.0:
                up = L - 1 if L - 1 >= 1 else (nx if periodic else -1)
            else:
                up = R + 1 if R + 1 <= nx else (1 if periodic else -1)
            has_up = up >= 1 and bool(fluid[up, j])
            gx = (a[R, j] - a[L, j]) / dx
            jn = j + 1 if j < ny else j
            js = j - 1 if j > 1 else j
            gy = 0.25 * ((a[L, jn] - a[L, js]) + (a[R, jn] - a[R, js])) / dy
            flux = _vof_face_flux(uf, a[L, j], a[R, j], a[up, j] if has_up else 0.0, has_up, gx, gy, c_alpha)
            out[L, j] -= dt * flux / dx
            out[R, j] += dt * flux / dx
    for i in range(1, nx + 1):
        for j in range(0, ny + 1):
            vf = v[i, j]
            if j == 0 or j == ny:
                P = 1 if j == 0 else ny
                if fluid[i, P]:
                    into = vf if j == 0 else -vf
                    ab = a_in if into > 0 else a[i, P]
                    out[i, P] += dt * into * ab / dy
                continue
            B, T = j, j + 1
            if not (fluid[i, B] and fluid[i, T]):
                continue
            up = B - 1 if vf >= 0.0 else T + 1
            has_up = 1 <= up <= ny and bool(fluid[i, up])
            gy = (a[i, T] - a[i, B]) / dy
            ie = i + 1 if (i < nx or periodic) else i
            iw = i - 1 if (i > 1 or periodic) else i
            ie = 1 if ie > nx else ie
            iw = nx if iw < 1 else iw
            gx = 0.25 * ((a[ie, B] - a[iw, B]) + (a[ie, T] - a[iw, T])) / dx
            flux = _vof_face_flux(vf, a[i, B], a[i, T], a[i, up] if has_up else 0.0, has_up, gy, gx, c_alpha)
            out[i, B] -= dt * flux / dy
            out[i, T] += dt * flux / dy
    inner = out[1:-1, 1:-1]
    f = fluid[1:-1, 1:-1]
    inner[f] = np.minimum(np.maximum(inner[f], 0.0), 1.0)


class OVOF(OModel):
    """Two-phase VOF, interFoam-like (cfd2d/vof.py:140-306)."""
    kind = "multiphase"

    def __init__(self, alpha0, rho1=1000.0, rho2=1.0, nu1=1e-6, nu2=1.48e-5, sigma=0.07,
                 gravity=(0.0, -9.81), c_alpha=1.0, cfl_alpha=0.25, alpha_inflow=0.0):
        self.alpha0 = np.asarray(alpha0, dtype=float)
        self.rho1, self.rho2 = float(rho1), float(rho2)
        self.mu1, self.mu2 = float(nu1 * rho1), float(nu2 * rho2)
        self.sigma = float(sigma)
        self.gravity = (float(gravity[0]), float(gravity[1]))
        self.c_alpha, self.cfl, self.alpha_inflow = float(c_alpha), float(cfl_alpha), float(alpha_inflow)

    def attach(self, sim):
        # cfd2d/vof.py:184-197
        super().attach(sim)
        g = sim.grid
        self.alpha = np.zeros((g.nx + 2, g.ny + 2))
        self.alpha[1:-1, 1:-1] = np.where(g.fluid[1:-1, 1:-1], np.clip(self.alpha0, 0, 1), 0.0)
        self._tmp = np.zeros_like(self.alpha)
        sim.variable_density = True
        sim.variable_viscosity = True
        sim.body_force = (sim.body_force[0] + self.gravity[0], sim.body_force[1] + self.gravity[1])
        self.update_properties()
        self.volume0 = self.volume()

    def fill_ghosts(self):
        # cfd2d/vof.py:200-220: copies at the sides, solids the mean of their fluid neighbours
        a, g = self.alpha, self.sim.grid
        nx = g.nx
        if self.sim.periodic:
            a[0, :] = a[nx, :]
            a[nx + 1, :] = a[1, :]
        else:
            a[0, :] = a[1, :]
            a[-1, :] = a[-2, :]
        a[:, 0] = a[:, 1]
        a[:, -1] = a[:, -2]
        solid = ~g.fluid
        solid[0, :] = solid[-1, :] = solid[:, 0] = solid[:, -1] = False
        if solid.any():
            fl = g.fluid.astype(float)
            af = np.where(g.fluid, a, 0.0)
            s = np.zeros_like(a)
            c = np.zeros_like(a)
            s[1:-1, 1:-1] = af[2:, 1:-1] + af[:-2, 1:-1] + af[1:-1, 2:] + af[1:-1, :-2]
            c[1:-1, 1:-1] = fl[2:, 1:-1] + fl[:-2, 1:-1] + fl[1:-1, 2:] + fl[1:-1, :-2]
            a[solid] = np.where(c[solid] > 0, s[solid] / np.maximum(c[solid], 1), 0.0)

    def update_properties(self):
        # cfd2d/vof.py:222-227: mixture density and dynamic viscosity (held in nu_eff)
        self.fill_ghosts()
        a = self.alpha
        self.sim.rho[:] = a * self.rho1 + (1 - a) * self.rho2
        self.sim.nu_eff[:] = a * self.mu1 + (1 - a) * self.mu2

    def volume(self):
        g = self.sim.grid
        return float(self.alpha[1:-1, 1:-1][g.fluid[1:-1, 1:-1]].sum() * g.dx * g.dy)

    def momentum_source(self, sim, hu, hv):
        # cfd2d/vof.py:234-258: CSF surface tension sigma kappa grad(alpha) / rho
        if self.sigma <= 0:
            return
        g = sim.grid
        a = self.alpha
        As = a.copy()
        As[1:-1, 1:-1] = (4 * a[1:-1, 1:-1] + a[2:, 1:-1] + a[:-2, 1:-1] + a[1:-1, 2:] + a[1:-1, :-2]) / 8.0
        gx = 0.5 * ((As[1:, 1:] - As[:-1, 1:]) + (As[1:, :-1] - As[:-1, :-1])) / g.dx
        gy = 0.5 * ((As[1:, 1:] - As[1:, :-1]) + (As[:-1, 1:] - As[:-1, :-1])) / g.dy
        gm = np.sqrt(gx ** 2 + gy ** 2) + 1e-8 / g.dx
        nxn, nyn = gx / gm, gy / gm
        kappa = np.zeros_like(a)
        kappa[1:-1, 1:-1] = -(0.5 * ((nxn[1:, 1:] - nxn[:-1, 1:]) + (nxn[1:, :-1] - nxn[:-1, :-1])) / g.dx
                              + 0.5 * ((nyn[1:, 1:] - nyn[1:, :-1]) + (nyn[:-1, 1:] - nyn[:-1, :-1])) / g.dy)
        rho = sim.rho
        fxs = self.sigma * 0.5 * (kappa[:-1, :] + kappa[1:, :]) * (a[1:, :] - a[:-1, :]) / g.dx
        fys = self.sigma * 0.5 * (kappa[:, :-1] + kappa[:, 1:]) * (a[:, 1:] - a[:, :-1]) / g.dy
        rx = 0.5 * (rho[:-1, :] + rho[1:, :])
        ry = 0.5 * (rho[:, :-1] + rho[:, 1:])
        hu[sim.u_fluid] += (fxs / rx)[sim.u_fluid]
        hv[sim.v_fluid] += (fys / ry)[sim.v_fluid]

    def post_step(self, sim, dt):
        # cfd2d/vof.py:260-271: sub-steps at the alpha Courant number cfl
        g = sim.grid
        umax = max(np.abs(sim.u).max() / g.dx, np.abs(sim.v).max() / g.dy, 1e-12)
        nsub = max(1, int(np.ceil(dt * umax / self.cfl)))
        h = dt / nsub
        for _ in range(nsub):
            vof_advect(self.alpha, sim.u, sim.v, g.fluid, g.nx, g.ny, g.dx, g.dy, h, self.c_alpha,
                       sim.periodic, self.alpha_inflow, self._tmp)
            self.alpha[:] = self._tmp
            self.fill_ghosts()
        self.update_properties()

    def fields(self, sim):
        # cfd2d/vof.py:302-306
        solid = ~sim.grid.fluid[1:-1, 1:-1]
        return {"alpha": ("Volumenanteil α (Phase 1)", np.where(solid, np.nan, self.alpha[1:-1, 1:-1])),
                "rho": ("Dichte ρ", np.where(solid, np.nan, sim.rho[1:-1, 1:-1]))}

    def dt_limit(self, sim):
        # cfd2d/vof.py:273-284
        g = sim.grid
        lim = None
        if self.sigma > 0:
            h = min(g.dx, g.dy)
            lim = np.sqrt(0.5 * (self.rho1 + self.rho2) * h ** 3 / (2 * np.pi * self.sigma))
        gmag = np.hypot(*self.gravity)
        if gmag > 0:
            lg = np.sqrt(min(g.dx, g.dy) / gmag)
            lim = lg if lim is None else min(lim, lg)
        return lim


def dam_break(n=96, size=0.584, column_width=0.1461, column_height=0.292, obstacle=True, sigma=0.07,
              open_top=True, gamma=0.5, tau=0.5):
    # cfd2d/cases.py:294-320
    g = OGrid(n, n, size, size)
    if obstacle:
        x0 = 0.5 * size - 0.012
        g.add_obstacle(rectangle_mask(g, x0, 0.0, x0 + 0.024, 0.048))
    X, Y = g.centres()
    alpha0 = ((X <= column_width) & (Y <= column_height)).astype(float)
    bcs = {"left": OBC("noslip"), "right": OBC("noslip"), "bottom": OBC("noslip"),
           "top": OBC("outflow") if open_top else OBC("noslip")}
    return OSimulation(g, bcs, nu=1e-6, models=[OVOF(alpha0, sigma=sigma)], gamma=gamma, tau=tau)

"""Force coefficients (cfd2d/validation.py:73-78), used by reports and the bench."""

from __future__ import annotations

import numpy as np


def force_coefficients(fx, fy, U: float, L: float, rho: float = 1.0):
    q = 0.5 * rho * U ** 2 * L
    return np.asarray(fx) / q, np.asarray(fy) / q


def poiseuille_profile(y, H: float = 1.0, U_mean: float = 1.0):
    """Developed laminar channel profile u(y) = 6 U y (H - y) / H^2 (cfd2d/validation.py:64-66)."""
    y = np.asarray(y, dtype=float)
    return 6.0 * U_mean * y * (H - y) / H**2


def poiseuille_pressure_gradient(nu: float, H: float = 1.0, U_mean: float = 1.0) -> float:
    """dp/dx = -12 nu U / H^2 of that profile (cfd2d/validation.py:69-70)."""
    return -12.0 * nu * U_mean / H**2


def reattachment_length(sim, x_step: float, wall: str = "bottom"):
    """Distance from the step edge to where the near-wall u turns from backflow to
    forward flow, by linear interpolation (cfd2d/validation.py:132-152); None if no
    backflow or no reattachment."""
    g = sim.grid
    j = 1 if wall == "bottom" else g.ny
    x = np.arange(g.nx + 1) * g.dx
    u = sim.u[:, j]
    keep = x > x_step + 0.5 * g.dx
    xs, us = x[keep], u[keep]
    back = np.flatnonzero(us < 0)
    if back.size == 0:
        return None
    for k in range(int(back[0]), len(us) - 1):
        if us[k] < 0 <= us[k + 1]:
            return float(xs[k] - us[k] * (xs[k + 1] - xs[k]) / (us[k + 1] - us[k]) - x_step)
    return None

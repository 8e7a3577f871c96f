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


def dominant_frequency(t, signal, t_start: float | None = None):
    """Dominant frequency of a signal sampled at adaptive times (cfd2d/validation.py:81-114):
    resampled on 2^k equidistant points, mean removed, Hann-windowed FFT, the peak
    refined by a parabola through the log-magnitudes of its neighbours. Returns
    (frequency, amplitude, freqs, spectrum), or None for fewer than 64 samples or a
    constant signal."""
    t = np.asarray(t, dtype=float)
    s = np.asarray(signal, dtype=float)
    if t_start is not None:
        keep = t >= t_start
        t, s = t[keep], s[keep]
    if len(t) < 64 or t[-1] - t[0] <= 0:
        return None
    n = int(2 ** np.ceil(np.log2(len(t))))
    tu = np.linspace(t[0], t[-1], n)
    su = np.interp(tu, t, s)
    su = su - su.mean()
    if np.allclose(su, 0):
        return None
    spec = np.abs(np.fft.rfft(su * np.hanning(n)))
    freqs = np.fft.rfftfreq(n, tu[1] - tu[0])
    k = int(np.argmax(spec[1:]) + 1)
    f = freqs[k]
    if 1 <= k < len(spec) - 1:
        lm, l0, lp = np.log(spec[k - 1:k + 2] + 1e-300)
        curv = lm - 2 * l0 + lp
        if curv != 0:
            f = freqs[k] + 0.5 * (lm - lp) / curv * (freqs[1] - freqs[0])
    return float(f), float(spec[k]), freqs, spec


def strouhal_number(t, cl, D: float, U: float, t_start: float | None = None):
    """St = f D / U from the lift signal (cfd2d/validation.py:117-127); None without an
    oscillation (peak-to-peak below 1e-3)."""
    res = dominant_frequency(t, cl, t_start)
    if res is None:
        return None
    if np.ptp(np.asarray(cl)[np.asarray(t) >= (t_start or 0)]) < 1e-3:
        return None
    return res[0] * D / U


def separation_bubbles(sim, wall: str = "top", x_min: float = 0.0):
    """(start, end) of every backflow region of the near-wall u along a wall
    (cfd2d/validation.py:155-175)."""
    g = sim.grid
    j = 1 if wall == "bottom" else g.ny
    x = np.arange(g.nx + 1) * g.dx
    u = sim.u[:, j]
    bubbles, start = [], None
    for k in range(1, g.nx):
        if x[k] < x_min or not (g.fluid[k, j] and g.fluid[k + 1, j]):
            continue
        if start is None and u[k] < 0:
            start = x[k]
        elif start is not None and u[k] >= 0:
            bubbles.append((float(start), float(x[k])))
            start = None
    if start is not None:
        bubbles.append((float(start), float(x[g.nx - 1])))
    return bubbles

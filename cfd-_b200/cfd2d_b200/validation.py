"""Force coefficients (cfd2d/validation.py:73-78), used by reports and the bench."""

from __future__ import annotations

import numpy as np


def force_coefficients(fx, fy, U: float, L: float, rho: float = 1.0):
    q = 0.5 * rho * U ** 2 * L
    return np.asarray(fx) / q, np.asarray(fy) / q

"""Host post-processing helpers of cfd2d_b200.validation (CPU only)."""

from __future__ import annotations

import numpy as np
import pytest


def test_strouhal_from_synthetic_signal():
    # tests/test_cfd2d.py:105-110
    from cfd2d_b200 import validation

    t = np.linspace(0, 20, 4000)
    cl = np.sin(2 * np.pi * 3.0 * t)
    st = validation.strouhal_number(t, cl, D=0.1, U=1.0)
    assert st == pytest.approx(0.3, rel=0.01)


def test_dominant_frequency_short_or_flat_signal_is_none():
    from cfd2d_b200 import validation

    assert validation.dominant_frequency(np.linspace(0, 1, 10), np.ones(10)) is None
    assert validation.dominant_frequency(np.linspace(0, 1, 100), np.ones(100)) is None
    t = np.linspace(0, 20, 4000)
    assert validation.strouhal_number(t, 1e-5 * np.sin(t), D=0.1, U=1.0) is None


def test_poiseuille_formulas():
    from cfd2d_b200 import validation

    y = np.linspace(0, 1, 11)
    u = validation.poiseuille_profile(y)
    assert u.max() == pytest.approx(1.5) and np.trapezoid(u, y) == pytest.approx(1.0, rel=1e-2)
    assert validation.poiseuille_pressure_gradient(0.05) == pytest.approx(-0.6)

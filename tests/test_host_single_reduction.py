"""The single-reduction Jacobi-PCG recurrence (Chronopoulos and Gear, 1989) that the
device's opt-in solver forms run (k_pcg_slab1 and k_pcg_cluster1, selected by
grid_ctas = -2), restated here in NumPy in the kernels' order of operations and
checked on the CPU against the oracle's scipy-form trajectory on the reference's own
pressure operators: the same iteration count within 2 and the same solution to the
solver's tolerance. The recurrence is algebraically scipy's CG (one reduction of
r.z, z.w and r.r per iteration instead of two); only the rounding differs."""

from __future__ import annotations

import math

import numpy as np
import pytest

import oracle as O


def cg_single_reduction(matvec, b, x0, rtol, maxiter, dinv):
    """Jacobi-PCG by the single-reduction recurrence, as the device kernels order it:
    w = A z and delta = z.w of the initial z; each iteration p = z + beta p,
    q = w + beta q (= A p), p.q = delta - beta rho / alpha_prev, then x, r, z, w = A z
    and the three dot products together. Returns (x, iterations)."""
    bnrm2 = math.sqrt(np.dot(b, b))
    atol = rtol * bnrm2
    if bnrm2 == 0.0:
        return b, 0
    x = x0.copy()
    r = b - matvec(x) if x.any() else b.copy()
    z = dinv * r
    rho, rr = np.dot(r, z), np.dot(r, r)
    w = matvec(z)
    delta = np.dot(z, w)
    rho_prev = alpha_prev = 1.0
    p = q = None
    for it in range(maxiter):
        if math.sqrt(rr) < atol:
            return x, it
        if it == 0:
            beta, pq = 0.0, delta
            p, q = z.copy(), w.copy()
        else:
            beta = rho / rho_prev
            pq = delta - (beta * rho) / alpha_prev
            p = p * beta + z
            q = q * beta + w
        alpha = rho / pq
        x = x + alpha * p
        r = r - alpha * q
        z = dinv * r
        w = matvec(z)
        rho_prev, alpha_prev = rho, alpha
        rho, delta, rr = np.dot(r, z), np.dot(z, w), np.dot(r, r)
    return x, maxiter


def _system(sim, seed):
    """The reference's pressure operator of ``sim`` and a right-hand side with its
    Neumann-component means removed, as cfd2d/pressure.py:143-185 forms it."""
    ps = sim.pressure
    rng = np.random.default_rng(seed)
    rhs = rng.standard_normal(ps.fluid.shape)
    b = rhs[ps.fluid].astype(float)
    if ps.neumann_components:
        lab = ps.labels[ps.fluid]
        for c in ps.neumann_components:
            m = lab == c
            b[m] -= b[m].mean()
    return ps, -b


@pytest.mark.parametrize("case", ["cavity64", "cylinder440x82", "cylinder110x22"])
@pytest.mark.parametrize("rtol", [1e-8, 1e-10])
def test_single_reduction_follows_scipy_cg(case, rtol):
    if case == "cavity64":
        sim = O.cavity(re=100, n=64)
    elif case == "cylinder440x82":
        sim = O.cylinder(re=100, nx=440, ny=82)
    else:
        sim = O.cylinder(re=20, nx=110, ny=22)
    ps, b = _system(sim, 7)
    x0 = np.zeros_like(b)
    x_ref, info, its_ref = O.pcg_scipy_trajectory(ps.matvec, b, x0, rtol, 20000, ps.dinv)
    assert info == 0
    x, its = cg_single_reduction(ps.matvec, b, x0, rtol, 20000, ps.dinv)
    assert abs(its - its_ref) <= 2, (its, its_ref)
    # the true residual meets the tolerance, and the iterates differ only by rounding
    # (measured: 7e-14 on the cavity, 1.2e-13 on the 440 x 82 cylinder)
    res = b - ps.matvec(x)
    assert np.linalg.norm(res) < rtol * np.linalg.norm(b)
    assert np.abs(x - x_ref).max() / np.abs(x_ref).max() < 1e-10

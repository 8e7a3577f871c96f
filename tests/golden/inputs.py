"""Seeded inputs for the stencil-kernel fixtures.

Both ``make_golden.py`` (which runs the reference on them) and the tests (which run
the oracle and the CUDA kernels on them) rebuild the same arrays from these
functions, so only the reference's outputs are stored. NumPy's PCG64 stream behind
``default_rng(seed)`` is stable across releases.
"""

from __future__ import annotations

import numpy as np

SIZES = ((13, 9), (24, 17))


def rand_fluid(rng, nx, ny, periodic, n_blobs):
    """Fluid mask with random rectangular solids; ghost layer as the reference sets it."""
    f = np.zeros((nx + 2, ny + 2), dtype=bool)
    f[1:-1, 1:-1] = True
    for _ in range(n_blobs):
        i0 = rng.integers(1, nx)
        j0 = rng.integers(1, ny)
        w = rng.integers(1, 4)
        h = rng.integers(1, 4)
        f[i0:i0 + w, j0:j0 + h] = False
    f[0, :] = f[-1, :] = f[:, 0] = f[:, -1] = False
    if periodic:
        f[0, :] = f[nx, :]
        f[nx + 1, :] = f[1, :]
        f[:, 0] = False
        f[:, -1] = False
    return f


def momentum_cases():
    """Yield dicts of inputs for momentum_tendencies / obstacle_bc."""
    rng = np.random.default_rng(1234)
    for nx, ny in SIZES:
        for periodic in (False, True):
            for variable in (False, True):
                for var_density in (False, True):
                    fl = rand_fluid(rng, nx, ny, periodic, 6)
                    u = rng.standard_normal((nx + 1, ny + 2))
                    v = rng.standard_normal((nx + 2, ny + 1))
                    nu = 0.01 + 0.05 * rng.random((nx + 2, ny + 2))
                    if not variable:
                        nu[:] = 0.013
                    rho = 0.5 + rng.random((nx + 2, ny + 2))
                    yield dict(nx=nx, ny=ny, dx=1.0 / nx, dy=0.7 / ny, gamma=float(rng.random()),
                               variable=variable, periodic=periodic, var_density=var_density,
                               fluid=fl, u=u, v=v, nu=nu, rho=rho)


def scalar_cases():
    """Yield dicts of inputs for scalar_transport (every limiter, both obstacle modes)."""
    rng = np.random.default_rng(4321)
    for nx, ny in SIZES:
        for periodic in (False, True):
            for limiter in range(6):
                for obs_t in (0, 1):
                    fl = rand_fluid(rng, nx, ny, periodic, 5)
                    u = rng.standard_normal((nx + 1, ny + 2))
                    v = rng.standard_normal((nx + 2, ny + 1))
                    phi = rng.standard_normal((nx + 2, ny + 2))
                    diff = 1e-3 + 0.05 * rng.random((nx + 2, ny + 2))
                    diff[rng.random(diff.shape) < 0.1] = 0.0
                    bt = {s: rng.integers(0, 3, n).astype(np.int64)
                          for s, n in (("l", ny), ("r", ny), ("b", nx), ("t", nx))}
                    bv = {s: rng.standard_normal(n) for s, n in (("l", ny), ("r", ny), ("b", nx), ("t", nx))}
                    yield dict(nx=nx, ny=ny, dx=1.3 / nx, dy=0.9 / ny, limiter=limiter,
                               periodic=periodic, obs_t=obs_t, obs_v=float(rng.standard_normal()),
                               fluid=fl, u=u, v=v, phi=phi, diff=diff, bt=bt, bv=bv)


def vof_cases():
    """Yield dicts of inputs for vof_advect (cfd2d/vof.py:36-137): a column of
    phase 1 with a smeared interface, random velocities, random solids."""
    rng = np.random.default_rng(4321)
    for nx, ny in SIZES:
        for periodic in (False, True):
            for c_alpha in (0.0, 1.0):
                fluid = rand_fluid(rng, nx, ny, periodic, n_blobs=2)
                dx, dy = 1.0 / nx, 0.7 / ny
                a = np.zeros((nx + 2, ny + 2))
                xs = (np.arange(nx) + 0.5) / nx
                ys = (np.arange(ny) + 0.5) / ny
                X, Y = np.meshgrid(xs, ys, indexing="ij")
                a[1:-1, 1:-1] = np.clip(0.5 - 4.0 * (X - 0.4 - 0.1 * np.sin(6 * Y)), 0.0, 1.0)
                a[1:-1, 1:-1] += 0.05 * rng.uniform(-1, 1, (nx, ny))
                a[1:-1, 1:-1] = np.clip(a[1:-1, 1:-1], 0.0, 1.0)
                a[~fluid] = rng.uniform(0, 1, (~fluid).sum())
                u = rng.uniform(-1, 1, (nx + 1, ny + 2))
                v = rng.uniform(-1, 1, (nx + 2, ny + 1))
                yield dict(a=a, u=u, v=v, fluid=fluid, nx=nx, ny=ny, dx=dx, dy=dy,
                           dt=0.2 * min(dx, dy), c_alpha=c_alpha, periodic=periodic,
                           a_in=float(rng.integers(0, 2)))


def rho_field(rng, nx, ny, fluid):
    """Two-phase density (1000 / 1) with a smeared, wavy interface, padded."""
    xs = (np.arange(nx + 2) - 0.5) / nx
    ys = (np.arange(ny + 2) - 0.5) / ny
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    a = np.clip(0.5 - 5.0 * (Y - 0.45 - 0.1 * np.sin(5 * X + rng.uniform(0, 3))), 0.0, 1.0)
    return a * 1000.0 + (1 - a) * 1.0

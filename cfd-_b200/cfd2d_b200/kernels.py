"""Drop-in for cfd2d/kernels.py: the stencil kernels, run on the GPU.

Same signatures and in-place semantics as the reference's Numba kernels. Arrays
may be host numpy arrays (copied to the device and the outputs copied back into
the caller's arrays) or CUDA tensors (used in place, no copies).
"""

from __future__ import annotations

import numpy as np

from . import _lib

HAVE_NUMBA = False
# cfd2d/kernels.py:33-41
LIMITERS = {"upwind": 0, "vanleer": 1, "minmod": 2, "superbee": 3, "linear": 4, "mc": 5}
LIMITER_NAMES_DE = {
    "upwind": "Upwind (1. Ordnung, beschränkt)",
    "vanleer": "van Leer (TVD, 2. Ordnung)",
    "minmod": "Minmod (TVD, sehr robust)",
    "superbee": "Superbee (TVD, kantenscharf)",
    "mc": "MC / monotonized central (TVD)",
    "linear": "linear / zentral (2. Ordnung, unbeschränkt)",
}


def _f64(a):
    return _lib.to_dev(a, _lib.torch().float64)


def _u8(a):
    return _lib.to_dev(np.asarray(a, dtype=np.uint8) if isinstance(a, np.ndarray) else a,
                       _lib.torch().uint8)


def _back(host, dev):
    if isinstance(host, np.ndarray):
        host[...] = dev.cpu().numpy()
    elif dev.data_ptr() != host.data_ptr():
        host.copy_(dev)


def momentum_tendencies(u, v, fluid, nx, ny, dx, dy, nu, variable, gamma, periodic, hu, hv,
                        rho, var_density):
    """hu, hv = diffusion - convection on fluid faces (cfd2d/kernels.py:44-155)."""
    ud, vd, fd, nud = _f64(u), _f64(v), _u8(fluid), _f64(nu)
    hud, hvd = _f64(hu), _f64(hv)
    rhod = _f64(rho) if var_density else None
    rc = _lib.lib().cfd2d_momentum_tendencies(
        _lib.ptr(ud), _lib.ptr(vd), _lib.ptr(fd), int(nx), int(ny), float(dx), float(dy), _lib.ptr(nud),
        int(bool(variable)), float(gamma), int(bool(periodic)), _lib.ptr(hud), _lib.ptr(hvd),
        _lib.ptr(rhod), int(bool(var_density)), _lib.stream_ptr())
    _lib.check(rc, "cfd2d_momentum_tendencies")
    _back(hu, hud)
    _back(hv, hvd)


def obstacle_bc(u, v, fluid, nx, ny, periodic):
    """Solid-face velocities in place (cfd2d/kernels.py:158-209)."""
    ud, vd, fd = _f64(u), _f64(v), _u8(fluid)
    rc = _lib.lib().cfd2d_obstacle_bc(_lib.ptr(ud), _lib.ptr(vd), _lib.ptr(fd), int(nx), int(ny),
                                      int(bool(periodic)), _lib.stream_ptr())
    _lib.check(rc, "cfd2d_obstacle_bc")
    _back(u, ud)
    _back(v, vd)


def scalar_transport(phi, u, v, fluid, nx, ny, dx, dy, diff, limiter, periodic,
                     bt_l, bv_l, bt_r, bv_r, bt_b, bv_b, bt_t, bv_t, obs_t, obs_v, out):
    """out = -div(u phi) + div(D grad phi) on fluid cells (cfd2d/kernels.py:254-391)."""
    t = _lib.torch()
    pd, ud, vd, fd, dd = _f64(phi), _f64(u), _f64(v), _u8(fluid), _f64(diff)
    bts = [_lib.to_dev(np.asarray(b, dtype=np.int64) if not isinstance(b, t.Tensor) else b, t.int64)
           for b in (bt_l, bt_r, bt_b, bt_t)]
    bvs = [_f64(np.asarray(b, dtype=np.float64) if not isinstance(b, t.Tensor) else b)
           for b in (bv_l, bv_r, bv_b, bv_t)]
    od = _f64(out)
    rc = _lib.lib().cfd2d_scalar_transport(
        _lib.ptr(pd), _lib.ptr(ud), _lib.ptr(vd), _lib.ptr(fd), int(nx), int(ny), float(dx), float(dy),
        _lib.ptr(dd), int(limiter), int(bool(periodic)),
        _lib.ptr(bts[0]), _lib.ptr(bvs[0]), _lib.ptr(bts[1]), _lib.ptr(bvs[1]),
        _lib.ptr(bts[2]), _lib.ptr(bvs[2]), _lib.ptr(bts[3]), _lib.ptr(bvs[3]),
        int(obs_t), float(obs_v), _lib.ptr(od), _lib.stream_ptr())
    _lib.check(rc, "cfd2d_scalar_transport")
    _back(out, od)


def warmup() -> None:
    """Load the library and touch the device once (cfd2d/kernels.py:394-411)."""
    nx = ny = 4
    u = np.zeros((nx + 1, ny + 2))
    v = np.zeros((nx + 2, ny + 1))
    fl = np.zeros((nx + 2, ny + 2), dtype=np.bool_)
    fl[1:-1, 1:-1] = True
    hu = np.zeros_like(u)
    hv = np.zeros_like(v)
    nu = np.full((nx + 2, ny + 2), 0.01)
    momentum_tendencies(u, v, fl, nx, ny, 0.1, 0.1, nu, False, 0.5, False, hu, hv, nu, False)

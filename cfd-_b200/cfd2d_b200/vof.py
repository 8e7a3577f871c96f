"""Two-phase flow with the volume-of-fluid method on the device (drop-in for cfd2d/vof.py).

The volume fraction alpha (1 = phase 1, e.g. water; 0 = phase 2, e.g. air) is
transported by a bounded van Leer scheme with the interface-compression flux
u_r alpha (1 - alpha) of interFoam, in sub-steps at the alpha Courant number. The
mixture density and dynamic viscosity follow alpha; the momentum update divides the
viscous term by rho, surface tension enters as the CSF force sigma kappa grad(alpha)
(Brackbill 1992), and the projection solves div((1/rho) grad p) = div(u*) / dt.
Every part runs in CUDA kernels inside the step (cfd-_b200/csrc/vof.cu): the host
sets up alpha and the constants once.
"""

from __future__ import annotations

import numpy as np

from . import _lib
from .models import Model


def vof_advect(a, u, v, fluid, nx, ny, dx, dy, dt, c_alpha, periodic, a_in, out):
    """One explicit conservative transport step of alpha (cfd2d/vof.py:36-137) on the
    device; numpy or CUDA arrays, ``out`` written in place."""
    from .kernels import _back, _f64, _u8

    ad, ud, vd, fd = _f64(a), _f64(u), _f64(v), _u8(fluid)
    od = _f64(out)
    if od.data_ptr() == ad.data_ptr():
        od = od.clone()
    rc = _lib.lib().cfd2d_vof_advect(_lib.ptr(ad), _lib.ptr(ud), _lib.ptr(vd), _lib.ptr(fd), int(nx), int(ny),
                                     float(dx), float(dy), float(dt), float(c_alpha), int(bool(periodic)),
                                     float(a_in), _lib.ptr(od), _lib.stream_ptr())
    _lib.check(rc, "cfd2d_vof_advect")
    _back(out, od)


class VOF(Model):
    """Two-phase model, interFoam-like (cfd2d/vof.py:140-306).

    Parameters as the reference: alpha0 (nx, ny) initial phase-1 fraction, densities
    rho1/rho2, kinematic viscosities nu1/nu2, surface tension sigma (0: none),
    gravity (added to the body force), compression factor c_alpha, alpha Courant
    number cfl_alpha, alpha at inflowing open boundaries. ``nsub_max`` bounds the
    transport sub-steps queued per step (the device raises an error when a step
    would need more)."""

    kind = "multiphase"

    def __init__(self, alpha0, rho1: float = 1000.0, rho2: float = 1.0, nu1: float = 1e-6,
                 nu2: float = 1.48e-5, sigma: float = 0.07, gravity=(0.0, -9.81),
                 c_alpha: float = 1.0, cfl_alpha: float = 0.25, alpha_inflow: float = 0.0,
                 nsub_max: int = 16):
        self.alpha0 = np.asarray(alpha0, dtype=float)
        self.rho1, self.rho2 = float(rho1), float(rho2)
        self.mu1, self.mu2 = float(nu1 * rho1), float(nu2 * rho2)
        self.sigma = float(sigma)
        self.gravity = (float(gravity[0]), float(gravity[1]))
        self.c_alpha = float(c_alpha)
        self.cfl = float(cfl_alpha)
        self.alpha_inflow = float(alpha_inflow)
        self.nsub_max = int(nsub_max)
        self.title = (f"VOF zweiphasig: rho1 = {rho1:g}, rho2 = {rho2:g}, sigma = {sigma:g}, "
                      f"g = {self.gravity}, c_alpha = {c_alpha:g}")

    def attach(self, sim) -> None:
        super().attach(sim)
        if sim._sst is not None or sim._smag is not None:
            raise ValueError("VOF lässt sich nicht mit einem Turbulenzmodell kombinieren")
        g = sim.grid
        nx, ny = g.nx, g.ny
        if self.alpha0.shape != (nx, ny):
            raise ValueError(f"alpha0 muss die Form {(nx, ny)} haben.")
        t = _lib.torch()
        dev = _lib.device()
        alpha = np.zeros((nx + 2, ny + 2))
        alpha[1:-1, 1:-1] = np.where(g.fluid_interior, np.clip(self.alpha0, 0, 1), 0.0)
        z = lambda *shape: t.zeros(shape, dtype=t.float64, device=dev)  # noqa: E731
        self._alpha = _lib.to_dev(alpha, t.float64)
        self._tmp = z(nx + 2, ny + 2)
        self._smooth = z(nx + 2, ny + 2)
        self._nrm = z(2, nx + 1, ny + 1)
        self._kappa = z(nx + 2, ny + 2)
        self._bx = z(nx + 1, ny + 2)
        self._by = z(nx + 2, ny + 1)
        self._vdiag = z(nx, ny)
        self._vdinv = z(nx, ny)
        self._scal = z(4)
        # outflow (Dirichlet) sides and pinned cells of the pressure operator
        ps = sim.pressure
        flags = np.zeros((nx, ny), dtype=np.uint8)
        flags[0, :] |= np.where(ps.dirichlet["left"], 1, 0).astype(np.uint8)
        flags[-1, :] |= np.where(ps.dirichlet["right"], 2, 0).astype(np.uint8)
        flags[:, 0] |= np.where(ps.dirichlet["bottom"], 4, 0).astype(np.uint8)
        flags[:, -1] |= np.where(ps.dirichlet["top"], 8, 0).astype(np.uint8)
        for fi, fj in ps._pinned:
            flags[fi, fj] |= 16
        self._vflags = _lib.to_dev(flags)
        self.volume0 = 0.0
        ps.ensure_workspace()
        sim.variable_density = True
        sim.variable_viscosity = True
        sim.body_force = (sim.body_force[0] + self.gravity[0], sim.body_force[1] + self.gravity[1])
        sim._set_vof(self)
        sim._vof_properties()
        self.volume0 = self.volume()
        sim._invalidate()  # the volume error monitor refers to volume0

    def fill_struct(self, V) -> None:
        sim = self.sim
        for name in ("alpha", "tmp", "smooth", "nrm", "kappa", "bx", "by", "vdiag", "vdinv", "scal", "vflags"):
            setattr(V, "alpha_tmp" if name == "tmp" else name, getattr(self, "_" + name).data_ptr())
        V.rho = sim._rho.data_ptr()
        V.rho1, V.rho2, V.mu1, V.mu2 = self.rho1, self.rho2, self.mu1, self.mu2
        V.sigma, V.c_alpha, V.cfl, V.alpha_in = self.sigma, self.c_alpha, self.cfl, self.alpha_inflow
        lim = self.dt_limit(sim)
        V.dt_limit = float(lim) if lim is not None else 0.0
        # the reference solves this system directly (scipy spsolve)
        V.rtol = 1e-13
        V.maxiter = 20000
        V.nsub_max = self.nsub_max

    # ------------------------------------------------------------------ host views
    @property
    def alpha(self) -> np.ndarray:
        return self.sim._mirror("vof_alpha", self._alpha)

    def volume(self) -> float:
        g = self.sim.grid
        return float(self.alpha[1:-1, 1:-1][g.fluid_interior].sum() * g.dx * g.dy)

    def dt_limit(self, sim):
        """Capillary and gravity-wave time step limits (cfd2d/vof.py:273-284)."""
        g = sim.grid
        lim = None
        if self.sigma > 0:
            h = min(g.dx, g.dy)
            lim = np.sqrt(0.5 * (self.rho1 + self.rho2) * h**3 / (2 * np.pi * self.sigma))
        gmag = np.hypot(*self.gravity)
        if gmag > 0:
            lg = np.sqrt(min(g.dx, g.dy) / gmag)
            lim = lg if lim is None else min(lim, lg)
        return lim

    def monitors(self, sim) -> dict:
        g = sim.grid
        a = self.alpha[1:-1, 1:-1]
        out = {"volumen_phase1": self.volume(),
               "volumenfehler_rel": self.volume() / max(self.volume0, 1e-300) - 1.0}
        row = np.where(a[:, 0] > 0.5)[0]
        out["front_x"] = float(g.xc[row.max()] + 0.5 * g.dx) if row.size else 0.0
        col = np.where(a[0, :] > 0.5)[0]
        out["hoehe_links"] = float(g.yc[col.max()] + 0.5 * g.dy) if col.size else 0.0
        return out

    def device_monitors(self, sim):
        a = self._alpha.data_ptr()
        M = _lib.Monitor
        return [("volumen_phase1", M(_lib.MON_SUM_FLUID, 0, 0, 0, a, 0.0)),
                ("volumenfehler_rel", M(_lib.MON_VOLUME_ERROR, 0, 0, 0, a, float(self.volume0))),
                ("front_x", M(_lib.MON_FRONT_X, 0, 0, 0, a, 0.0)),
                ("hoehe_links", M(_lib.MON_HEIGHT_LEFT, 0, 0, 0, a, 0.0))]

    def state(self) -> dict:
        return {"alpha": self.alpha, "volume0": np.array(self.volume0)}

    def set_state(self, sim, state: dict) -> None:
        with sim._on_stream():
            self._alpha.copy_(_lib.to_dev(np.asarray(state["alpha"], dtype=np.float64)))
        m = sim._mirrors.get("vof_alpha")
        if m is not None and m.host is not None:
            m.host[...] = state["alpha"]
            m.snap[...] = state["alpha"]
        if "volume0" in state:
            self.volume0 = float(state["volume0"])
            sim._invalidate()
        sim._vof_properties()

    def fields(self, sim) -> dict:
        solid = sim.grid.solid
        return {"alpha": ("Volumenanteil α (Phase 1)", np.where(solid, np.nan, self.alpha[1:-1, 1:-1])),
                "rho": ("Dichte ρ", np.where(solid, np.nan, sim.rho[1:-1, 1:-1]))}

    def device_fields(self, sim):
        return {"alpha": ("Volumenanteil α (Phase 1)", _lib.FIELD_CELL, self._alpha),
                "rho": ("Dichte ρ", _lib.FIELD_CELL, sim._rho)}

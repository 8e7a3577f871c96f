"""Domain boundary conditions (drop-in for cfd2d/boundary.py).

The host computes the setup data once: which boundary segments are open (the
adjacent interior cell is fluid) and the inflow profile of every open run. The
per-step application to u and v runs on the GPU (``cfd2d_domain_bc``), fused
into the step by the simulation.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib
from .grid import Grid

SIDES = ("left", "right", "bottom", "top")
SIDE_NAMES_DE = {"left": "links", "right": "rechts", "bottom": "unten", "top": "oben"}
KINDS = ("noslip", "slip", "inflow", "outflow", "periodic")
KIND_NAMES_DE = {"noslip": "Haftende Wand", "slip": "Reibungsfreie Wand", "inflow": "Einströmung",
                 "outflow": "Ausströmung", "periodic": "Periodisch"}


@dataclass
class BoundaryCondition:
    """Condition of one side (cfd2d/boundary.py:41-60)."""

    kind: str = "noslip"
    velocity: float = 0.0
    profile: str = "uniform"

    def __post_init__(self):
        if self.kind not in KINDS:
            raise ValueError(f"Unbekannte Randbedingung {self.kind!r}, erlaubt: {KINDS}")
        if self.profile not in ("uniform", "parabolic"):
            raise ValueError("Einströmprofil muss 'uniform' oder 'parabolic' sein.")

    def describe(self) -> str:
        s = KIND_NAMES_DE[self.kind]
        if self.kind == "noslip" and self.velocity != 0.0:
            s += f" (bewegt, U={self.velocity:g})"
        if self.kind == "inflow":
            prof = "parabolisch" if self.profile == "parabolic" else "Blockprofil"
            s += f" ({prof}, U_mittel={self.velocity:g})"
        return s


def inflow_profile(coords: np.ndarray, open_mask: np.ndarray, h: float, mean_velocity: float,
                   profile: str) -> np.ndarray:
    """Inflow velocity along one side: one profile per contiguous open run.

    Parabolic runs a..b (cell faces around the run) get 6 U (s-a)(b-s)/(b-a)^2, uniform
    runs U (cfd2d/boundary.py:63-89).
    """
    values = np.zeros_like(coords)
    open_mask = np.asarray(open_mask, dtype=bool)
    n = len(open_mask)
    starts = np.flatnonzero(open_mask & ~np.concatenate(([False], open_mask[:-1])))
    for j in starts:
        k = j
        while k + 1 < n and open_mask[k + 1]:
            k += 1
        a = coords[j] - 0.5 * h
        b = coords[k] + 0.5 * h
        s = coords[j:k + 1]
        if profile == "parabolic":
            values[j:k + 1] = 6.0 * mean_velocity * (s - a) * (b - s) / (b - a) ** 2
        else:
            values[j:k + 1] = mean_velocity
    return values


class DomainBoundary:
    """Boundary data of the four sides; ``apply`` sets ghost and boundary-face values."""

    def __init__(self, grid: Grid, bcs: dict):
        missing = [s for s in SIDES if s not in bcs]
        if missing:
            raise ValueError(f"Randbedingungen fehlen für: {missing}")
        self.grid, self.bcs = grid, bcs
        pl = bcs["left"].kind == "periodic"
        pr = bcs["right"].kind == "periodic"
        if pl != pr:
            raise ValueError("Periodische Ränder müssen links UND rechts gesetzt werden.")
        if bcs["bottom"].kind == "periodic" or bcs["top"].kind == "periodic":
            raise ValueError("Periodische Ränder werden nur in x-Richtung (links/rechts) unterstützt.")
        self.periodic = pl
        if pl:
            grid.set_periodic_x()
        fl, nx, ny = grid.fluid, grid.nx, grid.ny
        self.open = {"left": fl[1, 1:ny + 1].copy(), "right": fl[nx, 1:ny + 1].copy(),
                     "bottom": fl[1:nx + 1, 1].copy(), "top": fl[1:nx + 1, ny].copy()}
        self.inflow_values = {}
        for side, bc in bcs.items():
            if bc.kind != "inflow":
                continue
            coords, h = (grid.yc, grid.dy) if side in ("left", "right") else (grid.xc, grid.dx)
            vals = inflow_profile(coords, self.open[side], h, bc.velocity, bc.profile)
            self.inflow_values[side] = (1.0 if side in ("left", "bottom") else -1.0) * vals
        self._dev = None

    @property
    def has_outflow(self) -> bool:
        return any(bc.kind == "outflow" for bc in self.bcs.values())

    def outflow_mask(self, side: str) -> np.ndarray:
        """Boundary faces with the pressure Dirichlet condition (cfd2d/boundary.py:137-141)."""
        if self.bcs[side].kind != "outflow":
            return np.zeros_like(self.open[side])
        return self.open[side]

    # -------------------------------------------------------------- device data
    def device_data(self):
        """Device copies of the open masks and inflow profiles (uploaded once)."""
        if self._dev is None:
            opens = [_lib.to_dev(self.open[s].astype(np.uint8)) for s in SIDES]
            inflow = [(_lib.to_dev(self.inflow_values[s].astype(np.float64)) if s in self.inflow_values
                       else None) for s in SIDES]
            self._dev = (opens, inflow)
        return self._dev

    def fill_struct(self, S) -> None:
        opens, inflow = self.device_data()
        for k, s in enumerate(SIDES):
            S.bc_kind[k] = _lib.BC_CODES[self.bcs[s].kind]
            S.bc_vel[k] = float(self.bcs[s].velocity)
            S.open[k] = opens[k].data_ptr()
            S.inflow[k] = inflow[k].data_ptr() if inflow[k] is not None else 0

    def apply(self, u, v) -> None:
        """Set all boundary values on u and v in place (cfd2d/boundary.py:143-223).

        u, v may be host numpy arrays (copied to the device and back) or CUDA tensors.
        """
        import ctypes as C

        g = self.grid
        S = _lib.Sim()
        S.nx, S.ny, S.dx, S.dy, S.periodic = g.nx, g.ny, g.dx, g.dy, int(self.periodic)
        self.fill_struct(S)
        ud, vd = _lib.to_dev(u, _lib.torch().float64), _lib.to_dev(v, _lib.torch().float64)
        rc = _lib.lib().cfd2d_domain_bc(C.byref(S), _lib.ptr(ud), _lib.ptr(vd), _lib.stream_ptr())
        _lib.check(rc, "cfd2d_domain_bc")
        if isinstance(u, np.ndarray):
            u[...] = ud.cpu().numpy()
            v[...] = vd.cpu().numpy()
        else:
            if ud.data_ptr() != u.data_ptr():
                u.copy_(ud)
            if vd.data_ptr() != v.data_ptr():
                v.copy_(vd)

    def describe(self) -> str:
        return "\n".join(f"  {SIDE_NAMES_DE[s]:>6}: {self.bcs[s].describe()}" for s in SIDES)

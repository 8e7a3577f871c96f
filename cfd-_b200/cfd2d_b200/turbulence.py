"""Turbulence models on the device path (drop-in for cfd2d/turbulence.py):
k-omega SST and LES Smagorinsky.

Setup (cfd2d/turbulence.py:199-236): inlet/initial k and omega, the wall-adjacent
cells and their viscous omega on the host; the wall distance (exact Euclidean
distance transform of the wall cells) on the device. Every step, the
CUDA kernels evaluate the blending functions, nu_t and the blended diffusivities
before the momentum update and transport k and omega with their sources after
the projection. Smagorinsky keeps only its squared length scale on the device; its
kernel evaluates nu_t before each momentum update. One turbulence model per
simulation: attaching a second raises ValueError.
"""

from __future__ import annotations

import numpy as np

from . import _lib
from .boundary import SIDES
from .models import Model, ScalarBC, ScalarField

KAPPA = 0.41


def wall_mask_padded(sim) -> np.ndarray:
    """Cells that count as wall: no-slip sides and interior solids (turbulence.py:28-40)."""
    g = sim.grid
    wall = g.interior_solid_padded()
    if sim.bcs["left"].kind == "noslip":
        wall[0, :] = True
    if sim.bcs["right"].kind == "noslip":
        wall[-1, :] = True
    if sim.bcs["bottom"].kind == "noslip":
        wall[:, 0] = True
    if sim.bcs["top"].kind == "noslip":
        wall[:, -1] = True
    return wall


def wall_distance(sim) -> np.ndarray:
    """Cell-centre distance to the nearest wall face, (nx+2, ny+2) (turbulence.py:43-70).

    Computed on the device (``cfd2d_sim_wall_distance``: exact separable Euclidean
    distance transform of the wall cells, periodic in x when the case is)."""
    g = sim.grid
    t = _lib.torch()
    dev = _lib.device()
    lib = _lib.lib()
    nbytes = int(lib.cfd2d_wall_distance_workspace_bytes(g.nx, g.ny))
    work = t.empty(nbytes, dtype=t.uint8, device=dev)
    dist = t.empty((g.nx + 2, g.ny + 2), dtype=t.float64, device=dev)
    with sim._on_stream():
        sim._flush_mirrors()
        sim._call("cfd2d_sim_wall_distance", _lib.ptr(dist), _lib.ptr(work), nbytes)
        out = dist.cpu().numpy()
    return out


def wall_adjacent_cells(sim):
    """Fluid cells next to a wall and their half-cell wall distance (turbulence.py:73-86)."""
    g = sim.grid
    wall = wall_mask_padded(sim)
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


def strain_rate_squared(sim) -> np.ndarray:
    """S^2 = 2 S_ij S_ij at the cell centres, (nx, ny) (cfd2d/turbulence.py:89-100), from
    the host view of the velocities (the model kernels evaluate it on the device)."""
    g = sim.grid
    u, v = sim.u, sim.v
    dudx = (u[1:, 1:-1] - u[:-1, 1:-1]) / g.dx
    dvdy = (v[1:-1, 1:] - v[1:-1, :-1]) / g.dy
    shear = (u[:, 1:] - u[:, :-1]) / g.dy + (v[1:, :] - v[:-1, :]) / g.dx
    sh2 = 0.25 * (shear[:-1, :-1] ** 2 + shear[1:, :-1] ** 2 + shear[:-1, 1:] ** 2 + shear[1:, 1:] ** 2)
    return 2.0 * (dudx ** 2 + dvdy ** 2) + sh2


class KOmegaSST(Model):
    """Menter SST k-omega, low-Re form (cfd2d/turbulence.py:166-325)."""

    kind = "turbulence"
    a1, beta_star = 0.31, 0.09
    sk1, so1, beta1, gamma1 = 0.85, 0.5, 0.075, 5.0 / 9.0
    sk2, so2, beta2, gamma2 = 1.0, 0.856, 0.0828, 0.44

    def __init__(self, intensity: float = 0.05, viscosity_ratio: float = 10.0, U_ref: float = 1.0,
                 limiter: str = "upwind"):
        self.I = float(intensity)
        self.ratio = float(viscosity_ratio)
        self.U_ref = float(U_ref)
        self.limiter = limiter
        self.title = f"RANS k-ω SST (Menter 2003), I = {intensity:g}, ν_t/ν = {viscosity_ratio:g}"

    def attach(self, sim) -> None:
        super().attach(sim)
        if sim._smag is not None:
            raise ValueError("nur ein Turbulenzmodell je Simulation")
        sim.variable_viscosity = True
        nu = sim.nu
        k0 = 1.5 * (self.I * self.U_ref) ** 2
        w0 = k0 / (nu * self.ratio)
        self.k_in, self.w_in = k0, w0
        kb, wb = {}, {}
        for side in SIDES:
            kind = sim.bcs[side].kind
            if kind == "inflow":
                kb[side], wb[side] = ScalarBC("fixed", k0), ScalarBC("fixed", w0)
            elif kind == "noslip":
                kb[side], wb[side] = ScalarBC("fixed", 0.0), ScalarBC("zerogradient")
            else:
                kb[side], wb[side] = ScalarBC("zerogradient"), ScalarBC("zerogradient")
        self.k = ScalarField("k", nu, kb, ScalarBC("fixed", 0.0), self.limiter, k0, source="sst_k",
                             lower=1e-14, label="Turbulente kin. Energie k")
        self.w = ScalarField("omega", nu, wb, ScalarBC("zerogradient"), self.limiter, w0,
                             source="sst_omega", lower=1e-8, label="Spez. Dissipationsrate ω")
        g = sim.grid
        nx, ny = g.nx, g.ny
        d = np.maximum(wall_distance(sim)[1:-1, 1:-1], 1e-12)
        adj, dist = wall_adjacent_cells(sim)
        self.wall_adj = adj[1:-1, 1:-1]
        self.w_wall = np.where(self.wall_adj, 6.0 * nu / (self.beta1 * np.where(
            np.isfinite(dist[1:-1, 1:-1]), dist[1:-1, 1:-1], 1.0) ** 2), 0.0)
        self.d = d
        # the viscous wall omega goes into the initial field before the ghosts are
        # filled (turbulence.py:232-242)
        w_init = np.full((nx + 2, ny + 2), float(w0))
        w_init[1:-1, 1:-1][self.wall_adj] = self.w_wall[self.wall_adj]
        self.w.initial = w_init
        self.k.attach(sim)
        self.w.attach(sim)
        sim.scalars["k"] = self.k
        sim.scalars["omega"] = self.w
        t = _lib.torch()
        dev = _lib.device()
        z = lambda: t.zeros((nx, ny), dtype=t.float64, device=dev)  # noqa: E731
        self._S2, self._F1, self._cross, self._Pk = z(), z(), z(), z()
        self._F1.fill_(1.0)
        self._d = _lib.to_dev(d)
        self._wall_adj = _lib.to_dev(self.wall_adj.astype(np.uint8))
        self._w_wall = _lib.to_dev(self.w_wall)
        sim._set_sst(self)
        # initial ghosts of k and omega, then the first pre-momentum evaluation
        sim._scalar_fill_ghosts(self.k.slot)
        sim._scalar_fill_ghosts(self.w.slot)
        sim._sst_pre_momentum()

    def fill_struct(self, sst) -> None:
        sst.S2, sst.F1 = self._S2.data_ptr(), self._F1.data_ptr()
        sst.cross, sst.Pk = self._cross.data_ptr(), self._Pk.data_ptr()
        sst.d, sst.wall_adj, sst.w_wall = self._d.data_ptr(), self._wall_adj.data_ptr(), self._w_wall.data_ptr()
        sst.k_index, sst.w_index = self.k.slot, self.w.slot

    @property
    def F1(self) -> np.ndarray:
        return self._F1.cpu().numpy()

    def dt_limit(self, sim):
        return min(self.k.dt_limit(), self.w.dt_limit())

    def monitors(self, sim) -> dict:
        return {"k_mittel": float(np.nanmean(self.k.cell())), "nu_t_max": float(sim.nu_t.max())}

    def device_monitors(self, sim):
        return [("k_mittel", _lib.Monitor(_lib.MON_MEAN_FLUID, 0, 0, 0, self.k._phi.data_ptr(), 0.0)),
                ("nu_t_max", _lib.Monitor(_lib.MON_MAX_ALL, 0, 0, 0, sim._nu_t.data_ptr(), 0.0))]

    def device_fields(self, sim):
        return {"k": (self.k.label, _lib.FIELD_CELL, self.k._phi),
                "omega": ("log10 ω (spez. Dissipationsrate)", _lib.FIELD_CELL_LOG10, self.w._phi),
                "nu_t": ("Turbulente Viskosität ν_t", _lib.FIELD_CELL, sim._nu_t)}

    def fields(self, sim) -> dict:
        solid = sim.grid.solid
        return {"k": (self.k.label, self.k.cell()),
                "omega": ("log10 ω (spez. Dissipationsrate)", np.log10(np.maximum(self.w.cell(), 1e-30))),
                "nu_t": ("Turbulente Viskosität ν_t", np.where(solid, np.nan, sim.nu_t[1:-1, 1:-1]))}


class Smagorinsky(Model):
    """LES Smagorinsky, nu_t = l^2 |S| (cfd2d/turbulence.py:130-160).

    The squared length l^2 = min(C_s sqrt(dx dy), kappa d)^2 (wall damping with the
    same wall distance as SST) is computed once on the host when the model attaches;
    every step a CUDA kernel evaluates the strain rate, nu_t, its ghost values and
    nu_eff before the momentum update."""

    kind = "turbulence"

    def __init__(self, cs: float = 0.17, wall_damping: bool = True):
        self.cs = float(cs)
        self.wall_damping = wall_damping
        self.title = f"LES Smagorinsky (C_s = {cs:g}" + (", Wanddämpfung" if wall_damping else "") + ")"

    def attach(self, sim) -> None:
        super().attach(sim)
        if sim._sst is not None:
            raise ValueError("nur ein Turbulenzmodell je Simulation")
        sim.variable_viscosity = True
        g = sim.grid
        length = np.full((g.nx, g.ny), self.cs * np.sqrt(g.dx * g.dy))
        if self.wall_damping:
            length = np.minimum(length, KAPPA * wall_distance(sim)[1:-1, 1:-1])
        self.l2 = length ** 2
        self._l2 = _lib.to_dev(self.l2)
        sim._set_smagorinsky(self)
        sim._smagorinsky_pre_momentum()

    def l2_ptr(self) -> int:
        return self._l2.data_ptr()

    def monitors(self, sim) -> dict:
        return {"nu_t_max": float(sim.nu_t.max())}

    def fields(self, sim) -> dict:
        return {"nu_t": ("Turbulente Viskosität ν_t",
                         np.where(sim.grid.solid, np.nan, sim.nu_t[1:-1, 1:-1]))}

    def device_fields(self, sim):
        return {"nu_t": ("Turbulente Viskosität ν_t", _lib.FIELD_CELL, sim._nu_t)}

    def device_monitors(self, sim):
        return [("nu_t_max", _lib.Monitor(_lib.MON_MAX_ALL, 0, 0, 0, sim._nu_t.data_ptr(), 0.0))]


TURBULENCE_MODELS = {"laminar": None, "kOmegaSST": KOmegaSST, "Smagorinsky": Smagorinsky}

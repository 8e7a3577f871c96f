"""Physics models on the device path (drop-in for cfd2d/models.py).

The reference's models hook Python code into every step. Here each built-in model
declares device data instead: scalar transport slots (TVD transport, Euler update,
point-implicit sources, clipping, ghost filling), the Boussinesq momentum source
and the k-omega SST terms, all executed by the fused CUDA step. Models that are not
built in cannot be attached (they would need host round trips every step).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib
from .boundary import SIDES
from .kernels import LIMITERS


@dataclass
class ScalarBC:
    """Scalar boundary condition (cfd2d/models.py:28-58): zerogradient, fixed, flux."""

    kind: str = "zerogradient"
    value: object = 0.0

    _CODES = {"zerogradient": 0, "fixed": 1, "flux": 2}

    def __post_init__(self):
        if self.kind not in self._CODES:
            raise ValueError(f"Unbekannte Skalar-Randbedingung {self.kind!r}, erlaubt: {list(self._CODES)}")

    @property
    def code(self) -> int:
        return self._CODES[self.kind]

    def describe(self) -> str:
        names = {"zerogradient": "Gradient null", "fixed": "fester Wert", "flux": "fester Fluss"}
        v = self.value
        vs = f" = {v:g}" if isinstance(v, (int, float)) else ""
        return names[self.kind] + (vs if self.kind != "zerogradient" else "")


def default_scalar_bcs(sim, inflow_value: float = 0.0) -> dict:
    """Inflow sides get a fixed value, all others zero gradient (cfd2d/models.py:61-70)."""
    return {s: (ScalarBC("fixed", inflow_value) if sim.bcs[s].kind == "inflow" else ScalarBC("zerogradient"))
            for s in SIDES}


class ScalarField:
    """d(phi)/dt + div(u phi) = div(D grad phi) + S on the device (cfd2d/models.py:73-250).

    ``source`` selects a built-in source term: None, "sst_k" or "sst_omega".
    """

    def __init__(self, name: str, diffusivity: float, bcs: dict | None = None,
                 obstacle: ScalarBC | None = None, limiter: str = "vanleer", initial=0.0,
                 source=None, lower: float | None = None, upper: float | None = None,
                 label: str | None = None):
        if limiter not in LIMITERS:
            raise ValueError(f"Unbekannter Limiter {limiter!r}, erlaubt: {list(LIMITERS)}")
        if source not in (None, "sst_k", "sst_omega"):
            raise NotImplementedError("eigene Quellterme laufen nicht auf dem Gerät; "
                                      "eingebaut sind nur die SST-Quellen")
        self.name, self.label = name, label or name
        self.D0 = float(diffusivity)
        self.bcs_in = bcs
        self.obstacle = obstacle or ScalarBC("zerogradient")
        self.limiter, self.initial, self.source = limiter, initial, source
        self.lower, self.upper = lower, upper
        self.sim = None
        self.slot = -1
        self.turb_number = None  # turbulent Schmidt/Prandtl number: diff = D0 + nu_t / it

    def attach(self, sim) -> None:
        # cfd2d/models.py:102-136
        self.sim = sim
        g = sim.grid
        nx, ny = g.nx, g.ny
        phi = np.zeros((nx + 2, ny + 2))
        if np.isscalar(self.initial):
            phi[:] = float(self.initial)
        else:
            init = np.asarray(self.initial, dtype=float)
            if init.shape == (nx, ny):
                phi[1:-1, 1:-1] = init
            elif init.shape == phi.shape:
                phi[:] = init
            else:
                raise ValueError(f"Anfangsfeld für {self.name} hat falsche Form {init.shape}")
        bcs = default_scalar_bcs(sim)
        bcs.update(self.bcs_in or {})
        self.bcs = bcs
        coords = {"left": g.yc, "right": g.yc, "bottom": g.xc, "top": g.xc}
        self.bt, self.bv = {}, {}
        for side in SIDES:
            s = coords[side]
            bc = bcs[side]
            self.bt[side] = np.full(len(s), bc.code, dtype=np.int64)
            val = bc.value
            if callable(val):
                self.bv[side] = np.asarray(val(s), dtype=float)
            else:
                self.bv[side] = np.broadcast_to(np.asarray(val, dtype=float), s.shape).copy()
        self._phi = _lib.to_dev(phi)
        self._diff = _lib.to_dev(np.full((nx + 2, ny + 2), self.D0))
        self._rhs = _lib.to_dev(np.zeros((nx + 2, ny + 2)))
        self._bt = [_lib.to_dev(self.bt[s]) for s in SIDES]
        self._bv = [_lib.to_dev(self.bv[s]) for s in SIDES]
        self.slot = sim._register_scalar(self)

    @property
    def turb_div(self) -> float:
        if self.turb_number is not None and self.sim is not None and self.sim.variable_viscosity:
            return float(self.turb_number)
        return 0.0

    def fill_struct(self, sc) -> None:
        sc.phi, sc.diff, sc.rhs = self._phi.data_ptr(), self._diff.data_ptr(), self._rhs.data_ptr()
        for k in range(4):
            sc.bt[k] = self._bt[k].data_ptr()
            sc.bv[k] = self._bv[k].data_ptr()
        sc.limiter = LIMITERS[self.limiter]
        sc.obs_t = self.obstacle.code
        sc.obs_v = float(self.obstacle.value) if self.obstacle.kind == "fixed" else 0.0
        sc.D0 = self.D0
        sc.turb_div = float(self.turb_div)
        sc.has_lower, sc.lower = int(self.lower is not None), float(self.lower or 0.0)
        sc.has_upper, sc.upper = int(self.upper is not None), float(self.upper or 0.0)
        sc.source = {None: 0, "sst_k": 1, "sst_omega": 2}[self.source]

    def dt_limit_const(self) -> float:
        """Constant diffusion limit (cfd2d/models.py:210-215), 0 if the diffusivity varies."""
        if self.source is not None or self.turb_div > 0.0:
            return 0.0
        g = self.sim.grid
        if self.D0 <= 0:
            return float("inf")
        return 0.5 / (self.D0 * (1.0 / g.dx ** 2 + 1.0 / g.dy ** 2))

    # ------------------------------------------------------------ host views
    @property
    def phi(self) -> np.ndarray:
        return self.sim._mirror(f"phi_{self.slot}", self._phi)

    @property
    def diff(self) -> np.ndarray:
        return self.sim._mirror(f"diff_{self.slot}", self._diff)

    @property
    def rhs(self) -> np.ndarray:
        return self.sim._mirror(f"rhs_{self.slot}", self._rhs)

    @property
    def phi_gpu(self):
        return self._phi

    def fill_ghosts(self) -> None:
        self.sim._scalar_fill_ghosts(self.slot)

    def dt_limit(self) -> float:
        g = self.sim.grid
        d = self.diff
        dmax = float(d[g.fluid].max()) if g.fluid.any() else self.D0
        if dmax <= 0:
            return np.inf
        return 0.5 / (dmax * (1.0 / g.dx ** 2 + 1.0 / g.dy ** 2))

    def cell(self) -> np.ndarray:
        return np.where(self.sim.grid.solid, np.nan, self.phi[1:-1, 1:-1])

    def total(self) -> float:
        g = self.sim.grid
        return float(np.nansum(self.cell()) * g.dx * g.dy)

    def wall_flux(self, side: str) -> np.ndarray:
        # cfd2d/models.py:226-250
        g = self.sim.grid
        phi, diff = self.phi, self.diff
        code, val = self.bt[side], self.bv[side]
        if side == "left":
            inner, D, h = phi[1, 1:-1], diff[1, 1:-1], g.dx
        elif side == "right":
            inner, D, h = phi[g.nx, 1:-1], diff[g.nx, 1:-1], g.dx
        elif side == "bottom":
            inner, D, h = phi[1:-1, 1], diff[1:-1, 1], g.dy
        else:
            inner, D, h = phi[1:-1, g.ny], diff[1:-1, g.ny], g.dy
        q = np.zeros_like(inner)
        m = code == 1
        q[m] = -D[m] * (val[m] - inner[m]) / (0.5 * h)
        m2 = code == 2
        q[m2] = -val[m2]
        return q


class Model:
    """Base of the built-in models (hook names as cfd2d/models.py:256-290)."""

    kind = "model"
    title = "Modell"

    def attach(self, sim) -> None:
        self.sim = sim

    def dt_limit(self, sim):
        return None

    def monitors(self, sim) -> dict:
        return {}

    def fields(self, sim) -> dict:
        return {}

    def device_fields(self, sim):
        """{key: (label, CFD2D_FIELD_* kind, device tensor)} of the fields() this model
        offers, read on the device by the function objects; None when the model has
        only host fields (they are then uploaded when sampled)."""
        return None

    def device_monitors(self, sim):
        """[(key, cfd2d_monitor)] of the monitors() this model records in the history
        after every step, evaluated on the device; None: not recorded per step."""
        return None

    def state(self) -> dict:
        return {}

    def set_state(self, sim, state: dict) -> None:
        pass

    def describe(self) -> str:
        return self.title


class PassiveScalar(Model):
    """Passive scalar (cfd2d/models.py:296-333)."""

    kind = "scalar"

    def __init__(self, name: str = "c", diffusivity: float = 1e-3, bcs: dict | None = None,
                 obstacle: ScalarBC | None = None, limiter: str = "vanleer", initial=0.0,
                 source=None, turbulent_schmidt: float = 0.7, label: str | None = None):
        self.field = ScalarField(name, diffusivity, bcs, obstacle, limiter, initial, source,
                                 label=label or f"Skalar {name}")
        self.title = f"Passiver Skalar '{name}' (D = {diffusivity:g}, {limiter})"
        self.sct = turbulent_schmidt
        self.name = name

    def attach(self, sim) -> None:
        super().attach(sim)
        self.field.turb_number = float(self.sct)
        self.field.attach(sim)
        sim.scalars[self.name] = self.field

    def dt_limit(self, sim):
        lim = self.field.dt_limit()
        return lim if np.isfinite(lim) else None

    def monitors(self, sim) -> dict:
        return {f"{self.name}_integral": self.field.total()}

    def fields(self, sim) -> dict:
        return {self.name: (self.field.label, self.field.cell())}

    def device_fields(self, sim):
        return {self.name: (self.field.label, _lib.FIELD_CELL, self.field._phi)}

    def device_monitors(self, sim):
        return [(f"{self.name}_integral", _lib.Monitor(_lib.MON_SUM_FLUID, 0, 0, 0, self.field._phi.data_ptr(), 0.0))]


class BoussinesqTemperature(Model):
    """Temperature with Boussinesq buoyancy (cfd2d/models.py:339-426)."""

    kind = "thermal"

    def __init__(self, alpha: float, bcs: dict | None = None, gravity=(0.0, -1.0), T_ref: float = 0.0,
                 initial=0.0, obstacle: ScalarBC | None = None, limiter: str = "vanleer",
                 prandtl_turbulent: float = 0.85, buoyancy: bool = True):
        self.field = ScalarField("T", alpha, bcs, obstacle, limiter, initial, label="Temperatur T")
        self.alpha = float(alpha)
        self.gravity = (float(gravity[0]), float(gravity[1]))
        self.T_ref = float(T_ref)
        self.prt = prandtl_turbulent
        self.buoyancy = buoyancy
        self.title = (f"Temperatur (alpha = {alpha:.4g}"
                      + (f", Auftrieb beta*g = {self.gravity}" if buoyancy else ", ohne Auftrieb") + ")")

    @property
    def T(self) -> np.ndarray:
        return self.field.phi

    def attach(self, sim) -> None:
        super().attach(sim)
        self.field.turb_number = float(self.prt)
        self.field.attach(sim)
        sim.scalars["T"] = self.field
        if self.buoyancy:
            sim._set_thermal(self.field.slot, self.gravity, self.T_ref)

    def dt_limit(self, sim):
        lim = self.field.dt_limit()
        return lim if np.isfinite(lim) else None

    def nusselt(self, side: str, L: float = 1.0, dT: float = 1.0):
        if not np.any(self.field.bt[side] == 1):
            return None
        q = self.field.wall_flux(side)
        return abs(float(np.mean(q))) * L / (self.alpha * dT) if q.size else None

    def local_nusselt(self, side: str, L: float = 1.0, dT: float = 1.0) -> np.ndarray:
        return np.abs(self.field.wall_flux(side)) * L / (self.alpha * dT)

    def monitors(self, sim) -> dict:
        out = {"T_mittel": float(np.nanmean(self.field.cell()))}
        for side in SIDES:
            nu = self.nusselt(side)
            if nu is not None:
                out[f"Nu_{side}"] = nu
        return out

    def fields(self, sim) -> dict:
        return {"T": ("Temperatur T", self.field.cell())}

    def device_fields(self, sim):
        return {"T": ("Temperatur T", _lib.FIELD_CELL, self.field._phi)}

    def device_monitors(self, sim):
        ptr = self.field._phi.data_ptr()
        out = [("T_mittel", _lib.Monitor(_lib.MON_MEAN_FLUID, 0, 0, 0, ptr, 0.0))]
        for k, side in enumerate(SIDES):
            if np.any(self.field.bt[side] == 1):
                out.append((f"Nu_{side}", _lib.Monitor(_lib.MON_NUSSELT, self.field.slot, k, 0, ptr, self.alpha)))
        return out

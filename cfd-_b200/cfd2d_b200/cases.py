"""Predefined cases and the JSON case spec (drop-in for cfd2d/cases.py).

Each factory sets up the same grid, obstacles, boundary conditions and viscosity
as its counterpart in the reference (cfd2d/cases.py:60-379); the simulation it
returns runs on the GPU. The two-phase dam break (VOF) is not part of this path.
"""

from __future__ import annotations

import json
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import geometry
from .boundary import BoundaryCondition as BC
from .grid import Grid
from .models import BoussinesqTemperature, PassiveScalar, ScalarBC, default_scalar_bcs
from .solver import Simulation


@dataclass
class Case:
    """A fully set-up case (cfd2d/cases.py:20-48)."""

    key: str
    title: str
    sim: Simulation
    t_end: float
    steady_tol: float | None
    U_ref: float
    L_ref: float
    re: float
    info: dict = field(default_factory=dict)
    spec: dict | None = None

    def describe(self) -> str:
        s = [f"=== {self.title} ===",
             f"Reynolds-Zahl Re = {self.re:g} (U_ref = {self.U_ref:g}, L_ref = {self.L_ref:g})",
             f"Endzeit t_end = {self.t_end:g}"
             + (f", stationäres Abbruchkriterium: Residuum < {self.steady_tol:g}" if self.steady_tol else ""),
             self.sim.summary()]
        if self.sim.models:
            s.append("Modelle:")
            s += [f"  - {m.describe()}" for m in self.sim.models]
        return "\n".join(s)


_NUMERIC_KEYS = ("scheme", "gamma", "tau", "dt", "pressure_solver")


def _numerics(kw: dict) -> dict:
    """The numerical settings among the keyword arguments (cfd2d/cases.py:51-54)."""
    return {k: kw[k] for k in _NUMERIC_KEYS if kw.get(k) is not None}


def lid_driven_cavity(re: float = 100.0, n: int = 64, t_end: float = 50.0,
                      steady_tol: float | None = 1e-5, **num) -> Case:
    """Unit box with a lid moving at U = 1 (cfd2d/cases.py:60-70)."""
    grid = Grid(n, n, 1.0, 1.0)
    bcs = {"left": BC("noslip"), "right": BC("noslip"), "bottom": BC("noslip"),
           "top": BC("noslip", velocity=1.0)}
    sim = Simulation(grid, bcs, nu=1.0 / re, **_numerics(num))
    return Case("cavity", "Lid-Driven Cavity", sim, t_end, steady_tol, 1.0, 1.0, re)


CYLINDER_REFERENCE = {
    20: {"cd": (5.57, 5.59), "cl": (0.0104, 0.0110), "typ": "stationär (Test 2D-1)"},
    100: {"cd_max": (3.22, 3.24), "cl_max": (0.99, 1.01), "st": (0.295, 0.305),
          "typ": "periodisch (Test 2D-2)"},
}


def cylinder_flow(re: float = 100.0, nx: int = 440, ny: int = 82, t_end: float = 8.0,
                  profile: str = "parabolic", length: float = 2.2, **num) -> Case:
    """Channel 2.2 x 0.41 with a cylinder D = 0.1 at (0.2, 0.2) (cfd2d/cases.py:84-104)."""
    H, D, xc, yc = 0.41, 0.1, 0.2, 0.2
    grid = Grid(nx, ny, length, H)
    grid.add_obstacle(geometry.circle(grid, xc, yc, D / 2))
    bcs = {"left": BC("inflow", velocity=1.0, profile=profile), "right": BC("outflow"),
           "bottom": BC("noslip"), "top": BC("noslip")}
    sim = Simulation(grid, bcs, nu=1.0 * D / re, compute_forces=True, initial_velocity=(0.0, 0.0),
                     **_numerics(num))
    info = {"D": D, "xc": xc, "yc": yc, "H": H}
    ref = CYLINDER_REFERENCE.get(int(round(re))) if profile == "parabolic" and length == 2.2 else None
    if ref:
        info["referenz"] = ref
    return Case("cylinder", "Zylinderumströmung (Schäfer-Turek-Kanal)", sim, t_end, None, 1.0, D, re, info)


def channel_flow(re: float = 20.0, length: float = 6.0, ny: int = 32, nx: int | None = None,
                 profile: str = "uniform", t_end: float = 40.0, steady_tol: float | None = 1e-5,
                 **num) -> Case:
    """Plane channel H = 1, mean velocity 1 (cfd2d/cases.py:110-127)."""
    if nx is None:
        nx = int(round(length * ny))
    grid = Grid(nx, ny, length, 1.0)
    bcs = {"left": BC("inflow", velocity=1.0, profile=profile), "right": BC("outflow"),
           "bottom": BC("noslip"), "top": BC("noslip")}
    sim = Simulation(grid, bcs, nu=1.0 / re, initial_velocity=(1.0, 0.0), **_numerics(num))
    info = {"H": 1.0, "einlauflaenge": 0.05 * re}
    return Case("channel", "Kanalströmung (Poiseuille)", sim, t_end, steady_tol, 1.0, 1.0, re, info)


def backward_facing_step(re: float = 400.0, length: float = 15.0, ny: int = 40, nx: int | None = None,
                         inlet_length: float = 1.0, t_end: float = 100.0,
                         steady_tol: float | None = 1e-5, **num) -> Case:
    """Channel H = 1 with a step of height H/2 (cfd2d/cases.py:133-155)."""
    H, h = 1.0, 0.5
    if nx is None:
        nx = int(round(length / H * ny))
    grid = Grid(nx, ny, length, H)
    if inlet_length > 0:
        grid.add_obstacle(geometry.rectangle(grid, 0.0, 0.0, inlet_length, h))
    bcs = {"left": BC("inflow", velocity=1.0, profile="parabolic"), "right": BC("outflow"),
           "bottom": BC("noslip"), "top": BC("noslip")}
    sim = Simulation(grid, bcs, nu=1.0 * H / re, **_numerics(num))
    info = {"H": H, "h": h, "x_stufe": inlet_length}
    return Case("step", "Rückwärtsgewandte Stufe (Backward-Facing Step)", sim, t_end, steady_tol,
                1.0, H, re, info)


def custom_obstacles(obstacles: list, lx: float = 4.0, ly: float = 1.0, nx: int = 320, ny: int = 80,
                     re: float = 100.0, U: float = 1.0, L_ref: float | None = None,
                     inflow_profile: str = "uniform", walls: str = "slip", t_end: float = 10.0,
                     bcs: dict | None = None, steady_tol: float | None = None,
                     flow_rate: float | None = None, **num) -> Case:
    """Channel with arbitrary obstacles (cfd2d/cases.py:161-201)."""
    grid = Grid(nx, ny, lx, ly)
    for spec in obstacles:
        grid.add_obstacle(geometry.build_obstacle(grid, spec))
    if L_ref is None:
        solid = grid.solid
        L_ref = solid.any(axis=0).sum() * grid.dy if solid.any() else ly
    if bcs is None:
        bcs = {"left": BC("inflow", velocity=U, profile=inflow_profile), "right": BC("outflow"),
               "bottom": BC(walls), "top": BC(walls)}
    else:
        bcs = {k: (BC(**b) if isinstance(b, dict) else b) for k, b in bcs.items()}
    sim = Simulation(grid, bcs, nu=U * L_ref / re, compute_forces=bool(obstacles), flow_rate=flow_rate,
                     initial_velocity=(U, 0.0) if flow_rate is not None else (0.0, 0.0), **_numerics(num))
    info = {"hindernisse": obstacles, "L_ref": L_ref}
    return Case("custom", "Eigene Hindernisse", sim, t_end, steady_tol, U, L_ref, re, info)


def random_obstacles(rng, lx: float = 2.0, ly: float = 1.0, nmin: int = 2, nmax: int = 12) -> list:
    """Seeded obstacle list of the obstacle-flow workload: 2-12 circles, ellipses or
    rectangles (``custom_obstacles`` specs), centres uniform in the middle 70 % of
    each side, sizes (radius, semi-axis, half-width) uniform in 0.02-0.08 of the
    domain height. Draws from ``rng`` in a fixed order, so a seed names the list."""
    specs = []
    for _ in range(int(rng.integers(nmin, nmax + 1))):
        kind = rng.integers(0, 3)
        x = float(rng.uniform(0.15 * lx, 0.85 * lx))
        y = float(rng.uniform(0.15 * ly, 0.85 * ly))
        size = float(rng.uniform(0.02, 0.08) * ly)
        if kind == 0:
            specs.append({"typ": "kreis", "x": x, "y": y, "r": size})
        elif kind == 1:
            specs.append({"typ": "ellipse", "x": x, "y": y, "a": size, "b": size * float(rng.uniform(0.4, 1.0)),
                          "winkel": float(rng.uniform(0, 180))})
        else:
            specs.append({"typ": "rechteck", "x0": x - size, "y0": y - 0.6 * size, "x1": x + size,
                          "y1": y + 0.6 * size})
    return specs


def random_obstacle_spec(rng, lx: float = 2.0, ly: float = 1.0) -> tuple[list, float]:
    """(obstacles, Re) of one seeded obstacle flow: Re log-uniform in 200-2000 (drawn
    first), then ``random_obstacles``."""
    re = float(np.exp(rng.uniform(np.log(200.0), np.log(2000.0))))
    return random_obstacles(rng, lx, ly), re


def random_obstacle_flow(rng, nx: int, ny: int, lx: float = 2.0, ly: float = 1.0, **num) -> Case:
    """One seeded obstacle flow: ``custom_obstacles`` with a block inflow U = 1,
    outflow p = 0, slip walls and the obstacles and Re of ``random_obstacle_spec``."""
    obstacles, re = random_obstacle_spec(rng, lx, ly)
    return custom_obstacles(obstacles, lx=lx, ly=ly, nx=nx, ny=ny, re=re, inflow_profile="uniform",
                            walls="slip", **num)


def obstacle_flow(seed: int = 13, nx: int = 1024, ny: int = 512, **num) -> Case:
    """The obstacle-flow benchmark case: ``random_obstacle_flow`` on a 2 x 1 domain
    drawn from ``np.random.default_rng(seed)``."""
    return random_obstacle_flow(np.random.default_rng(seed), nx, ny, **num)


def heated_cavity(ra: float = 1e4, pr: float = 0.71, n: int = 48, t_end: float = 500.0,
                  steady_tol: float | None = 1e-6, limiter: str = "vanleer", **num) -> Case:
    """Differentially heated square cavity (cfd2d/cases.py:207-223)."""
    grid = Grid(n, n, 1.0, 1.0)
    bcs = {s: BC("noslip") for s in ("left", "right", "bottom", "top")}
    thermal = BoussinesqTemperature(
        alpha=1.0 / np.sqrt(ra * pr), limiter=limiter,
        bcs={"left": ScalarBC("fixed", 0.5), "right": ScalarBC("fixed", -0.5),
             "bottom": ScalarBC("zerogradient"), "top": ScalarBC("zerogradient")})
    sim = Simulation(grid, bcs, nu=np.sqrt(pr / ra), models=[thermal], **_numerics(num))
    info = {"ra": ra, "pr": pr, "geschw_skala_alpha": np.sqrt(ra * pr)}
    return Case("heated_cavity", "Beheizte Cavity (natürliche Konvektion)", sim, t_end, steady_tol,
                1.0, 1.0, float(np.sqrt(ra / pr)), info)


def rayleigh_benard(ra: float = 1e4, pr: float = 0.71, aspect: float = 4.032, ny: int = 24,
                    nx: int | None = None, t_end: float = 300.0, steady_tol: float | None = 1e-6,
                    seed: int = 1, limiter: str = "vanleer", **num) -> Case:
    """Fluid layer heated from below, periodic in x (cfd2d/cases.py:229-252)."""
    if nx is None:
        nx = int(round(aspect * ny))
    grid = Grid(nx, ny, aspect, 1.0)
    bcs = {"left": BC("periodic"), "right": BC("periodic"), "bottom": BC("noslip"), "top": BC("noslip")}
    rng = np.random.default_rng(seed)
    X, Y = grid.cell_centers()
    T0 = 0.5 - Y + 0.01 * rng.standard_normal(X.shape) * np.sin(np.pi * Y)
    thermal = BoussinesqTemperature(alpha=1.0 / np.sqrt(ra * pr), initial=T0, limiter=limiter,
                                    bcs={"bottom": ScalarBC("fixed", 0.5), "top": ScalarBC("fixed", -0.5)})
    sim = Simulation(grid, bcs, nu=np.sqrt(pr / ra), models=[thermal], **_numerics(num))
    info = {"ra": ra, "pr": pr, "ra_krit": 1707.76}
    return Case("rayleigh_benard", "Rayleigh-Bénard-Konvektion", sim, t_end, steady_tol, 1.0, 1.0,
                float(np.sqrt(ra / pr)), info)


def dean_cf(re_b: float) -> float:
    """Dean (1978): Cf = 0.073 Re_b^(-1/4) (cfd2d/cases.py:258-260)."""
    return 0.073 * re_b ** -0.25


def turbulent_channel(re_tau: float = 180.0, ny: int | None = None, y_plus_1: float = 1.0,
                      model: str = "kOmegaSST", t_end: float = 400.0, steady_tol: float | None = 1e-6,
                      **num) -> Case:
    """Periodic channel, half height 1, bulk velocity 1 (cfd2d/cases.py:263-288)."""
    from .turbulence import TURBULENCE_MODELS

    re_b = (re_tau / 0.09) ** (1 / 0.88)
    nu = 2.0 / re_b
    if ny is None:
        ny = int(np.ceil(re_tau / y_plus_1))
        ny += ny % 2
    grid = Grid(4, ny, 0.5, 2.0)
    bcs = {"left": BC("periodic"), "right": BC("periodic"), "bottom": BC("noslip"), "top": BC("noslip")}
    cls = TURBULENCE_MODELS[model]
    models = [cls(intensity=0.05, viscosity_ratio=50.0)] if model == "kOmegaSST" else ([cls()] if cls else [])
    sim = Simulation(grid, bcs, nu=nu, flow_rate=1.0, initial_velocity=(1.0, 0.0), models=models,
                     **_numerics(num))
    info = {"re_tau_soll": re_tau, "re_b": re_b, "cf_dean": dean_cf(re_b), "modell": model}
    return Case("turbulent_channel", "Turbulente Kanalströmung (RANS)", sim, t_end, steady_tol,
                1.0, 2.0, re_b, info)


def dam_break(n: int = 96, size: float = 0.584, column_width: float = 0.1461,
              column_height: float = 0.292, obstacle: bool = True, sigma: float = 0.07,
              t_end: float = 1.0, open_top: bool = True, **num) -> Case:
    """Dam break in a square tank, water and air in SI units (cfd2d/cases.py:294-320):
    a 0.1461 m x 0.292 m water column at the left wall (Martin & Moyce 1952), an
    optional 0.024 m x 0.048 m obstacle on the floor, the top open (p = 0) or closed."""
    from .vof import VOF

    grid = Grid(n, n, size, size)
    if obstacle:
        x0 = 0.5 * size - 0.012
        grid.add_obstacle(geometry.rectangle(grid, x0, 0.0, x0 + 0.024, 0.048))
    X, Y = grid.cell_centers()
    alpha0 = ((X <= column_width) & (Y <= column_height)).astype(float)
    bcs = {"left": BC("noslip"), "right": BC("noslip"), "bottom": BC("noslip"),
           "top": BC("outflow") if open_top else BC("noslip")}
    vof = VOF(alpha0, sigma=sigma)
    num.setdefault("gamma", 0.5)
    sim = Simulation(grid, bcs, nu=1e-6, models=[vof], **_numerics(num))
    info = {"a": column_width, "h0": column_height, "g": 9.81}
    U = np.sqrt(2 * 9.81 * column_height)
    return Case("dam_break", "Dammbruch (VOF, Wasser/Luft)", sim, t_end, None, U, column_width,
                float(U * column_width / 1e-6), info)


def add_turbulence(case: Case, model: str = "kOmegaSST", **kw) -> Case:
    """Add a turbulence model (cfd2d/cases.py:326-337)."""
    from .turbulence import TURBULENCE_MODELS

    cls = TURBULENCE_MODELS[model]
    if cls is None:
        return case
    if model == "kOmegaSST":
        kw.setdefault("U_ref", case.U_ref)
    case.sim.add_model(cls(**kw))
    case.info["turbulenz"] = model
    return case


def add_temperature(case: Case, alpha: float, T_inflow: float = 0.0, T_obstacle: float | None = None,
                    wall_temperatures: dict | None = None, buoyancy: bool = False,
                    gravity=(0.0, -1.0), limiter: str = "vanleer") -> Case:
    """Add temperature transport, optionally with buoyancy (cfd2d/cases.py:340-356)."""
    bcs = default_scalar_bcs(case.sim, T_inflow)
    for side, T in (wall_temperatures or {}).items():
        bcs[side] = ScalarBC("fixed", T)
    obs = ScalarBC("fixed", T_obstacle) if T_obstacle is not None else ScalarBC("zerogradient")
    case.sim.add_model(BoussinesqTemperature(alpha, bcs, gravity=gravity, obstacle=obs, limiter=limiter,
                                             buoyancy=buoyancy, initial=T_inflow))
    return case


def add_scalar(case: Case, name: str = "c", diffusivity: float = 1e-3, inflow_value=1.0,
               inflow_band: tuple | None = None, obstacle_value: float | None = None,
               limiter: str = "vanleer") -> Case:
    """Add a passive scalar; inflow_band (s0, s1) restricts the inflow value to a strip
    of the inflow side (cfd2d/cases.py:359-379)."""
    bcs = default_scalar_bcs(case.sim, 0.0)
    for bc in bcs.values():
        if bc.kind == "fixed":
            if inflow_band is None:
                bc.value = inflow_value
            else:
                a, b = inflow_band
                bc.value = lambda s, a=a, b=b: np.where((s >= a) & (s <= b), inflow_value, 0.0)
    obs = ScalarBC("fixed", obstacle_value) if obstacle_value is not None else None
    case.sim.add_model(PassiveScalar(name, diffusivity, bcs, obs, limiter))
    return case


CASES = {
    "cavity": lid_driven_cavity, "cylinder": cylinder_flow, "channel": channel_flow,
    "step": backward_facing_step, "custom": custom_obstacles, "heated_cavity": heated_cavity,
    "rayleigh_benard": rayleigh_benard, "turbulent_channel": turbulent_channel, "dam_break": dam_break,
}

CASE_TITLES = {
    "cavity": "Lid-Driven Cavity", "cylinder": "Zylinderumströmung (Schäfer-Turek)",
    "channel": "Kanalströmung (Poiseuille)", "step": "Rückwärtsgewandte Stufe",
    "custom": "Eigene Hindernisse", "heated_cavity": "Beheizte Cavity (natürliche Konvektion, de Vahl Davis)",
    "rayleigh_benard": "Rayleigh-Bénard-Konvektion", "turbulent_channel": "Turbulenter Kanal (RANS k-ω SST)",
    "dam_break": "Dammbruch (Zweiphasen-VOF)",
}


def build_case(spec: dict) -> Case:
    """Build a case from a spec dict (cfd2d/cases.py:411-442)."""
    key = spec["fall"]
    if key not in CASES:
        raise ValueError(f"Unbekannter Fall {key!r}, erlaubt: {list(CASES)}")
    params = dict(spec.get("parameter", {}))
    num = dict(spec.get("numerik", {}))
    case = CASES[key](**params, **num)
    turb = spec.get("turbulenz")
    if turb and turb.get("modell", "laminar") != "laminar":
        add_turbulence(case, turb["modell"], **{k: v for k, v in turb.items() if k != "modell"})
    if spec.get("temperatur"):
        add_temperature(case, **spec["temperatur"])
    if spec.get("skalar"):
        sk = dict(spec["skalar"])
        if sk.get("inflow_band") is not None:
            sk["inflow_band"] = tuple(sk["inflow_band"])
        add_scalar(case, **sk)
    case.spec = spec
    return case


def save_case(spec: dict, path) -> None:
    Path(path).parent.mkdir(parents=True, exist_ok=True)
    with open(path, "w", encoding="utf-8") as f:
        json.dump(spec, f, indent=2, ensure_ascii=False, default=float)


def load_case(path) -> dict:
    with open(path, encoding="utf-8") as f:
        return json.load(f)

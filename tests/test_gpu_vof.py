"""Two-phase VOF on the device (cfd2d_b200.vof) against the reference (GPU).

Kernel level: the alpha transport bit for bit against the reference's Numba
vof_advect on seeded inputs; the variable-coefficient pressure solve against the
reference's sparse direct solve. Step level: the 32 x 32 dam break (CSF surface
tension, mixture density, variable-density projection, sub-stepped transport)
against the reference's run. The reference's own VOF tests are mirrored.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden

pytestmark = [pytest.mark.gpu, pytest.mark.filterwarnings("ignore::RuntimeWarning")]


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    s = np.abs(b).max()
    return np.abs(a - b).max() / s if s > 0 else np.abs(a - b).max()


def test_vof_advect_bitwise(cuda_lib):
    from inputs import vof_cases

    from cfd2d_b200 import vof

    g = golden("golden_vof")
    k = 0
    for c in vof_cases():
        out = np.full_like(c["a"], 5.0)
        vof.vof_advect(c["a"], c["u"], c["v"], c["fluid"], c["nx"], c["ny"], c["dx"], c["dy"], c["dt"],
                       c["c_alpha"], c["periodic"], c["a_in"], out)
        assert np.array_equal(out, g[f"adv{k}_out"]), k
        k += 1
    assert k == int(g["n_adv"])


def _sims():
    from cfd2d_b200 import geometry
    from cfd2d_b200.boundary import BoundaryCondition as BC
    from cfd2d_b200.grid import Grid
    from cfd2d_b200.solver import Simulation

    sims = {}
    grid = Grid(30, 20, 1.5, 1.0)
    grid.add_obstacle(geometry.rectangle(grid, 0.7, -1.0, 0.8, 2.0))
    sims["two"] = Simulation(grid, {s: BC("noslip") for s in ("left", "right", "bottom", "top")}, nu=0.02)
    grid = Grid(32, 32, 0.584, 0.584)
    grid.add_obstacle(geometry.rectangle(grid, 0.28, 0.0, 0.304, 0.048))
    sims["open"] = Simulation(grid, {"left": BC("noslip"), "right": BC("noslip"), "bottom": BC("noslip"),
                                     "top": BC("outflow")}, nu=1e-6)
    grid = Grid(32, 24, 1.0, 0.75)
    grid.add_obstacle(geometry.circle(grid, 0.5, 0.4, 0.12))
    sims["per"] = Simulation(grid, {"left": BC("periodic"), "right": BC("periodic"), "bottom": BC("noslip"),
                                    "top": BC("slip")}, nu=0.01)
    return sims


@pytest.mark.parametrize("name", ["two", "open", "per"])
def test_solve_variable_against_direct(cuda_lib, name):
    """PressureSolver.solve_variable (cfd2d/pressure.py:187-244) with a 1000:1
    density interface: two Neumann components, an open top, periodic x."""
    g = golden("golden_vof")
    sim = _sims()[name]
    rho = g[f"sv_{name}_rho"]
    nx = sim.grid.nx
    bx = 2.0 / (rho[:-1, :] + rho[1:, :])
    by = 2.0 / (rho[:, :-1] + rho[:, 1:])
    if sim.periodic:
        bx[nx, :] = 2.0 / (rho[nx, :] + rho[1, :])
    p = sim.pressure.solve_variable(g[f"sv_{name}_rhs"], bx[:, 1:-1], by[1:-1, :])
    assert rel(p, g[f"sv_{name}_p"]) < 1e-9, name


def test_dam_break_against_reference(cuda_lib):
    """cfd2d/cases.py:294-320 on 32 x 32, 20 steps: u, v, p, alpha and the dt series."""
    from cfd2d_b200 import cases

    g = golden("golden_vof")
    case = cases.dam_break(n=32)
    sim = case.sim
    vof = sim.model("multiphase")
    sim.step()
    for f in "uvp":
        assert rel(getattr(sim, f), g[f"dam_{f}_1"]) < 1e-9, f
    assert rel(vof.alpha, g["dam_alpha_1"]) < 1e-9
    sim.advance(19)
    for f in "uvp":
        assert rel(getattr(sim, f), g[f"dam_{f}_20"]) < 1e-8, f
    assert rel(vof.alpha, g["dam_alpha_20"]) < 1e-8
    assert rel(sim.history.dt, g["dam_dt"]) < 1e-10
    assert vof.volume() == pytest.approx(float(g["dam_volume"]), rel=1e-10)


def test_vof_hydrostatic_rest(cuda_lib):
    # tests/test_models.py:135-150
    from cfd2d_b200.boundary import BoundaryCondition as BC
    from cfd2d_b200.grid import Grid
    from cfd2d_b200.solver import Simulation
    from cfd2d_b200.vof import VOF

    grid = Grid(20, 20, 0.2, 0.2)
    X, Y = grid.cell_centers()
    alpha0 = (Y < 0.1).astype(float)
    bcs = {s: BC("noslip") for s in ("left", "right", "bottom")}
    bcs["top"] = BC("outflow")
    vof = VOF(alpha0, sigma=0.0)
    sim = Simulation(grid, bcs, nu=1e-6, models=[vof])
    sim.run(0.2, verbose=False)
    uc, vc = sim.cell_velocity()
    assert np.nanmax(np.hypot(uc, vc)) < 1e-6
    p_bottom = sim.cell_pressure()[10, 0]
    assert p_bottom == pytest.approx(1000 * 9.81 * (0.1 - 0.005), rel=0.02)
    assert abs(vof.volume() / vof.volume0 - 1) < 1e-10


def test_dam_break_runs_conserves_volume(cuda_lib):
    # tests/test_models.py:153-162 (front position from the model's monitors)
    from cfd2d_b200 import cases

    case = cases.dam_break(n=32, obstacle=True, t_end=0.15)
    case.sim.run(case.t_end, verbose=False)
    vof = case.sim.model("multiphase")
    assert abs(vof.volume() / vof.volume0 - 1) < 1e-3
    a = vof.alpha[1:-1, 1:-1]
    assert a.min() >= 0 and a.max() <= 1
    assert vof.monitors(case.sim)["front_x"] > case.info["a"] * 1.3
    assert case.sim.max_divergence() < 1e-8


def test_checkpoint_restart_vof(cuda_lib, tmp_path):
    # tests/test_functions.py:73-89
    from cfd2d_b200 import cases, functions

    spec = {"fall": "dam_break", "parameter": {"n": 24, "t_end": 0.1}}
    ref = cases.build_case(spec)
    for _ in range(30):
        ref.sim.step()
    a = cases.build_case(spec)
    for _ in range(15):
        a.sim.step()
    functions.save_checkpoint(a.sim, tmp_path / "cp.npz")
    b = cases.build_case(spec)
    functions.load_checkpoint(b.sim, tmp_path / "cp.npz")
    for _ in range(15):
        b.sim.step()
    va = b.sim.model("multiphase").alpha
    vr = ref.sim.model("multiphase").alpha
    assert np.allclose(va, vr, atol=1e-10)


def test_dam_break_96_100_steps(cuda_lib):
    """The reference's default dam break (96 x 96), 100 steps: the direct solve of the
    reference against the device PCG at rtol 1e-13 over a longer trajectory."""
    from cfd2d_b200 import cases

    g = golden("golden_vof")
    case = cases.dam_break(n=96)
    sim = case.sim
    vof = sim.model("multiphase")
    sim.advance(100)
    errs = {f: rel(getattr(sim, f), g[f"d96_{f}_100"]) for f in "uvp"}
    errs["alpha"] = rel(vof.alpha, g["d96_alpha_100"])
    errs["dt"] = rel(sim.history.dt, g["d96_dt"])
    assert max(errs.values()) < 1e-7, errs
    assert sim.history.extra["front_x"] == list(g["d96_extra_front_x"])

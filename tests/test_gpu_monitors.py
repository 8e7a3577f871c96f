"""Per-step model monitors in the history (cfd2d/solver.py:441-443) (GPU).

Every model's monitors are evaluated on the device after each step and appended to
``history.extra`` in the reference's order: scalar integrals, mean temperature and
Nusselt numbers, k mean and nu_t max, the VOF volume, its error, front position and
column height. Compared with the series the reference itself recorded (golden
fixtures); sums run in another order than numpy's pairwise ones.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden

pytestmark = [pytest.mark.gpu, pytest.mark.filterwarnings("ignore::RuntimeWarning")]


def _check(sim, g, prefix, tol=1e-9):
    keys = [k[len(prefix) + 7:] for k in g if k.startswith(prefix + "_extra_")]
    assert keys, prefix
    mine = [k for k in sim.history.extra if k in keys]
    assert mine == [k for k in sim.history.extra if k not in ("antriebskraft", "cg_iterationen")]
    for k in keys:
        a, b = np.asarray(sim.history.extra[k]), g[f"{prefix}_extra_{k}"]
        assert a.shape == b.shape, k
        # values that vanish up to rounding (the mean temperature of the antisymmetric
        # heated cavity, the relative volume error) are compared on the field's scale, 1
        scale = max(np.abs(b).max(), 1.0 if k in ("volumenfehler_rel", "T_mittel") else 1e-300)
        assert np.abs(a - b).max() / scale < tol, (k, np.abs(a - b).max())


def test_scalar_integral_cylinder(cuda_lib):
    from cfd2d_b200 import cases

    case = cases.build_case({"fall": "cylinder", "parameter": {"re": 100, "nx": 440, "ny": 82},
                             "numerik": {"pressure_solver": "cg"},
                             "skalar": {"name": "c", "diffusivity": 1e-3, "inflow_band": [0.15, 0.25],
                                        "limiter": "vanleer"}})
    case.sim.pressure.tol = 1e-8
    case.sim.advance(10)
    _check(case.sim, golden("golden_cylinder440"), "cyl")


def test_temperature_and_nusselt_heated_cavity(cuda_lib):
    from cfd2d_b200 import cases

    case = cases.heated_cavity(ra=1e5, n=32, pressure_solver="cg")
    case.sim.pressure.tol = 1e-8
    case.sim.advance(100)
    _check(case.sim, golden("golden_misc"), "hot")


def test_dam_break_monitors(cuda_lib):
    from cfd2d_b200 import cases

    case = cases.dam_break(n=32)
    case.sim.advance(20)
    _check(case.sim, golden("golden_vof"), "dam", tol=1e-8)
    vof = case.sim.model("multiphase")
    last = {k: v[-1] for k, v in case.sim.history.extra.items()}
    for k, v in vof.monitors(case.sim).items():
        assert last[k] == pytest.approx(v, rel=1e-12, abs=1e-14), k


@pytest.mark.parametrize("name", ["smc", "smy"])
def test_smagorinsky_monitors(cuda_lib, name):
    from cfd2d_b200 import cases

    if name == "smc":
        sim = cases.add_turbulence(cases.lid_driven_cavity(re=1000, n=32, pressure_solver="cg"),
                                   "Smagorinsky").sim
        n = 100
    else:
        case = cases.cylinder_flow(re=1000, nx=110, ny=21, pressure_solver="cg")
        cases.add_turbulence(case, "Smagorinsky", cs=0.1, wall_damping=False)
        cases.add_scalar(case, "c", 1e-4, inflow_band=(0.15, 0.25))
        sim = case.sim
        n = 30
    sim.pressure.tol = 1e-8
    sim.advance(n)
    _check(sim, golden("golden_smagorinsky"), name)

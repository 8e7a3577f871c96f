"""Mixed-precision pressure solve (FP32 iterations, FP64 refinement and reductions) (GPU).

No counterpart in the reference: the checks are against the FP64 solver of this
library, which is itself checked against the reference, and against the stop test
itself (the true residual is recomputed in FP64 on the host).
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu]


def _relerr(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _rhs(sim):
    g = sim.grid
    F, G = sim.F, sim.G
    return ((F[1:, 1:-1] - F[:-1, 1:-1]) / g.dx + (G[1:-1, 1:] - G[1:-1, :-1]) / g.dy) / sim.dt


@pytest.mark.parametrize("case_name", ["cylinder", "cavity"])
def test_mixed_solve_reaches_the_fp64_residual(cuda_lib, case_name):
    from cfd2d_b200 import cases

    if case_name == "cylinder":
        case = cases.cylinder_flow(re=100, nx=440, ny=82, pressure_solver="cg")
    else:  # all walls: one Neumann component, mean removed before and after
        case = cases.lid_driven_cavity(re=100, n=64, pressure_solver="cg")
    sim = case.sim
    ps = sim.pressure
    ps.tol = 1e-8
    sim.advance(3)
    rhs = _rhs(sim)
    zero = np.zeros(int(ps.fluid.sum()))
    ps._x0 = zero
    p64 = ps.solve(rhs)
    ps.precision = "mixed"
    ps._x0 = zero
    pmx = ps.solve(rhs)
    its = ps.last_iterations
    ps.precision = "fp64"
    assert its > 0
    assert _relerr(pmx, p64) < 1e-5
    # the stop test is the FP64 true residual: recompute it here
    A = ps.A
    b = -rhs[ps.fluid]
    if ps.neumann_components:
        b = b - b.mean()
    x = ps._x0
    assert np.linalg.norm(b - A @ x) <= 1.0001e-8 * np.linalg.norm(b)


def test_mixed_steps_track_the_fp64_steps(cuda_lib):
    """Cylinder 440 x 82 with the van Leer scalar: 200 steps in each precision from
    the same start; velocity, pressure, scalar and force coefficients agree to the
    solver tolerance."""
    from cfd2d_b200 import cases

    spec = {"fall": "cylinder", "parameter": {"re": 100, "nx": 440, "ny": 82},
            "numerik": {"pressure_solver": "cg"},
            "skalar": {"name": "c", "diffusivity": 1e-3, "inflow_band": [0.15, 0.25], "limiter": "vanleer"}}
    out = {}
    for prec in ("fp64", "mixed"):
        case = cases.build_case(spec)
        sim = case.sim
        sim.pressure.tol = 1e-8
        sim.pressure.precision = prec
        sim.advance(200)
        fx = np.array(sim.history.fx[-50:])
        out[prec] = (sim.u.copy(), sim.v.copy(), sim.p.copy(), sim.scalars["c"].phi.copy(), fx)
    (u0, v0, p0, c0, f0), (u1, v1, p1, c1, f1) = out["fp64"], out["mixed"]
    assert _relerr(u1, u0) < 1e-6 and _relerr(v1, v0) < 1e-6
    assert _relerr(p1, p0) < 1e-5 and _relerr(c1, c0) < 1e-6
    assert _relerr(f1, f0) < 1e-5

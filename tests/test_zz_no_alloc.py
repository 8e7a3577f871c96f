"""cfd2d_pressure_solve_static: the pressure solve with static scratch (GPU).

The entry point runs the grid-persistent solver on a workspace that is a static
device array of the library. It must give what cfd2d_pressure_solve gives on the
same operator, right-hand side and warm start, call after call (the second call
reuses the scratch the first one left behind), and reject grids above its capacity.
This file is collected last so that it also runs after every other GPU test.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu]

# same-kernel comparison: identical launch shape, so the results agree to rounding
SAME_VARIANT_RTOL = 1e-12
# against the solver's default (on-chip cluster) variant: another summation order
OTHER_VARIANT_RTOL = 1e-7


def _rhs(sim):
    g = sim.grid
    F, G = sim.F, sim.G
    return ((F[1:, 1:-1] - F[:-1, 1:-1]) / g.dx + (G[1:-1, 1:] - G[1:-1, :-1]) / g.dy) / sim.dt


def _solve(lib_fn, op, rhs_d, x0_d, start, rtol, maxiter, torch, _lib):
    x0_d.copy_(start)
    p = torch.empty_like(rhs_d)
    iters = torch.zeros(2, dtype=torch.int32, device=rhs_d.device)
    st = torch.zeros(1, dtype=torch.int32, device=rhs_d.device)
    rc = lib_fn(C.byref(op), _lib.ptr(rhs_d), _lib.ptr(p), rtol, maxiter, _lib.ptr(iters), _lib.ptr(st),
                _lib.stream_ptr())
    _lib.check(rc, lib_fn.__name__)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    return p.cpu().numpy(), x0_d.cpu().numpy(), int(iters[0].item())


def _relerr(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_static_scratch_solve_matches_pressure_solve_twice(cuda_lib):
    import torch

    from cfd2d_b200 import _lib, cases

    case = cases.cylinder_flow(re=100, nx=440, ny=82, pressure_solver="cg")
    sim = case.sim
    ps = sim.pressure
    ps.tol = 1e-8
    lib = _lib.lib()
    # the grid-persistent variant of the existing entry point, with a caller workspace
    work = torch.zeros(int(lib.cfd2d_pcg_workspace_bytes(ps.grid.nx, ps.grid.ny)) // 8, dtype=torch.float64,
                       device=_lib.device())
    op_grid = _lib.Poisson.from_buffer_copy(ps.op)
    op_grid.cluster = 0
    op_grid.work, op_grid.work_bytes = work.data_ptr(), work.numel() * 8
    op_default = _lib.Poisson.from_buffer_copy(ps.op)
    op_static = _lib.Poisson.from_buffer_copy(ps.op)
    op_static.work, op_static.work_bytes = 0, 0  # ignored by the static entry point
    x0_d = ps._d_x0
    prev = torch.zeros_like(x0_d)  # first call from a cold start
    for call in range(2):
        sim.advance(2)
        rhs_d = _lib.to_dev(_rhs(sim), torch.float64)
        # the second call starts from the first call's solution, a warm start that
        # is not yet the solution of this right-hand side
        start = prev.clone()
        p_s, x_s, it_s = _solve(lib.cfd2d_pressure_solve_static, op_static, rhs_d, x0_d, start, ps.rtol,
                                ps.maxiter, torch, _lib)
        p_g, x_g, it_g = _solve(lib.cfd2d_pressure_solve, op_grid, rhs_d, x0_d, start, ps.rtol, ps.maxiter,
                                torch, _lib)
        p_c, _, it_c = _solve(lib.cfd2d_pressure_solve, op_default, rhs_d, x0_d, start, ps.rtol, ps.maxiter,
                              torch, _lib)
        assert it_s > 0 and it_s == it_g, (call, it_s, it_g)
        assert _relerr(p_s, p_g) < SAME_VARIANT_RTOL, call
        assert _relerr(x_s, x_g) < SAME_VARIANT_RTOL, call
        assert abs(it_s - it_c) <= max(2, it_c // 20), (call, it_s, it_c)
        assert _relerr(p_s, p_c) < OTHER_VARIANT_RTOL, call
        prev = torch.from_numpy(x_s).to(x0_d.device)


def test_static_scratch_rejects_grids_above_capacity(cuda_lib):
    import torch

    from cfd2d_b200 import _lib

    lib = _lib.lib()
    dev = _lib.device()
    nx, ny = 513, 512  # one row above CFD2D_STATIC_MAX_CELLS = 512 * 512
    op = _lib.Poisson()
    op.nx, op.ny = nx, ny
    buf = torch.zeros(nx * ny, dtype=torch.float64, device=dev)
    rc = lib.cfd2d_pressure_solve_static(C.byref(op), _lib.ptr(buf), _lib.ptr(buf), 1e-8, 10, None, None,
                                         _lib.stream_ptr())
    assert rc == _lib.E_CAPACITY


@pytest.mark.parametrize("kind", ["variable_coefficients", "neumann_components"])
def test_static_scratch_other_operators(cuda_lib, kind):
    """The other operators the entry point accepts: variable face coefficients (the
    two-phase projection's, here random positive 1/rho on a cavity) and a domain with
    two Neumann-only components (walls all round, split by a solid column), each
    against cfd2d_pressure_solve's grid-persistent form on a caller workspace, two
    calls in a row."""
    import torch

    from cfd2d_b200 import _lib, geometry
    from cfd2d_b200.boundary import BoundaryCondition as BC
    from cfd2d_b200.grid import Grid
    from cfd2d_b200.solver import Simulation

    nx, ny = 96, 80
    grid = Grid(nx, ny, 1.2, 1.0)
    if kind == "neumann_components":
        grid.add_obstacle(geometry.rectangle(grid, 0.58, -1.0, 0.62, 2.0))
    bcs = {s: BC("noslip") for s in ("left", "right", "bottom", "top")}
    sim = Simulation(grid, bcs, nu=0.01, pressure_solver="cg")
    ps = sim.pressure
    ps.tol = 1e-10
    ps.ensure_workspace()
    rng = np.random.default_rng(5)
    keep = []
    if kind == "variable_coefficients":
        bx = rng.uniform(0.001, 1.0, (nx + 1, ny))
        by = rng.uniform(0.001, 1.0, (nx, ny + 1))
        op, keep = ps.variable_operator(bx, by)
        x0_d = keep[-1].view(-1)
    else:
        assert len(ps.neumann_components) == 2
        op = _lib.Poisson.from_buffer_copy(ps.op)
        x0_d = ps._d_x0.view(-1)
    lib = _lib.lib()
    work = torch.zeros(int(lib.cfd2d_pcg_workspace_bytes(nx, ny)) // 8, dtype=torch.float64, device=_lib.device())
    op_grid = _lib.Poisson.from_buffer_copy(op)
    op_grid.cluster, op_grid.grid_ctas = 0, 0
    op_grid.work, op_grid.work_bytes = work.data_ptr(), work.numel() * 8
    op_static = _lib.Poisson.from_buffer_copy(op)
    op_static.work, op_static.work_bytes = 0, 0
    start = torch.zeros_like(x0_d)
    for call in range(2):
        rhs = rng.standard_normal((nx, ny)) * grid.fluid_interior
        rhs_d = _lib.to_dev(rhs, torch.float64)
        p_s, x_s, it_s = _solve(lib.cfd2d_pressure_solve_static, op_static, rhs_d, x0_d, start.clone(), 1e-10,
                                20000, torch, _lib)
        p_g, x_g, it_g = _solve(lib.cfd2d_pressure_solve, op_grid, rhs_d, x0_d, start.clone(), 1e-10, 20000,
                                torch, _lib)
        assert it_s > 0 and it_s == it_g, (kind, call, it_s, it_g)
        assert _relerr(p_s, p_g) < SAME_VARIANT_RTOL, (kind, call)
        assert _relerr(x_s, x_g) < SAME_VARIANT_RTOL, (kind, call)
        start = torch.from_numpy(x_s).to(x0_d.device).view_as(x0_d)
    del keep

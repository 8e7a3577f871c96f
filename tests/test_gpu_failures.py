"""Failure detection without a GPU fault (GPU).

Every failure is made on the host or by a wait that nothing releases: a non-finite
value written into the velocity field (FloatingPointError, as cfd2d/solver.py:395-399),
an exhausted CG (the reference's warning, cfd2d/pressure.py:174-176), a flexible CG
with an untrained network (it stalls and the plain solver finishes the solve), and
the bounded grid barrier of the persistent solvers left without its peers (it gives
up, sets the timeout status and the context stays usable).
"""

from __future__ import annotations

import ctypes as C
import warnings

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu]


def test_nonfinite_velocity_raises_floating_point_error(cuda_lib):
    from cfd2d_b200 import cases

    case = cases.lid_driven_cavity(re=100, n=16)
    case.sim.advance(3)
    u = case.sim.u
    u[5, 5] = np.nan
    with pytest.raises(FloatingPointError):
        case.sim.step()


def test_exhausted_cg_warns_and_keeps_running(cuda_lib):
    from cfd2d_b200 import cases

    case = cases.lid_driven_cavity(re=100, n=256, pressure_solver="cg")
    sim = case.sim
    sim.pressure.tol = 1e-8
    sim.advance(3)
    # far below what 5000 Jacobi-PCG iterations reach on 256 x 256 (and above the range
    # where the squared residual would underflow): the CG runs to its 5000 iterations
    sim.pressure.tol = 1e-100
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        sim.step()
    its = sim.history.extra["cg_iterationen"][-1]
    assert any("nicht konvergiert" in str(x.message) for x in w), its
    assert its == sim.pressure.maxiter == 5000
    assert np.isfinite(sim.u).all()


def test_untrained_network_stalls_and_the_plain_solver_finishes(cuda_lib):
    from cfd2d_b200 import _lib, learned

    out = {}
    for mode in ("plain", "random"):
        rng = np.random.default_rng(7)
        sim = learned.obstacle_case(rng, 128, 64).sim
        sim.pressure.tol = 1e-8
        sim.advance(5)
        if mode == "random":
            sim.set_pressure_preconditioner(learned.LPCNet(seed=3), stall_window=20)
        sim.advance(1)
        if mode == "random":
            assert sim._learned.last_reason in (_lib.FCG_STALLED, _lib.FCG_MAXITER, _lib.FCG_CONVERGED)
            out["reason"] = sim._learned.last_reason
            sim.set_pressure_preconditioner(None)
        out[mode] = sim.u.copy()
    rel = np.abs(out["random"] - out["plain"]).max() / np.abs(out["plain"]).max()
    assert rel < 1e-6, (rel, out["reason"])


def test_bounded_grid_barrier_gives_up_and_the_context_stays_usable(cuda_lib):
    import torch

    from cfd2d_b200 import _lib, cases

    lib = _lib.lib()
    dev = _lib.device()
    # bar = [counter, CTAs taking part]: alone it passes at once; told that 8 CTAs take
    # part, it waits for 7 that never come, gives up and reports the timeout
    for ctas, passes in ((1, True), (8, False)):
        bar = torch.tensor([0, ctas], dtype=torch.int32, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        ok = torch.full((1,), -1, dtype=torch.int32, device=dev)
        rc = lib.cfd2d_barrier_selftest(_lib.ptr(bar), _lib.ptr(status), _lib.ptr(ok), _lib.stream_ptr())
        _lib.check(rc, "cfd2d_barrier_selftest")
        torch.cuda.synchronize()
        assert int(ok.item()) == (1 if passes else 0)
        assert bool(int(status.item()) & _lib.S_BARRIER_TIMEOUT) == (not passes)
    case = cases.lid_driven_cavity(re=100, n=16)
    case.sim.advance(5)
    assert case.sim.max_divergence() < 1e-10


def test_stage_times(cuda_lib):
    """Simulation.stage_times: event-timed parts of the step (the solve dominates)."""
    from cfd2d_b200 import cases

    case = cases.lid_driven_cavity(re=100, n=64, pressure_solver="cg")
    sim = case.sim
    sim.pressure.tol = 1e-8
    sim.advance(3)
    st = sim.stage_times(5)
    assert sim.n == 8 and len(sim.history.t) == 8
    assert st["solve_ms"] > 0 and st["pre_solve_ms"] > 0 and st["post_solve_ms"] > 0
    assert st["solve_ms"] > st["pre_solve_ms"] and st["kernels_per_step"] >= 8

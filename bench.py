"""Benchmark of the projection step on B200 (one JSON line on rank 0).

Workload (headline): the seeded obstacle flow -- 1024 x 512 MAC grid on a 2 x 1
channel, 2-12 circles, ellipses or rectangles from the obstacle-flow generator
(``cases.obstacle_flow(seed=13)``: 11 obstacles, Re 1465), block inflow U = 1,
outflow p = 0, slip walls, AB2 with automatic upwind fraction, tau 0.5; pressure
by Jacobi-PCG to a relative residual of 1e-8 in FP64. Synthetic: the flow starts
from rest, as the reference's cases do.

A step is one full projection step (all stages, one captured CUDA graph).
value     = cell-updates/s (nx*ny cells per step, summed over ranks) from CUDA
            events around every timed step on the solver's stream; L2 is flushed
            (256 MiB write) between timed steps.
poisson_ms = event time of the pressure solve inside the step graph.
e2e       = the same metric through the public API (``sim.step()``) with u, v copied
            in from pinned host memory and u, v, p copied back out every step.
roofline  = the pressure solver kernel: algorithmic bytes 88 B per cell per CG
            iteration (FP64 x, r, p, q, z traffic of a streaming implementation)
            over its event-timed duration.
learned   = the same workload with the pressure solved by flexible CG with the
            shipped learned preconditioner (to the same 1e-8): per-step time and
            cell-updates/s inside sim.step(), and Poisson ms and iterations of
            both solvers on the same system from the same warm start.
single_reduction = the headline workload with the slab solver's single-reduction
            form (one grid reduction per CG iteration instead of scipy's two).
batch_64_cavities = 64 seeded uneven cavities stepped together against the per-case loop.
sst_channel_mixed_precision = the k-omega SST channel 128 x 192 over 5000 steps with the FP64 and the
            mixed-precision solver: time and the mixed run's error in the u profile, nu_t, tau_w, c_f.
grid_2048x1024 = the same generator and seed at 2048 x 1024: plain steps and the
            Poisson comparison (the CG cap is raised so that both reach 1e-8).
cylinder_440x82 = the cylinder channel with a van Leer scalar (plain FP64 path), and the same run with the
            on-chip solver's single-reduction form.
stencils  = the kernel-level stencil drop-ins on a 4096 x 2048 grid against the
            measured HBM peak (compulsory bytes per cell over event time).
--impl reference times the CPU restatement of the reference (the oracle: NumPy
stencils, scipy's CG called as the reference calls it) on the same workload, a
bounded sample per step (see run_reference).
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
for p in (str(ROOT / "cfd-_b200"), str(ROOT)):
    if p not in sys.path:
        sys.path.insert(0, p)

METRIC = "cell-updates/s and Poisson ms at 1e-8 residual: learned-PC vs plain CG on B200"
NX, NY, SEED = 1024, 512, 13
CG_RTOL = 1e-8
BYTES_PER_CELL_ITER = 88.0
BYTES_PER_CELL_SOLVE = 32.0
WORKLOAD = (f"obstacle flow {NX}x{NY} (generator seed {SEED}: 2-12 circles/ellipses/rectangles, sizes "
            f"0.02-0.08 of the height, block inflow U=1, outflow p=0, slip walls, Re log-uniform 200-2000), "
            f"FP64 Jacobi-PCG rtol 1e-8")
CYL_NX, CYL_NY = 440, 82
CYL_SPEC = {"fall": "cylinder", "parameter": {"re": 100, "nx": CYL_NX, "ny": CYL_NY},
            "numerik": {"pressure_solver": "cg"},
            "skalar": {"name": "c", "diffusivity": 1e-3, "inflow_band": [0.15, 0.25], "limiter": "vanleer"}}
CYL_WORKLOAD = "cylinder 440x82 Re100 + van Leer scalar, FP64 Jacobi-PCG rtol 1e-8"
# the CPU arms time this many CG iterations per step and scale to the full solve
CPU_CG_SAMPLE = 150


def _peaks():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return None, 0, 1
    import torch
    import torch.distributed as dist

    backend = "nccl" if torch.cuda.is_available() else "gloo"
    from datetime import timedelta

    dist.init_process_group(backend=backend, timeout=timedelta(seconds=120))
    return dist, dist.get_rank(), dist.get_world_size()


def _max_over_ranks(dist, x: float) -> float:
    if dist is None:
        return x
    import torch

    dev = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(dist):
    if dist is not None:
        dist.barrier()


class _Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons during the timed region."""

    def __init__(self, path):
        self.path = path
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "50"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return self
        # nvidia-smi takes a moment to start: the timed region begins after its
        # first sample, and only later samples are summarised
        self.skip = 0
        t_end = time.time() + 5.0
        while time.time() < t_end and self.proc.poll() is None:
            self.f.flush()
            n = len(Path(self.path).read_text().splitlines())
            if n >= 1:
                self.skip = n
                break
            time.sleep(0.02)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.06)
            self.proc.terminate()
            self.proc.wait(timeout=5)
            self.f.close()

    def summary(self, dev_index: int):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in Path(self.path).read_text().splitlines()[self.skip:]:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9 or parts[0] != str(dev_index):
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": smax, "samples": len(sm),
                "reasons": sorted(reasons)}


def _clocks_path(name: str) -> str:
    """Where the nvidia-smi clock samples of the timed region go: CFD2D_CLOCKS_DIR if
    set (to keep them), else the temporary directory."""
    import tempfile

    return str(Path(os.environ.get("CFD2D_CLOCKS_DIR") or tempfile.gettempdir()) / name)


def _ncu_traffic(profile: str):
    """DRAM bytes per launch of a kernel from its committed ncu summary, if any."""
    f = ROOT / "profiles" / profile
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith("dram_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def _obstacle_spec(seed: int = SEED):
    from cfd2d_b200.cases import random_obstacle_spec
    import numpy as np

    return random_obstacle_spec(np.random.default_rng(seed))


# ------------------------------------------------------------------ CPU timings
def cpu_oracle_sample(full_steps: int, warm_steps: int, steps: int, threads: int | None,
                      iters_per_step: float | None = None) -> dict:
    """Bounded CPU sample of the headline workload, timed in a child process: the
    oracle's projection step (NumPy stencils; the pressure system solved by scipy's
    cg with the Jacobi preconditioner, the call cfd2d/pressure.py:171 makes).
    ``full_steps`` untimed steps from rest solve to 1e-8 (the last one's iteration
    count is the full solve's length unless ``iters_per_step`` is given); the
    ``warm_steps`` + ``steps`` steps after them run at most CPU_CG_SAMPLE CG
    iterations, and each timed step's time is scaled to the full solve: time
    outside the solve + solve time x (full iterations / sampled iterations). With
    ``iters_per_step`` given, the initial projection the case makes while it is
    built is capped as well (it only prepares a state to time)."""
    env = dict(os.environ)
    if threads is not None:
        for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
            env[k] = str(threads)
    obst, re = _obstacle_spec()
    code = f"""
import sys, time, json, warnings
sys.path.insert(0, {str(ROOT)!r})
warnings.simplefilter("ignore")
import oracle as O
O.OPressure.engine = "scipy"
if {iters_per_step!r}:
    O.OPressure.maxiter = {CPU_CG_SAMPLE}
sim = O.custom_obstacles({obst!r}, lx=2.0, ly=1.0, nx={NX}, ny={NY}, re={re!r}, tol={CG_RTOL})
O.OPressure.maxiter = 5000
ps = sim.pressure
spent = [0.0]
solve = ps.solve
def timed_solve(rhs):
    t0 = time.perf_counter()
    out = solve(rhs)
    spent[0] += time.perf_counter() - t0
    return out
ps.solve = timed_solve
n_full = None
for _ in range({full_steps}):
    sim.step()
    n_full = ps.last_iterations
n_target = {iters_per_step!r} or n_full
ps.maxiter = {CPU_CG_SAMPLE}
for _ in range({warm_steps}):
    sim.step()
est, raw, its = [], [], []
for _ in range({steps}):
    spent[0] = 0.0
    t0 = time.perf_counter()
    sim.step()
    el = time.perf_counter() - t0
    k = max(1, ps.last_iterations)
    its.append(k)
    raw.append(el)
    est.append(el - spent[0] + spent[0] * n_target / k)
print(json.dumps({{"est_s": est, "raw_s": raw, "sampled_iters": its, "full_iters": n_target}}))
"""
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, check=True)
    d = json.loads(out.stdout.strip().splitlines()[-1])
    d["seconds_per_step"] = sum(d["est_s"]) / len(d["est_s"])
    d["rate"] = NX * NY / d["seconds_per_step"]
    return d


def cpu_direct_lu_rate(steps: int = 3) -> dict:
    """The reference's other pressure solver on the same workload, timed in a child
    process on one host thread: the oracle's step with the pressure system factorised
    once by SuperLU (COLAMD ordering, as cfd2d/pressure.py:137) and solved by the
    factors every step."""
    env = dict(os.environ)
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        env[k] = "1"
    obst, re = _obstacle_spec()
    code = f"""
import sys, time, json, warnings
sys.path.insert(0, {str(ROOT)!r})
warnings.simplefilter("ignore")
import oracle as O
t0 = time.perf_counter()
sim = O.custom_obstacles({obst!r}, lx=2.0, ly=1.0, nx={NX}, ny={NY}, re={re!r}, tol={CG_RTOL},
                         pressure_solver="direct")
setup = time.perf_counter() - t0
sim.step()
t0 = time.perf_counter()
for _ in range({steps}):
    sim.step()
print(json.dumps({{"setup_s": setup, "seconds": time.perf_counter() - t0}}))
"""
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, check=True)
    d = json.loads(out.stdout.strip().splitlines()[-1])
    return {"value": NX * NY * steps / d["seconds"], "unit": "cell-updates/s", "ms_per_step": 1e3 * d["seconds"] / steps,
            "setup_s_incl_factorisation": d["setup_s"], "cores": 1, "steps": steps,
            "what": "oracle step with the pressure solved by SuperLU factors (the reference's 'direct' solver), "
                    "factorised once at set-up"}


def run_reference(args, dist, rank, world):
    """The CPU arm: the oracle (the reference's algorithm restated; its CG is scipy's
    cg as the reference calls it) on the headline workload with every host thread
    it can use. Each step is a bounded sample (cpu_oracle_sample): the first two
    warm-up steps solve in full (their iteration count sets the full-solve length),
    the other warm-up steps and the timed steps run CPU_CG_SAMPLE CG iterations and
    are scaled to the full solve. Rank 0 only; the other ranks exit without work."""
    if rank != 0:
        return
    full = min(2, args.warmup)
    d = cpu_oracle_sample(full, args.warmup - full, args.steps, None)
    value = d["rate"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "cell-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * d["seconds_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded obstacle flow from rest, as the reference's cases start)",
        "config": {"workload": WORKLOAD, "grid": [NX, NY], "cells": NX * NY, "parallelism": "replicas"},
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": f"oracle step (NumPy stencils, scipy cg + Jacobi as cfd2d/pressure.py:171); "
                                   f"{full} full warm-up steps from rest set the solve length "
                                   f"({d['full_iters']} CG iterations), then each step runs {CPU_CG_SAMPLE} CG "
                                   f"iterations and its solve time is scaled to the full length"},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "poisson_iters_per_step": float(d["full_iters"]),
        "raw_sample_ms_per_step": 1e3 * sum(d["raw_s"]) / len(d["raw_s"]),
        "direct_lu": cpu_direct_lu_rate(),
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ stencil roofline
STENCIL_NX, STENCIL_NY = 4096, 2048
# compulsory FP64 traffic per cell (each array read or written once; flags 1 B)
STENCIL_BYTES = {
    "momentum_tendencies": 8 + 8 + 1 + 8 + 8,          # R u, v, fluid; W hu, hv (constant nu)
    "scalar_transport": 8 + 8 + 8 + 8 + 1 + 8,         # R phi, u, v, D, fluid; W out
}


def stencil_roofline(peak: float, reps: int = 10) -> dict:
    """The kernel-level drop-ins (cfd2d/kernels.py entry points; van Leer for the
    scalar) on a 4096 x 2048 grid with random solid cells: event-timed per launch
    with L2 flushed before each launch, achieved GB/s from the compulsory bytes
    above."""
    import numpy as np
    import torch

    from cfd2d_b200 import _lib

    L = _lib.lib()
    nx, ny = STENCIL_NX, STENCIL_NY
    dev = _lib.device()
    g = torch.Generator(device=dev).manual_seed(0)
    u = torch.rand((nx + 1, ny + 2), dtype=torch.float64, device=dev, generator=g)
    v = torch.rand((nx + 2, ny + 1), dtype=torch.float64, device=dev, generator=g) - 0.5
    fluid = (torch.rand((nx + 2, ny + 2), device=dev, generator=g) > 0.05).to(torch.uint8)
    fluid[0, :] = 0
    fluid[-1, :] = 0
    fluid[:, 0] = 0
    fluid[:, -1] = 0
    phi = torch.rand((nx + 2, ny + 2), dtype=torch.float64, device=dev, generator=g)
    diff = torch.full((nx + 2, ny + 2), 1e-3, dtype=torch.float64, device=dev)
    out = torch.zeros_like(phi)
    hu, hv = torch.zeros_like(u), torch.zeros_like(v)
    # a cell field, as the reference's; the constant-viscosity form reads nu[1, 1]
    nu = torch.full((nx + 2, ny + 2), 1e-3, dtype=torch.float64, device=dev)
    bt = {k: torch.zeros(n, dtype=torch.int64, device=dev) for k, n in (("l", ny), ("r", ny), ("b", nx), ("t", nx))}
    bv = {k: torch.zeros(n, dtype=torch.float64, device=dev) for k, n in (("l", ny), ("r", ny), ("b", nx), ("t", nx))}
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    P = _lib.ptr
    sp = _lib.stream_ptr()
    dx, dy = 1.0 / nx, 0.5 / ny
    calls = {
        "momentum_tendencies": lambda: L.cfd2d_momentum_tendencies(
            P(u), P(v), P(fluid), nx, ny, dx, dy, P(nu), 0, 0.1, 0, P(hu), P(hv), None, 0, sp),
        "scalar_transport": lambda: L.cfd2d_scalar_transport(
            P(phi), P(u), P(v), P(fluid), nx, ny, dx, dy, P(diff), 1, 0, P(bt["l"]), P(bv["l"]), P(bt["r"]),
            P(bv["r"]), P(bt["b"]), P(bv["b"]), P(bt["t"]), P(bv["t"]), 0, 0.0, P(out), sp),
    }
    res = {}
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    for name, fn in calls.items():
        _lib.check(fn(), name)
        ms = []
        for _ in range(reps):
            flush.fill_(1.0)
            ev[0].record()
            _lib.check(fn(), name)
            ev[1].record()
            torch.cuda.synchronize()
            ms.append(ev[0].elapsed_time(ev[1]))
        med = float(np.median(ms))
        gbs = STENCIL_BYTES[name] * nx * ny / (med * 1e-3) / 1e9
        res[name] = {"ms": med, "bytes_per_cell": STENCIL_BYTES[name], "achieved_gbs": gbs, "frac": gbs / peak}
    # the tile autotuner on the momentum drop-in at this size (cfd2d_b200.autotune); the
    # shape changes no result, and the default shape is restored afterwards
    from cfd2d_b200 import autotune

    default = autotune.get_tile(autotune.MOMENTUM)
    try:
        best, timings = autotune.tune_momentum(nx, ny, reps=reps, store=False)
        ms_best = float(timings[best])
        gbs = STENCIL_BYTES["momentum_tendencies"] * nx * ny / (ms_best * 1e-3) / 1e9
        res["momentum_tendencies_tuned"] = {"tile": list(best), "ms": ms_best, "achieved_gbs": gbs,
                                            "frac": gbs / peak,
                                            "ms_by_tile": {f"{a}x{b}": t for (a, b), t in timings.items()}}
    finally:
        autotune.set_tile(autotune.MOMENTUM, *default)
    del u, v, fluid, phi, diff, out, hu, hv, flush
    torch.cuda.empty_cache()
    return {"grid": [nx, ny], "l2": "flushed before each launch", **res}


# ------------------------------------------------------------------ learned preconditioner
def _rhs_of(sim):
    """The pressure right-hand side div(F, G) / dt of the simulation's last predictor."""
    import torch

    g = sim.grid
    F, G = sim.F, sim.G
    return torch.from_numpy(((F[1:, 1:-1] - F[:-1, 1:-1]) / g.dx + (G[1:-1, 1:] - G[1:-1, :-1]) / g.dy)
                            / sim.dt).cuda()


def poisson_compare(sim, net, maxiter: int) -> dict:
    """One pressure system of ``sim`` (its last predictor) solved to 1e-8 by the plain
    Jacobi-PCG and by flexible CG with the learned preconditioner, each from the same
    warm start (the step's previous pressure), event-timed on the device after one
    untimed solve of the same system."""
    import torch

    from cfd2d_b200 import learned

    ps = sim.pressure
    xprev = ps._d_x0.clone()
    sim.advance(1)
    rhs = _rhs_of(sim)
    fcg = learned.LearnedPCG(ps, net, maxiter=maxiter)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    out = {}
    for name, solve in (("plain", lambda: ps.solve(rhs)), ("learned", lambda: fcg.solve(rhs))):
        for _timed in (False, True):
            ps._d_x0.copy_(xprev)
            torch.cuda.synchronize()
            ev[0].record()
            solve()
            ev[1].record()
            torch.cuda.synchronize()
        its = ps.last_iterations if name == "plain" else fcg.last_total_iterations
        out[name] = {"poisson_ms": ev[0].elapsed_time(ev[1]), "iterations": int(its)}
        if name == "learned":
            out[name]["fcg_iterations"] = int(fcg.last_iterations)
            out[name]["fell_back"] = bool(fcg.last_reason != 1)
    out["speedup_learned_vs_plain"] = out["plain"]["poisson_ms"] / out["learned"]["poisson_ms"]
    # one application of the network alone, launched directly (outside the solve's
    # graph, whose conditional node keeps profilers from seeing its kernels)
    fcg.precondition()
    torch.cuda.synchronize()
    reps = 5
    ev[0].record()
    for _ in range(reps):
        fcg.precondition()
    ev[1].record()
    torch.cuda.synchronize()
    out["network_ms_per_application"] = ev[0].elapsed_time(ev[1]) / reps
    fcg.close()
    ps._d_x0.copy_(xprev)
    return out


def learned_steps(nx: int, ny: int, steps: int, warmup: int, flush, maxiter: int = 5000) -> dict:
    """The obstacle flow with every step's pressure solved by flexible CG with the
    learned preconditioner (Simulation.set_pressure_preconditioner): device time of
    each sim.step() from events on the simulation's stream (L2 flushed before each),
    end-to-end wall time of the same calls, FCG iterations and fallbacks per step."""
    import numpy as np
    import torch

    from cfd2d_b200 import cases, learned

    case = cases.obstacle_flow(SEED, nx, ny, pressure_solver="cg")
    sim = case.sim
    sim.pressure.tol = CG_RTOL
    sim.pressure.maxiter = maxiter
    sim.set_pressure_preconditioner(learned.pretrained(), maxiter=maxiter)
    sim.advance(warmup)
    stream = sim.stream
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ms, fallbacks = [], 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    wall = 0.0
    for _ in range(steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        ev[0].record(stream)
        sim.step()
        ev[1].record(stream)
        ev[1].synchronize()
        wall += time.perf_counter() - t1
        ms.append(ev[0].elapsed_time(ev[1]))
        fallbacks += int(sim._learned.last_reason != 1)
    del t0
    its = np.array(sim.history.extra["cg_iterationen"][-steps:], dtype=float)
    dev_s = sum(ms) / 1e3
    out = {"steps": steps, "warmup": warmup, "ms_per_step": 1e3 * dev_s / steps,
           "cell_updates_per_s": nx * ny * steps / dev_s, "wall_cell_updates_per_s": nx * ny * steps / wall,
           "fcg_iters_per_step": float(its.mean()), "fallback_steps": fallbacks}
    sim.set_pressure_preconditioner(None)
    return out


def grid2048_section(steps: int, flush) -> dict:
    """The obstacle-flow generator's seed at 2048 x 1024: plain FP64 steps (event-timed
    over ``steps`` steps after 2, CG cap raised to 20000 so every solve reaches 1e-8)
    and the Poisson comparison with the learned preconditioner."""
    import numpy as np
    import torch

    from cfd2d_b200 import cases, learned

    nx, ny = 2 * NX, 2 * NY
    case = cases.obstacle_flow(SEED, nx, ny, pressure_solver="cg")
    sim = case.sim
    sim.pressure.tol = CG_RTOL
    sim.pressure.maxiter = 20000
    sim.advance(2)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    flush.fill_(1.0)
    torch.cuda.synchronize()
    with torch.cuda.stream(sim.stream):
        ev[0].record()
        sim.launch_steps(steps)
        ev[1].record()
    sim.finish_steps()
    torch.cuda.synchronize()
    ms = ev[0].elapsed_time(ev[1]) / steps
    its = np.array(sim.history.extra["cg_iterationen"][-steps:], dtype=float)
    out = {"workload": f"obstacle flow {nx}x{ny} (generator seed {SEED}), FP64 Jacobi-PCG rtol 1e-8",
           "plain": {"steps": steps, "ms_per_step": ms, "cell_updates_per_s": nx * ny / (ms / 1e3),
                     "poisson_iters_per_step": float(its.mean())}}
    out["poisson"] = poisson_compare(sim, learned.pretrained(), maxiter=20000)
    del sim, case
    torch.cuda.empty_cache()
    return out


def _graph_steps(sim, steps: int, warmup: int, flush, clock_name: str | None = None):
    """Replay a one-step graph with events at its start, around its pressure solve and
    at its end: ``warmup`` untimed steps, then ``steps`` timed ones with L2 flushed
    before each. Returns (step ms list, solve ms list, kernels per step, clocks)."""
    import torch

    from cfd2d_b200 import _lib

    L = _lib.lib()
    stream = sim._stream
    sptr = _lib.stream_ptr(stream)
    ev = (C.c_void_p * 4)()
    _lib.check(L.cfd2d_events_create(4, ev), "events")
    graph = C.c_void_p(0)
    knodes = C.c_int(0)
    clk = None
    try:
        with torch.cuda.stream(stream):
            sim._flush_mirrors()
            sim._set_run_limits()
            _lib.check(L.cfd2d_graph_capture_steps_ex(C.byref(sim._S), 1, sptr, ev, C.byref(graph),
                                                      C.byref(knodes)), "capture")

            def one_step():
                flush.fill_(1.0)  # L2 flush (256 MiB write) outside the timed events
                _lib.check(L.cfd2d_graph_launch(graph, sptr), "launch")
                ms_step, ms_solve = C.c_float(), C.c_float()
                _lib.check(L.cfd2d_event_elapsed_ms(ev[0], ev[3], C.byref(ms_step)), "elapsed")
                _lib.check(L.cfd2d_event_elapsed_ms(ev[1], ev[2], C.byref(ms_solve)), "elapsed")
                return ms_step.value, ms_solve.value

            for _ in range(warmup):
                one_step()
            torch.cuda.synchronize()
            step_ms, solve_ms = [], []
            if clock_name:
                clk = _Clocks(_clocks_path(clock_name)).__enter__()
            try:
                for _ in range(steps):
                    a, b = one_step()
                    step_ms.append(a)
                    solve_ms.append(b)
                torch.cuda.synchronize()
            finally:
                if clk is not None:
                    clk.__exit__(None, None, None)
            sim._st_fresh = False
            sim._after_steps()
    finally:
        if graph.value:
            L.cfd2d_graph_destroy(graph)
        L.cfd2d_events_destroy(4, ev)
    return step_ms, solve_ms, int(knodes.value), clk


def single_reduction_section(steps: int, warmup: int, flush) -> dict:
    """The headline workload with the slab solver's single-reduction form
    (PressureSolver.grid_ctas = -2: Chronopoulos-Gear recurrence, one grid reduction
    per CG iteration instead of scipy's two), graph-timed like the headline."""
    import numpy as np

    from cfd2d_b200 import cases

    case = cases.obstacle_flow(SEED, NX, NY, pressure_solver="cg")
    sim = case.sim
    sim.pressure.tol = CG_RTOL
    sim.pressure.grid_ctas = -2
    step_ms, solve_ms, knodes, _ = _graph_steps(sim, steps, warmup, flush)
    its = np.array(sim.history.extra["cg_iterationen"][-steps:], dtype=float)
    dev_s = sum(step_ms) / 1e3
    solve_s = sum(solve_ms) / 1e3
    cells = NX * NY
    return {"workload": WORKLOAD + "; single-reduction CG recurrence", "steps": steps,
            "ms_per_step": 1e3 * dev_s / steps, "cell_updates_per_s": cells * steps / dev_s,
            "poisson_ms": 1e3 * solve_s / steps, "poisson_iters_per_step": float(its.mean()),
            "us_per_iteration": 1e6 * solve_s / its.sum()}


def cylinder_section(steps: int, warmup: int, flush) -> dict:
    """The cylinder channel with a passive scalar (plain FP64 path), graph-timed."""
    import numpy as np

    from cfd2d_b200 import cases

    case = cases.build_case(CYL_SPEC)
    sim = case.sim
    sim.pressure.tol = CG_RTOL
    step_ms, solve_ms, knodes, _ = _graph_steps(sim, steps, warmup, flush)
    its = np.array(sim.history.extra["cg_iterationen"][-steps:], dtype=float)
    dev_s = sum(step_ms) / 1e3
    solve_s = sum(solve_ms) / 1e3
    cells = CYL_NX * CYL_NY
    achieved = (BYTES_PER_CELL_ITER * cells * its.sum() + BYTES_PER_CELL_SOLVE * cells * len(its)) / solve_s / 1e9
    peak, _ = _peaks()
    out = {"workload": CYL_WORKLOAD, "steps": steps, "ms_per_step": 1e3 * dev_s / steps,
           "cell_updates_per_s": cells * steps / dev_s, "poisson_ms": 1e3 * solve_s / steps,
           "poisson_iters_per_step": float(its.mean()), "kernels_per_step": knodes,
           "solver": "k_pcg_cluster (on-chip)", "solver_equiv_gbs": achieved, "solver_equiv_frac": achieved / peak,
           "us_per_iteration": 1e6 * solve_s / its.sum()}
    # the same run with the on-chip solver's single-reduction form (grid_ctas = -2)
    case = cases.build_case(CYL_SPEC)
    sim = case.sim
    sim.pressure.tol = CG_RTOL
    sim.pressure.grid_ctas = -2
    step_ms, solve_ms, _, _ = _graph_steps(sim, steps, warmup, flush)
    its1 = np.array(sim.history.extra["cg_iterationen"][-steps:], dtype=float)
    solve1 = sum(solve_ms) / 1e3
    out["single_reduction"] = {"solver": "k_pcg_cluster1 (on-chip, one cluster reduction per iteration)",
                               "ms_per_step": sum(step_ms) / steps, "poisson_ms": 1e3 * solve1 / steps,
                               "poisson_iters_per_step": float(its1.mean()),
                               "us_per_iteration": 1e6 * solve1 / its1.sum()}
    return out


# ------------------------------------------------------------------ mixed precision
def mixed_section(steps: int = 300) -> dict:
    """The bench workload from rest, `steps` steps with the FP64 solver and with the
    mixed one (FP32 iterations, FP64 refinement and reductions): ms per step from
    events around the run, and the end state of the mixed run against the FP64 one
    (max-norm of the difference over the max-norm of the FP64 field; the drag and
    lift series over the last 100 steps)."""
    import numpy as np
    import torch

    from cfd2d_b200 import cases

    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    res = {}
    for prec in ("fp64", "mixed"):
        case = cases.build_case(CYL_SPEC)
        sim = case.sim
        sim.pressure.tol = CG_RTOL
        sim.pressure.precision = prec
        sim.advance(5)
        torch.cuda.synchronize()
        ev[0].record(torch.cuda.current_stream())
        sim.advance(steps)
        ev[1].record(torch.cuda.current_stream())
        torch.cuda.synchronize()
        its = sim.history.extra["cg_iterationen"][-steps:]
        res[prec] = dict(ms_per_step=ev[0].elapsed_time(ev[1]) / steps, iters=float(np.mean(its)),
                         fields=(sim.u.copy(), sim.v.copy(), sim.p.copy(), sim.scalars["c"].phi.copy()),
                         fx=np.array(sim.history.fx[-100:]), fy=np.array(sim.history.fy[-100:]))
    e = lambda a, b: float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))  # noqa: E731
    f64, mx = res["fp64"], res["mixed"]
    return {
        "workload": f"{CYL_WORKLOAD}, {steps} steps after 5 from rest",
        "fp64": {"ms_per_step": f64["ms_per_step"], "poisson_iters_per_step": f64["iters"]},
        "mixed": {"ms_per_step": mx["ms_per_step"], "poisson_iters_per_step": mx["iters"]},
        "rel_err_vs_fp64": {"u": e(mx["fields"][0], f64["fields"][0]), "v": e(mx["fields"][1], f64["fields"][1]),
                            "p": e(mx["fields"][2], f64["fields"][2]), "c": e(mx["fields"][3], f64["fields"][3]),
                            "drag_force": e(mx["fx"], f64["fx"]), "lift_force": e(mx["fy"], f64["fy"])},
    }


def vof_section(steps: int = 50, n: int = 96) -> dict:
    """The reference's dam break (two-phase VOF, variable-density projection) at its
    default 96 x 96 from rest: ms per step from events over `steps` steps after 5,
    iterations of the variable-coefficient solve, and the reference's own direct
    solve of the same system (scipy spsolve, as cfd2d/pressure.py:236) timed on the
    host on the final state for comparison with the device solve."""
    import numpy as np
    import torch

    import oracle as O
    from cfd2d_b200 import cases

    case = cases.dam_break(n=n)
    sim = case.sim
    sim.advance(5)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    torch.cuda.synchronize()
    with torch.cuda.stream(sim.stream):
        ev[0].record()
        sim.advance(steps)
        ev[1].record()
    torch.cuda.synchronize()
    ms = ev[0].elapsed_time(ev[1]) / steps
    its = np.array(sim.history.extra["cg_iterationen"][-steps:], dtype=float)
    # the same variable-coefficient system on the host: rhs = div(F, G) / dt, b = 1/rho
    osim = O.dam_break(n=n)
    g = sim.grid
    F, G, rho, dt = sim.F, sim.G, sim.rho, sim.dt
    div = (F[1:, 1:-1] - F[:-1, 1:-1]) / g.dx + (G[1:-1, 1:] - G[1:-1, :-1]) / g.dy
    bx = 2.0 / (rho[:-1, :] + rho[1:, :])
    by = 2.0 / (rho[:, :-1] + rho[:, 1:])
    osim.pressure.solve_variable(div / dt, bx[:, 1:-1], by[1:-1, :])
    t0 = time.perf_counter()
    reps = 3
    for _ in range(reps):
        osim.pressure.solve_variable(div / dt, bx[:, 1:-1], by[1:-1, :])
    cpu_ms = 1e3 * (time.perf_counter() - t0) / reps
    # the variable-coefficient PCG moves the constant-coefficient 88 B/cell/iteration plus
    # the two face coefficients (16 B); charging the whole step to it gives a lower bound
    iters = float(its.mean())
    equiv = (88 + 16) * n * n * iters / (ms / 1e3) / 1e9
    peak, _ = _peaks()
    return {"workload": f"dam break {n}x{n} (two-phase VOF, CSF, variable density), {steps} steps after 5",
            "ms_per_step": ms, "cell_updates_per_s": n * n / (ms / 1e3),
            "poisson_iters_per_step": iters,
            "solver_equiv_gbs_lower_bound": equiv, "solver_equiv_frac_lower_bound": equiv / peak,
            "volume_error_rel": sim.model("multiphase").monitors(sim)["volumenfehler_rel"],
            "cpu_direct_solve_ms": cpu_ms,
            "cpu_direct_solve": "scipy spsolve of the same system on the host (the reference's solver, 1 thread "
                                "per call as scipy runs it), mean of 3 calls"}


def configs_section(cavity_steps: int = 2000, sst_steps: int = 500) -> dict:
    """The other two single-case workloads of the reference's benchmark list, timed by
    events around advance(): the lid-driven cavity 64 x 64 (AB2, gamma 0.1, tau 0.5,
    CG rtol 1e-8, 2000 steps from rest) and the periodic k-omega SST channel 128 x 192
    (bulk velocity 1, Re_b 1e4, laminar profile with 5 % seeded noise, CG rtol 1e-8)."""
    import numpy as np
    import torch

    from cfd2d_b200 import cases

    def timed(sim, n):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        sim.advance(3)
        torch.cuda.synchronize()
        with torch.cuda.stream(sim.stream):
            ev[0].record()
            sim.launch_steps(n)
            ev[1].record()
        sim.finish_steps()
        torch.cuda.synchronize()
        ms = ev[0].elapsed_time(ev[1])
        its = np.array(sim.history.extra["cg_iterationen"][-n:], dtype=float)
        g = sim.grid
        return {"ms_per_step": ms / n, "cell_updates_per_s": g.nx * g.ny * n / (ms / 1e3),
                "poisson_iters_per_step": float(its.mean())}

    case = cases.lid_driven_cavity(re=100, n=64, scheme="ab2", gamma=0.1, tau=0.5, pressure_solver="cg")
    case.sim.pressure.tol = CG_RTOL
    cav = timed(case.sim, cavity_steps)
    sim = sst_channel_sim()
    return {"cavity_64x64": {"steps": cavity_steps, **cav},
            "sst_channel_128x192": {"steps": sst_steps, **timed(sim, sst_steps)}}


def sst_channel_sim(precision: str = "fp64"):
    """The periodic k-omega SST channel 128 x 192 (domain 2 pi x 2, bulk velocity 1,
    Re_b 1e4 held by volume-flow forcing, laminar profile with 5 % seeded noise,
    k = 1e-3 and omega = 10, CG rtol 1e-8), re-projected, ready to step."""
    import numpy as np

    from cfd2d_b200.boundary import BoundaryCondition as BC
    from cfd2d_b200.grid import Grid
    from cfd2d_b200.solver import Simulation
    from cfd2d_b200.turbulence import KOmegaSST

    nx, ny = 128, 192
    grid = Grid(nx, ny, 2 * np.pi, 2.0)
    bcs = dict(left=BC("periodic"), right=BC("periodic"), bottom=BC("noslip"), top=BC("noslip"))
    nu = 2.0 / 1e4
    sst = KOmegaSST(intensity=np.sqrt(1e-3 / 1.5), viscosity_ratio=1e-3 / (nu * 10.0), U_ref=1.0)
    sim = Simulation(grid, bcs, nu=nu, flow_rate=1.0, models=[sst], pressure_solver="cg")
    sim.pressure.tol = CG_RTOL
    sim.pressure.precision = precision
    rng = np.random.default_rng(0)
    y = (np.arange(ny) + 0.5) * grid.dy
    u = sim.u
    u[1:nx + 1, 1:ny + 1] = (1.5 * y * (2.0 - y))[None, :] * (1.0 + 0.05 * rng.uniform(-1.0, 1.0, (nx, ny)))
    v = sim.v
    v[1:nx + 1, 1:ny] = 0.05 * rng.uniform(-1.0, 1.0, (nx, ny - 1))
    u[~sim.u_fluid] = 0.0
    v[~sim.v_fluid] = 0.0
    sim._apply_bc()
    sim._project_initial()
    return sim


def sst_mixed_section(steps: int = 5000) -> dict:
    """The SST channel over ``steps`` steps with the FP64 pressure solver and with the
    mixed one (FP32 CG iterations, FP64 refinement and reductions): ms per step, and
    the mixed run's error against the FP64 run (which follows the reference's CPU run
    to 6e-13 over 500 steps, tests/test_gpu_parity.py) in the x-mean u profile, nu_t and
    the wall shear stress and skin friction of cfd2d/report.py:455-462
    (tau_w = nu (u_1 + u_ny) / 2 / (dy / 2) on column i = 2, c_f = 2 tau_w / U^2)."""
    import numpy as np
    import torch

    out, res = {}, {}
    for prec in ("fp64", "mixed"):
        sim = sst_channel_sim(prec)
        sim.advance(2)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        torch.cuda.synchronize()
        with torch.cuda.stream(sim.stream):
            ev[0].record()
            sim.launch_steps(steps - 2)
            ev[1].record()
        sim.finish_steps()
        torch.cuda.synchronize()
        g = sim.grid
        u = sim.u
        ucol = u[2, 1:-1]
        tau_w = sim.nu * 0.5 * (ucol[0] + ucol[-1]) / (0.5 * g.dy)
        res[prec] = {"profile": u[1:g.nx + 1, 1:-1].mean(axis=0), "nut": sim.nu_t.copy(), "tau_w": float(tau_w),
                     "cf": float(2.0 * tau_w / 1.0 ** 2)}
        its = np.array(sim.history.extra["cg_iterationen"][-(steps - 2):], dtype=float)
        out[prec] = {"ms_per_step": ev[0].elapsed_time(ev[1]) / (steps - 2), "poisson_iters_per_step": float(its.mean())}
    a, b = res["mixed"], res["fp64"]
    out["mixed_vs_fp64"] = {
        "u_profile_rel": float(np.abs(a["profile"] - b["profile"]).max() / np.abs(b["profile"]).max()),
        "nu_t_rel": float(np.abs(a["nut"] - b["nut"]).max() / np.abs(b["nut"]).max()),
        "tau_w_rel": abs(a["tau_w"] / b["tau_w"] - 1.0), "c_f_rel": abs(a["cf"] / b["cf"] - 1.0)}
    out["fp64"]["c_f"] = b["cf"]
    out["workload"] = f"k-omega SST channel 128x192, {steps} steps from the perturbed laminar profile"
    return out


# ------------------------------------------------------------------ GPU arm
def _optional(flag: bool, fn):
    """An optional section: None when skipped, an error record if it fails (an
    optional section never costs the bench line)."""
    if flag:
        return None
    try:
        return fn()
    except Exception as exc:
        return {"error": f"{type(exc).__name__}: {exc}"}


def run_b200(args, dist, rank, world):
    import numpy as np
    import torch

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    from cfd2d_b200 import _lib, cases

    # the headline workload: the obstacle flow (default) or, with --workload cylinder,
    # the cylinder channel with a scalar (the form its committed profiles capture)
    cyl_head = args.workload == "cylinder"
    nxh, nyh = (CYL_NX, CYL_NY) if cyl_head else (NX, NY)
    workload = CYL_WORKLOAD if cyl_head else WORKLOAD
    case = cases.build_case(CYL_SPEC) if cyl_head else cases.obstacle_flow(SEED, NX, NY, pressure_solver="cg")
    sim = case.sim
    sim.pressure.tol = CG_RTOL
    stream = sim._stream
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    n0 = sim._pull().n
    _barrier(dist)
    step_ms, solve_ms, knodes, clk = _graph_steps(sim, args.steps, args.warmup, flush,
                                                  f"clocks_rank{rank}.csv")
    _barrier(dist)
    st = sim._pull()
    assert st.n - n0 == args.steps + args.warmup
    its = np.array(sim.history.extra["cg_iterationen"][-args.steps:], dtype=float)
    dev_s = sum(step_ms) / 1e3
    dev_s_max = _max_over_ranks(dist, dev_s)
    cells = nxh * nyh
    value = world * cells * args.steps / dev_s_max
    solve_s = sum(solve_ms) / 1e3
    iters = float(its.mean())
    achieved = (BYTES_PER_CELL_ITER * cells * its.sum() + BYTES_PER_CELL_SOLVE * cells * len(its)) / solve_s / 1e9
    peak, peak_kind = _peaks()

    # ---- end to end through the public API with host buffers
    e2e_steps = args.steps
    with torch.cuda.stream(stream):
        host = {nm: torch.empty(getattr(sim, "_" + nm).shape, dtype=torch.float64).pin_memory()
                for nm in ("u", "v")}
        for nm in host:
            host[nm].copy_(getattr(sim, "_" + nm))
        out = {nm: torch.empty(getattr(sim, "_" + nm).shape, dtype=torch.float64).pin_memory()
               for nm in ("u", "v", "p")}
        h2d = sum(t.numel() * 8 for t in host.values())
        d2h = sum(t.numel() * 8 for t in out.values())
        _barrier(dist)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            sim._u.copy_(host["u"], non_blocking=True)
            sim._v.copy_(host["v"], non_blocking=True)
            sim.step()
            for nm in out:
                out[nm].copy_(getattr(sim, "_" + nm), non_blocking=True)
            stream.synchronize()
            # this step's results are the next step's inputs: swap the pinned buffers
            for nm in ("u", "v"):
                host[nm], out[nm] = out[nm], host[nm]
        e2e_s = time.perf_counter() - t0
    e2e_s = _max_over_ranks(dist, e2e_s)
    e2e = world * cells * e2e_steps / e2e_s
    clocks = clk.summary(local) if clk is not None else None

    if rank != 0:
        return
    fluid_cells = int(sim.pressure.n)
    del sim, case
    torch.cuda.empty_cache()

    def learned_all():
        from cfd2d_b200 import learned

        steps_rec = learned_steps(NX, NY, args.steps, args.warmup, flush)
        c2 = cases.obstacle_flow(SEED, NX, NY, pressure_solver="cg")
        c2.sim.pressure.tol = CG_RTOL
        c2.sim.advance(args.warmup)
        cmp = poisson_compare(c2.sim, learned.pretrained(), maxiter=5000)
        return {"workload": f"{WORKLOAD}; pressure by flexible CG with the learned preconditioner to the same "
                            f"rtol (plain Jacobi-PCG continues if it stalls)",
                "value": steps_rec["cell_updates_per_s"], "unit": "cell-updates/s", "step": steps_rec,
                "poisson": cmp}

    learned_rec = _optional(args.no_learned, learned_all)
    big = _optional(args.no_large, lambda: grid2048_section(3, flush))
    single = _optional(args.no_single, lambda: single_reduction_section(args.steps, args.warmup, flush))
    cyl = _optional(args.no_cylinder, lambda: cylinder_section(100, 10, flush))
    stencils = _optional(args.no_stencils, lambda: stencil_roofline(peak))
    mixed = _optional(args.no_mixed, mixed_section)
    other = _optional(args.no_configs, configs_section)
    vof = _optional(args.no_vof, vof_section)
    bat = _optional(args.no_batch, lambda: batch_section(64, 3, 2))
    sstm = _optional(args.no_mixed, sst_mixed_section)
    cpu = None
    if world == 1 and not args.no_cpu_baseline and not cyl_head:
        d = cpu_oracle_sample(0, 1, 2, 1, iters_per_step=iters)
        cpu = {"value": d["rate"], "unit": "cell-updates/s", "cores": 1, "kind": "port",
               "sample": f"oracle step on 1 thread (NumPy stencils, scipy cg + Jacobi as cfd2d/pressure.py:171): "
                         f"1 warm-up and 2 timed steps from rest, each running {CPU_CG_SAMPLE} CG iterations, "
                         f"its solve time scaled to the {iters:.0f} iterations per step of this run"}
    line = {
        "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dev_s_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded obstacle flow from rest, as the reference's cases start)",
        "config": {"workload": workload, "grid": [nxh, nyh], "cells": cells, "fluid_cells": fluid_cells,
                   "l2": "flushed between timed steps (256 MiB write)", "parallelism": f"replicas x{world}",
                   "solver": "plain FP64 Jacobi-PCG (%s)" % ("k_pcg_cluster" if cyl_head else "k_pcg_slab")},
        "poisson_ms": 1e3 * solve_s / args.steps,
        "poisson_iters_per_step": iters,
        "e2e": {"value": e2e, "unit": "cell-updates/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": e2e_steps},
        "gpu_launches": knodes * args.steps,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "traffic": _ncu_traffic("pcg_cluster_cylinder440x82.txt" if cyl_head
                                             else "pcg_slab_obstacles1024x512.txt"),
                     "kernel": ("k_pcg_cluster (FP64 Jacobi-PCG on one thread-block cluster)" if cyl_head else
                                "k_pcg_slab (FP64 Jacobi-PCG, one persistent launch per solve, vectors in "
                                "shared memory)"),
                     "peak_kind": peak_kind},
        "cpu_baseline": cpu,
        "clocks": clocks,
        "learned": learned_rec,
        "single_reduction": single,
        "grid_2048x1024": big,
        "cylinder_440x82": cyl,
        "stencils": stencils,
        "mixed_precision": mixed,
        "vof_dam_break": vof,
        "batch_64_cavities": bat,
        "sst_channel_mixed_precision": sstm,
        "other_workloads": other,
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ batched uneven cases
def batch_section(n_cases: int, steps: int, warmup: int, dist=None, clk_name: str | None = None) -> dict:
    """Seeded uneven cavities (half lid-driven, half heated; side uniform in 32..512),
    every step of all of them queued on their own streams before any is waited for
    (grids beyond one on-chip cluster solve on one 16-CTA cluster each, so their solves
    overlap), against the per-case loop (the same cases one after another, each with
    the solver it would use alone), both timed on the device."""
    import numpy as np
    import torch

    from cfd2d_b200 import batch

    t0 = time.perf_counter()
    cs = batch.uneven_cavities(n_cases=n_cases, seed=0)
    for c in cs:
        c.sim.pressure.tol = CG_RTOL
    b = batch.Batch([c.sim for c in cs])
    setup_s = time.perf_counter() - t0
    b.advance(warmup)
    _barrier(dist)
    torch.cuda.synchronize()
    clk = _Clocks(_clocks_path(clk_name)).__enter__() if clk_name else None
    try:
        ms = b.timed_advance(steps, concurrent=True)
    finally:
        if clk is not None:
            clk.__exit__(None, None, None)
    ms_max = _max_over_ranks(dist, ms)
    # per-case loop: each case alone, one after another, timed per case on the device,
    # with the solver each case would use alone (the large grids over every SM)
    for sim in b.sims:
        sim.pressure.grid_ctas = 0
        sim.advance(1)  # captures the step graph again outside the timed region
    per_case = []
    main = torch.cuda.current_stream()
    for sim in b.sims:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(main)
        sim.stream.wait_event(e0)
        sim.launch_steps(steps)
        e1.record(sim.stream)
        sim.finish_steps()
        e1.synchronize()
        per_case.append(e0.elapsed_time(e1) / steps)
    loop_ms = sum(per_case) * steps
    cells = b.cells
    sizes = [sm.grid.nx for sm in b.sims]
    return {"workload": f"{len(b.sims)} cavities, side uniform in 32..512 step 32, half lid-driven "
                        f"(Re log-uniform 100-5000), half heated (Ra log-uniform 1e3-1e6, Pr 0.71), "
                        f"FP64 Jacobi-PCG rtol 1e-8",
            "steps": steps, "cells_per_step": cells, "ms_per_step": ms_max / steps,
            "cell_updates_per_s": cells * steps / (ms_max / 1e3),
            "cluster_solver_cases": sum(1 for sm in b.sims if sm.pressure.cluster > 0),
            "side_min_max": [min(sizes), max(sizes)], "setup_s": setup_s,
            "per_case_loop": {"cell_updates_per_s": cells * steps / (loop_ms / 1e3), "ms_per_step": loop_ms / steps,
                              "case_step_ms_p50": float(np.percentile(per_case, 50)),
                              "case_step_ms_p99": float(np.percentile(per_case, 99))},
            "speedup_vs_per_case_loop": loop_ms / ms_max,
            "clocks": clk.summary(int(os.environ.get("LOCAL_RANK", "0"))) if clk is not None else None}


def run_batch(args, dist, rank, world):
    """The batch as the headline workload (--workload batch): replicas over ranks as the
    main arm."""
    import torch

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    rec = batch_section(args.batch_cases, args.steps, args.warmup, dist, f"clocks_batch_rank{rank}.csv")
    if rank != 0:
        return
    line = {
        "metric": f"aggregate cell-updates/s, {args.batch_cases} uneven cavities stepped together",
        "value": world * rec["cell_updates_per_s"], "unit": "cell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": rec["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded cases from rest)",
        "config": {k: rec[k] for k in ("workload", "cells_per_step", "cluster_solver_cases", "side_min_max",
                                         "setup_s")},
        "per_case_loop": rec["per_case_loop"], "clocks": rec["clocks"],
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-stencils", action="store_true", help="skip the stencil-kernel roofline section")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-preconditioner section")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision section")
    ap.add_argument("--no-vof", action="store_true", help="skip the two-phase dam-break section")
    ap.add_argument("--no-configs", action="store_true", help="skip the cavity and SST channel section")
    ap.add_argument("--no-large", action="store_true", help="skip the 2048 x 1024 section")
    ap.add_argument("--no-cylinder", action="store_true", help="skip the cylinder 440 x 82 section")
    ap.add_argument("--no-single", action="store_true", help="skip the single-reduction solver section")
    ap.add_argument("--no-batch", action="store_true", help="skip the 64-cavity batch section")
    ap.add_argument("--workload", choices=["obstacles", "cylinder", "batch"], default="obstacles",
                    help="obstacles: the headline; cylinder: the cylinder channel as the headline workload "
                         "(the form the cylinder profiles capture); batch: 256 uneven cavities stepped together")
    ap.add_argument("--batch-cases", type=int, default=256)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference" and int(os.environ.get("RANK", "0")) != 0:
        return  # the CPU reference arm runs on rank 0 alone; other ranks exit without work
    if args.impl == "reference":
        run_reference(args, None, 0, int(os.environ.get("WORLD_SIZE", "1")))
        return
    dist, rank, world = _dist()
    try:
        if args.workload == "batch":
            run_batch(args, dist, rank, world)
        else:
            run_b200(args, dist, rank, world)
    finally:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""Many independent cases advanced side by side on one GPU (no counterpart in the reference).

Every Simulation owns a CUDA stream and replays its captured step graph there. A
Batch queues the steps of all its members before it waits for any, so the GPU runs
the latency-bound pressure solves of different cases at the same time, each on its
own cluster of SMs (or, for the grids too large for one cluster, on the grid-wide
solver), instead of one case after another.
"""

from __future__ import annotations

import numpy as np

from . import _lib


class Batch:
    """A set of independent simulations stepped together. Members whose pressure
    grid is too large for one on-chip cluster solve on one 16-CTA cluster with the
    vectors in global memory (``PressureSolver.grid_ctas = 16``) instead of on every
    SM, so that their solves can overlap too (set ``spread=False`` to keep them on
    the whole GPU)."""

    def __init__(self, sims, spread: bool = True):
        self.sims = list(sims)
        if spread:
            for s in self.sims:
                s.pressure.grid_ctas = 16

    @property
    def cells(self) -> int:
        """Cells updated by one step of every member (nx*ny summed)."""
        return sum(s.grid.nx * s.grid.ny for s in self.sims)

    def advance(self, nsteps: int) -> None:
        """nsteps steps of every member: all queued first, then all waited for."""
        for s in self.sims:
            s.launch_steps(nsteps)
        for s in self.sims:
            s.finish_steps()

    def timed_advance(self, nsteps: int, concurrent: bool = True) -> float:
        """advance(nsteps) timed on the device (ms): an event on the current stream
        before, every member's stream waiting on it, and an event after all of them.
        With concurrent=False the members run one after another (each waits for the
        previous one's last step): the per-case loop the batch is compared with."""
        t = _lib.torch()
        main = t.cuda.current_stream()
        start, end = t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)
        start.record(main)
        prev = start
        marks = []
        for s in self.sims:
            s.stream.wait_event(prev)
            s.launch_steps(nsteps)
            ev = t.cuda.Event()
            ev.record(s.stream)
            marks.append(ev)
            if not concurrent:
                prev = ev
        for ev in marks:
            main.wait_event(ev)
        end.record(main)
        for s in self.sims:
            s.finish_steps()
        end.synchronize()
        return start.elapsed_time(end)


def uneven_cavities(n_cases: int = 256, seed: int = 0, sizes=tuple(range(32, 513, 32))):
    """Seeded mix of uneven square cavities: half lid-driven with Re log-uniform in
    100-5000, half differentially heated (Boussinesq) with Ra log-uniform in 1e3-1e6
    and Pr = 0.71; the side of each drawn uniformly from ``sizes``."""
    from . import cases

    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_cases):
        n = int(rng.choice(sizes))
        if k % 2 == 0:
            re = float(np.exp(rng.uniform(np.log(100.0), np.log(5000.0))))
            out.append(cases.lid_driven_cavity(re=re, n=n, pressure_solver="cg"))
        else:
            ra = float(np.exp(rng.uniform(np.log(1e3), np.log(1e6))))
            out.append(cases.heated_cavity(ra=ra, pr=0.71, n=n, pressure_solver="cg"))
    return out

"""Tile-shape autotuner of the row kernels (no reference counterpart).

Sweeps the thread-block shapes of the momentum_tendencies drop-in and of the step's
row kernels (predictor, correction, turbulence, scalar update and ghosts) on the
device, keeps the fastest shape per (GPU, grid-size bucket) in a JSON cache
(``$CFD2D_TUNE_CACHE``, else ``~/.cache/cfd2d_b200/tiles.json``) and applies it. The
shape changes no result: every thread of these kernels computes its own cells.
"""

from __future__ import annotations

import ctypes as C
import json
import os
import tempfile
from pathlib import Path

import numpy as np

from . import _lib

MOMENTUM, STEP = 0, 1
CANDIDATES = ((32, 8), (32, 4), (64, 4), (128, 2), (16, 16), (32, 2), (64, 2), (256, 1), (32, 6))


def get_tile(which: int) -> tuple[int, int]:
    tx, ty = C.c_int(0), C.c_int(0)
    _lib.check(_lib.lib().cfd2d_get_tile(int(which), C.byref(tx), C.byref(ty)), "cfd2d_get_tile")
    return tx.value, ty.value


def set_tile(which: int, tx: int, ty: int) -> None:
    _lib.check(_lib.lib().cfd2d_set_tile(int(which), int(tx), int(ty)), "cfd2d_set_tile")


def bucket(nx: int, ny: int) -> int:
    """Grid-size bucket: ceil(log2) of the padded cell count."""
    return int(np.ceil(np.log2(max((nx + 2) * (ny + 2), 2))))


def cache_path() -> Path:
    env = os.environ.get("CFD2D_TUNE_CACHE")
    return Path(env) if env else Path.home() / ".cache" / "cfd2d_b200" / "tiles.json"


def _key(which: int, nx: int, ny: int) -> str:
    t = _lib.torch()
    return f"{t.cuda.get_device_name()}|{'momentum' if which == MOMENTUM else 'step'}|{bucket(nx, ny)}"


def load_cache() -> dict:
    p = cache_path()
    if not p.exists():
        return {}
    try:
        return json.loads(p.read_text())
    except (OSError, ValueError):
        return {}


def _store(key: str, tile, timings) -> None:
    p = cache_path()
    data = load_cache()
    data[key] = {"tile": list(tile), "ms": {f"{a}x{b}": ms for (a, b), ms in timings.items()}}
    p.parent.mkdir(parents=True, exist_ok=True)
    tmp = p.with_suffix(".tmp")
    tmp.write_text(json.dumps(data, indent=1))
    tmp.replace(p)


def apply_cached(nx: int, ny: int) -> dict:
    """Set the cached shapes for an nx x ny grid on this GPU; returns what was set."""
    data, done = load_cache(), {}
    for which in (MOMENTUM, STEP):
        entry = data.get(_key(which, nx, ny))
        if entry:
            set_tile(which, *entry["tile"])
            done[which] = tuple(entry["tile"])
    return done


def _events():
    t = _lib.torch()
    return t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)


def tune_momentum(nx: int, ny: int, reps: int = 20, candidates=CANDIDATES, store: bool = True):
    """Time cfd2d_momentum_tendencies (variable viscosity off) on seeded fields of an
    nx x ny grid for every candidate shape; keep and return the fastest."""
    t = _lib.torch()
    dev = _lib.device()
    rng = np.random.default_rng(0)
    u = _lib.to_dev(rng.uniform(-1, 1, (nx + 1, ny + 2)), t.float64)
    v = _lib.to_dev(rng.uniform(-1, 1, (nx + 2, ny + 1)), t.float64)
    fl = np.zeros((nx + 2, ny + 2), dtype=np.uint8)
    fl[1:-1, 1:-1] = 1
    fl = _lib.to_dev(fl)
    nu = t.full((nx + 2, ny + 2), 0.01, dtype=t.float64, device=dev)
    hu, hv = t.empty_like(u), t.empty_like(v)
    flush = t.empty(256 * 1024 * 1024 // 4, dtype=t.float32, device=dev) if (nx + 2) * (ny + 2) * 40 > 64e6 else None
    lib = _lib.lib()
    prev = get_tile(MOMENTUM)
    timings = {}
    stream = t.cuda.current_stream()

    def launch():
        rc = lib.cfd2d_momentum_tendencies(_lib.ptr(u), _lib.ptr(v), _lib.ptr(fl), nx, ny, 1.0 / nx, 1.0 / ny,
                                           _lib.ptr(nu), 0, 0.5, 0, _lib.ptr(hu), _lib.ptr(hv), None, 0,
                                           _lib.stream_ptr(stream))
        _lib.check(rc, "cfd2d_momentum_tendencies")

    try:
        for tile in candidates:
            set_tile(MOMENTUM, *tile)
            launch()
            total = 0.0
            for _ in range(reps):
                if flush is not None:
                    flush.fill_(1.0)
                e0, e1 = _events()
                e0.record(stream)
                launch()
                e1.record(stream)
                e1.synchronize()
                total += e0.elapsed_time(e1)
            timings[tuple(tile)] = total / reps
    finally:
        set_tile(MOMENTUM, *prev)
    best = min(timings, key=timings.get)
    set_tile(MOMENTUM, *best)
    if store:
        _store(_key(MOMENTUM, nx, ny), best, timings)
    return best, timings


def tune_step(sim, steps: int = 20, warmup: int = 3, candidates=CANDIDATES, store: bool = True):
    """Time `steps` steps of ``sim`` for every candidate shape of the step's row
    kernels (graphs recaptured per shape), keep and return the fastest. The
    simulation is put back to its state before tuning (checkpoint and restart)."""
    from . import functions

    t = _lib.torch()
    g = sim.grid
    prev = get_tile(STEP)
    timings = {}
    fos, sim.function_objects = sim.function_objects, []  # the tuning steps are not recorded
    with tempfile.TemporaryDirectory() as td:
        cp = Path(td) / "before_tuning.npz"
        functions.save_checkpoint(sim, cp)
        try:
            for tile in candidates:
                set_tile(STEP, *tile)
                sim._invalidate()
                sim.advance(warmup)
                e0, e1 = _events()
                with t.cuda.stream(sim.stream):
                    e0.record()
                    sim.launch_steps(steps)
                    e1.record()
                sim.finish_steps()
                e1.synchronize()
                timings[tuple(tile)] = e0.elapsed_time(e1) / steps
        finally:
            set_tile(STEP, *prev)
            functions.load_checkpoint(sim, cp)
            sim._invalidate()
            sim.function_objects = fos
    best = min(timings, key=timings.get)
    set_tile(STEP, *best)
    sim._invalidate()
    if store:
        _store(_key(STEP, g.nx, g.ny), best, timings)
    return best, timings

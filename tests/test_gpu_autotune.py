"""Tile-shape autotuner of the row kernels (cfd2d_b200.autotune) (GPU).

The shape changes only the speed: results under every tuned shape are bit-identical
to those of the default 32 x 8 tiles, tuning a simulation leaves its state where it
was, and the choice is cached per GPU and grid-size bucket.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu]


@pytest.fixture
def tiles(cuda_lib, tmp_path, monkeypatch):
    from cfd2d_b200 import autotune

    monkeypatch.setenv("CFD2D_TUNE_CACHE", str(tmp_path / "tiles.json"))
    yield autotune
    autotune.set_tile(autotune.MOMENTUM, 32, 8)
    autotune.set_tile(autotune.STEP, 32, 8)


def test_invalid_shapes_rejected(tiles):
    for bad in ((8, 8), (32, 16), (40, 1), (0, 4), (32, 0)):
        with pytest.raises(RuntimeError):
            tiles.set_tile(tiles.STEP, *bad)
    assert tiles.get_tile(tiles.STEP) == (32, 8)


def test_momentum_tuning_keeps_results(tiles):
    from inputs import momentum_cases

    from cfd2d_b200 import kernels

    def run_all():
        out = []
        for c in momentum_cases():
            hu, hv = np.full_like(c["u"], 7.0), np.full_like(c["v"], 7.0)
            kernels.momentum_tendencies(c["u"], c["v"], c["fluid"], c["nx"], c["ny"], c["dx"], c["dy"], c["nu"],
                                        c["variable"], c["gamma"], c["periodic"], hu, hv, c["rho"], c["var_density"])
            out += [hu, hv]
        return out

    ref = run_all()
    best, timings = tiles.tune_momentum(512, 256, reps=3)
    assert len(timings) == len(tiles.CANDIDATES) and best in timings
    assert tiles.get_tile(tiles.MOMENTUM) == best
    for tile in ((64, 4), (16, 16), (256, 1)):
        tiles.set_tile(tiles.MOMENTUM, *tile)
        assert all(np.array_equal(a, b) for a, b in zip(run_all(), ref)), tile
    assert tiles.apply_cached(512, 256)[tiles.MOMENTUM] == best


def test_step_tuning_restores_state_and_keeps_results(tiles):
    from cfd2d_b200 import cases

    spec = {"fall": "cylinder", "parameter": {"re": 100, "nx": 88, "ny": 17},
            "numerik": {"pressure_solver": "cg"},
            "skalar": {"name": "c", "diffusivity": 1e-3, "inflow_band": [0.15, 0.25]}}
    a = cases.build_case(spec).sim
    b = cases.build_case(spec).sim
    a.advance(5)
    b.advance(5)
    best, timings = tiles.tune_step(a, steps=5, warmup=1)
    assert best in timings and tiles.get_tile(tiles.STEP) == best
    assert a.n == 5 and len(a.history.t) == 5
    a.advance(10)  # tuned shape
    tiles.set_tile(tiles.STEP, 32, 8)
    b._invalidate()
    b.advance(10)  # default shape
    for name in ("u", "v", "p"):
        assert np.array_equal(getattr(a, name), getattr(b, name)), name
    assert np.array_equal(a.scalars["c"].phi, b.scalars["c"].phi)
    assert tiles.apply_cached(88, 17)[tiles.STEP] == best

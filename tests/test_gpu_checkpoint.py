"""Checkpoint and restart from the device state in the reference's file format (GPU).

Mirrors the reference's own tests (tests/test_functions.py:48-97) and adds the
cross-format check: a checkpoint written by the reference itself (golden fixture,
tests/golden/make_golden.py gen_checkpoint) loads here and the continued run matches
the reference's uninterrupted run.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden

pytestmark = [pytest.mark.gpu]

TOL = 1e-10


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _cyl_spec(**extra):
    spec = {"fall": "cylinder", "parameter": {"re": 100, "nx": 88, "ny": 17, "t_end": 0.2}}
    spec.update(extra)
    return spec


@pytest.mark.parametrize("extra", [
    {},
    {"turbulenz": {"modell": "kOmegaSST"}},
    {"skalar": {"name": "c", "diffusivity": 1e-3, "inflow_band": [0.15, 0.25]}},
])
def test_checkpoint_restart_is_exact(cuda_lib, tmp_path, extra):
    from cfd2d_b200 import cases, functions

    spec = _cyl_spec(**extra)
    ref = cases.build_case(spec)
    for _ in range(80):
        ref.sim.step()
    a = cases.build_case(spec)
    for _ in range(40):
        a.sim.step()
    functions.save_checkpoint(a.sim, tmp_path / "cp.npz")
    b = cases.build_case(spec)
    functions.load_checkpoint(b.sim, tmp_path / "cp.npz")
    for _ in range(40):
        b.sim.step()
    assert b.sim.n == ref.sim.n
    assert np.allclose(b.sim.u, ref.sim.u, atol=1e-12, rtol=0)
    for name in ref.sim.scalars:
        assert np.allclose(b.sim.scalars[name].phi, ref.sim.scalars[name].phi, atol=1e-12)
    assert len(b.sim.history.t) == 80


def test_checkpoint_wrong_geometry_rejected(cuda_lib, tmp_path):
    from cfd2d_b200 import cases, functions

    a = cases.lid_driven_cavity(re=100, n=16)
    functions.save_checkpoint(a.sim, tmp_path / "cp.npz")
    b = cases.lid_driven_cavity(re=100, n=20)
    with pytest.raises(ValueError):
        functions.load_checkpoint(b.sim, tmp_path / "cp.npz")


def test_reference_checkpoint_loads_and_continues(cuda_lib, tmp_path):
    from cfd2d_b200 import cases, functions

    g = golden("golden_checkpoint")
    np.savez_compressed(tmp_path / "ref_cp.npz", **{k[3:]: g[k] for k in g if k.startswith("cp_")})
    spec = {"fall": "cylinder", "parameter": {"re": 100, "nx": 88, "ny": 17, "t_end": 0.2},
            "numerik": {"pressure_solver": "cg"},
            "skalar": {"name": "c", "diffusivity": 1e-3, "inflow_band": [0.15, 0.25]}}
    case = cases.build_case(spec)
    sim = case.sim
    sim.pressure.tol = 1e-12
    functions.load_checkpoint(sim, tmp_path / "ref_cp.npz")
    assert sim.n == 40
    for _ in range(40):
        sim.step()
    assert sim.t == pytest.approx(float(g["ref80_t"]), rel=1e-13)
    assert _rel(sim.u, g["ref80_u"]) < TOL
    assert _rel(sim.v, g["ref80_v"]) < TOL
    assert _rel(sim.p, g["ref80_p"]) < 1e-8
    assert _rel(sim.scalars["c"].phi, g["ref80_c"]) < TOL

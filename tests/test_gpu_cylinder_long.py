"""Long-horizon parity on the cylinder channel with a passive scalar (GPU).

The fixture (tests/golden/golden_cylinder2000.npz, make_golden.py's
``cylinder_long`` group) is the reference's own run of the case over 2000 steps
from rest with its direct (SuperLU) pressure solver: digests of u, v, p and the
scalar at steps 1000 and 2000 (every 2nd value in both directions, all row and
column sums, the max-norm), the force history and the drag and lift coefficients
from the reference's validation.force_coefficients.

* FP64 path with pressure_solver="direct" (CG to 1e-13 on the device): fields
  within 1e-10 relative, c_D and c_L series within 1e-9 of the reference's scale.
* Mixed precision (FP32 CG iterations, FP64 refinement and reductions, rtol 1e-8,
  the upgrade beside the plain path): the error per field and of c_D and c_L
  against the same FP64 reference, asserted below 1e-6 and printed.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden

pytestmark = [pytest.mark.gpu]

SPEC = {"fall": "cylinder", "parameter": {"re": 100, "nx": 440, "ny": 82},
        "skalar": {"name": "c", "diffusivity": 1e-3, "inflow_band": [0.15, 0.25], "limiter": "vanleer"}}


def _fields(sim):
    return {"u": sim.u, "v": sim.v, "p": sim.p, "c": sim.scalars["c"].phi}


def _errors(sim, g, n):
    out = {}
    for name, a in _fields(sim).items():
        m = float(g[f"cyl2k_{n}_{name}_max"])
        out[name] = float(np.abs(a[::2, ::2] - g[f"cyl2k_{n}_{name}_sub"]).max() / m)
        for ax, key in ((1, "rows"), (0, "cols")):
            d = np.abs(a.sum(axis=ax) - g[f"cyl2k_{n}_{name}_{key}"]).max() / (m * a.shape[ax])
            out[name] = max(out[name], float(d))
    return out


def _coefficients(sim):
    from cfd2d_b200 import validation

    return validation.force_coefficients(sim.history.fx, sim.history.fy, U=1.0, L=0.1)


def _run(precision, solver):
    from cfd2d_b200 import cases

    spec = dict(SPEC, numerik={"pressure_solver": solver})
    case = cases.build_case(spec)
    sim = case.sim
    if solver == "cg":
        sim.pressure.tol = 1e-8
    sim.pressure.precision = precision
    g = golden("golden_cylinder2000")
    errs = {}
    for n in (1000, 2000):
        sim.advance(n - sim.n)
        errs[n] = _errors(sim, g, n)
    cd, cl = _coefficients(sim)
    scale = max(np.abs(g["cyl2k_cd"]).max(), np.abs(g["cyl2k_cl"]).max())
    errs["cd"] = float(np.abs(np.asarray(cd) - g["cyl2k_cd"]).max() / scale)
    errs["cl"] = float(np.abs(np.asarray(cl) - g["cyl2k_cl"]).max() / scale)
    return sim, errs


def test_cylinder_2000_steps_direct_fp64(cuda_lib):
    sim, errs = _run("fp64", "direct")
    print("fp64 direct vs reference:", errs)
    for n in (1000, 2000):
        for name, e in errs[n].items():
            assert e < 1e-10, (n, name, e)
    assert errs["cd"] < 1e-9 and errs["cl"] < 1e-9, errs
    assert sim.n == 2000


def test_cylinder_2000_steps_mixed_precision_error(cuda_lib):
    sim, errs = _run("mixed", "cg")
    print("mixed precision (rtol 1e-8) vs FP64 reference:", errs)
    for n in (1000, 2000):
        for name, e in errs[n].items():
            assert e < 1e-6, (n, name, e)
    assert errs["cd"] < 1e-6 and errs["cl"] < 1e-6, errs

"""Function objects fed from the device fields (cfd2d_b200.functions) (GPU).

Bit-for-bit against the oracle's restatement of cfd2d/functions.py applied to the
same GPU state (a twin simulation stepped one step at a time, its fields read back
after every step): probe series of every field kind (face u and v extrapolated,
cell fields clipped, NaN in the obstacle), the time average, the line sample, the
field catalogue and the VTK bytes. Against the reference's own run (golden fixture)
to trajectory accuracy. The reference's tests (tests/test_functions.py:19-47,
98-117) are mirrored.
"""

from __future__ import annotations

import json

import numpy as np
import pytest

from conftest import golden

pytestmark = [pytest.mark.gpu, pytest.mark.filterwarnings("ignore::RuntimeWarning")]

FO_POINTS = [(0.5, 0.2), (0.2, 0.2), (0.0, 0.0), (2.2, 0.41), (1.0, 0.05), (-0.1, 0.5), (0.31, 0.1337),
             (0.15, 0.2), (2.5, -0.2)]
FO_FIELDS = ("u", "v", "pressure", "vorticity", "speed", "streamfunction", "c")


def _case():
    from cfd2d_b200 import cases

    case = cases.cylinder_flow(re=100, nx=88, ny=17, pressure_solver="cg")
    cases.add_scalar(case, "c", 1e-3, inflow_band=(0.15, 0.25))
    case.sim.pressure.tol = 1e-8
    return case.sim


def _eq(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(a, b, equal_nan=True)


def _rel(a, b):
    a, b = np.nan_to_num(np.asarray(a, dtype=float)), np.nan_to_num(np.asarray(b, dtype=float))
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def runs(cuda_lib):
    """sim A with device function objects over 30 steps in one advance(); twin B
    stepped one step at a time with the oracle's function objects on its host state."""
    import oracle as O
    from cfd2d_b200 import functions

    a = _case()
    pr = functions.Probes(FO_POINTS, fields=FO_FIELDS)
    fa = functions.FieldAverage(t_start=0.01)
    ls = functions.LineSample((0.0, 0.1), (2.2, 0.3), n=37, fields=["u", "v", "pressure", "c"], label="schraeg")
    a.function_objects += [pr, fa, ls]
    a.advance(30)
    b = _case()
    ofa = O.OFieldAverage(t_start=0.01)
    xs, ys = [p[0] for p in FO_POINTS], [p[1] for p in FO_POINTS]
    rows = {f: [] for f in FO_FIELDS}
    ts = []
    for _ in range(30):
        b.step()
        ts.append(b.t)
        for f in FO_FIELDS:
            rows[f].append(O.sample_field(b, f, xs, ys))
        ofa.execute(b)
    return a, b, pr, fa, ls, ofa, rows, ts


def test_twin_is_bit_identical(runs):
    a, b = runs[0], runs[1]
    for name in ("u", "v", "p"):
        assert np.array_equal(getattr(a, name), getattr(b, name)), name
    assert a.n == b.n == 30


def test_probe_series_bitwise(runs):
    a, _, pr, _, _, _, rows, ts = runs
    assert pr.t == ts
    for f in FO_FIELDS:
        assert _eq(np.array(pr.data[f]), np.array(rows[f])), f


def test_field_average_bitwise(runs):
    _, _, _, fa, _, ofa, _, _ = runs
    assert fa.T == ofa.T
    for k in ("u", "v", "p"):
        assert _eq(fa.sum[k], ofa.sum[k]) and _eq(fa.sum2[k], ofa.sum2[k]), k
        assert _eq(fa.mean(k), ofa.mean(k)) and _eq(fa.rms(k), ofa.rms(k)), k


def test_line_sample_field_data_and_vtk_bitwise(runs, tmp_path):
    import oracle as O
    from cfd2d_b200 import functions, visualization

    a, b, _, _, ls, _, _, _ = runs
    d = ls.sample(a)
    s, x, y = O.line_points((0.0, 0.1), (2.2, 0.3), 37)
    assert _eq(d["s"], s) and _eq(d["x"], x) and _eq(d["y"], y)
    for f in ("u", "v", "pressure", "c"):
        assert _eq(d[f], O.sample_field(b, f, x, y)), f
    assert list(visualization.available_fields(a)) == list(O.available_fields(b))
    for f in visualization.available_fields(a):
        assert _eq(visualization.field_data(a, f), O.field_data(b, f)), f
    raw = functions.write_vtk(a, tmp_path / "f.vtk").read_bytes()
    assert raw == O.write_vtk_bytes(b)
    files = ls.write(tmp_path)
    assert files and files[0].read_text().splitlines()[0] == "s;x;y;u;v;pressure;c"


def test_against_the_reference_run(runs):
    """The same function objects in the reference (tests/golden/make_golden.py
    gen_functions): equal up to the trajectory difference of the iterative solve."""
    _, _, pr, fa, _, _, _, _ = runs
    g = golden("golden_functions")
    assert np.allclose(pr.t, g["fo_probe_t"], rtol=1e-13, atol=0)
    for f in FO_FIELDS:
        mine, ref = np.array(pr.data[f]), g[f"fo_probe_{f}"]
        assert np.array_equal(np.isnan(mine), np.isnan(ref)), f
        assert _rel(mine, ref) < 1e-8, f
    assert fa.T == pytest.approx(float(g["fo_avg_T"]), rel=1e-13)
    for k in ("u", "v", "p"):
        assert _rel(fa.sum[k], g[f"fo_avg_sum_{k}"]) < 1e-8, k
        assert _rel(fa.sum2[k], g[f"fo_avg_sum2_{k}"]) < 1e-8, k


def test_sst_fields_in_probes_and_vtk(cuda_lib, tmp_path):
    """k, log10 omega and nu_t of the SST model through the device paths."""
    import oracle as O
    from cfd2d_b200 import cases, functions

    spec = {"fall": "cylinder", "parameter": {"re": 1000, "nx": 88, "ny": 17},
            "numerik": {"pressure_solver": "cg"}, "turbulenz": {"modell": "kOmegaSST"}}
    a = cases.build_case(spec).sim
    pts = [(0.5, 0.2), (1.5, 0.05), (0.21, 0.2)]
    pr = functions.Probes(pts, fields=("k", "omega", "nu_t"))
    a.function_objects.append(pr)
    a.advance(5)
    xs, ys = [p[0] for p in pts], [p[1] for p in pts]
    for f in ("k", "nu_t"):
        assert _eq(pr.data[f][-1], O.sample_field(a, f, xs, ys)), f
    om = pr.data["omega"][-1]
    ref = O.sample_field(a, "omega", xs, ys)
    assert np.array_equal(np.isnan(om), np.isnan(ref))
    assert _rel(om, ref) < 1e-14  # CUDA log10 against numpy's
    raw = functions.write_vtk(a, tmp_path / "sst.vtk").read_bytes()
    assert b"SCALARS omega float 1" in raw and b"SCALARS nu_t float 1" in raw
    # every block but omega's is bit-identical; omega's float32 values agree to rounding
    ref = O.write_vtk_bytes(a)
    assert len(raw) == len(ref)
    i = raw.index(b"SCALARS omega float 1\nLOOKUP_TABLE default\n") + len(b"SCALARS omega float 1\nLOOKUP_TABLE default\n")
    n = 88 * 17 * 4
    assert raw[:i] == ref[:i] and raw[i + n:] == ref[i + n:]
    a32 = np.frombuffer(raw[i:i + n], dtype=">f4")
    b32 = np.frombuffer(ref[i:i + n], dtype=">f4")
    assert np.abs(a32.astype(float) - b32.astype(float)).max() <= 2 * np.abs(b32).max() * 2.0 ** -23


def test_probe_buffer_grows_and_every(cuda_lib):
    from cfd2d_b200 import cases, functions

    case = cases.lid_driven_cavity(re=100, n=16, pressure_solver="cg")
    p1 = functions.Probes([(0.5, 0.5)], fields=("u",))
    p3 = functions.Probes([(0.5, 0.5)], fields=("u",), every=3)
    case.sim.function_objects += [p1, p3]
    case.sim.advance(300)
    assert len(p1.t) == 300 and len(p3.t) == 100
    assert p3.t == p1.t[2::3]
    assert [v[0] for v in p3.data["u"]] == [v[0] for v in p1.data["u"]][2::3]


# ---------------------------------------------------------------- reference tests
def test_probes_and_line_sample(cuda_lib, tmp_path):
    # tests/test_functions.py:19-30
    from cfd2d_b200 import cases, functions

    case = cases.lid_driven_cavity(re=100, n=16)
    pr = functions.Probes([(0.5, 0.5), (0.5, 0.9)], fields=("u", "pressure", "vorticity"))
    ls = functions.LineSample((0.5, 0.0), (0.5, 1.0), n=21, fields=("u", "v"), label="mitte")
    case.sim.function_objects += [pr, ls]
    case.sim.run(0.5, verbose=False)
    files = pr.write(tmp_path) + ls.write(tmp_path)
    assert all(f.exists() for f in files)
    assert len(pr.t) == case.sim.n
    assert ls.result["u"][0] == pytest.approx(0.0, abs=1e-12)
    assert ls.result["u"][-1] == pytest.approx(1.0, abs=1e-12)


def test_vtk_file_structure(cuda_lib, tmp_path):
    # tests/test_functions.py:33-47
    from cfd2d_b200 import cases, functions

    spec = {"fall": "cylinder", "parameter": {"re": 100, "nx": 88, "ny": 17, "t_end": 0.2},
            "temperatur": {"alpha": 1e-3, "T_obstacle": 1.0}}
    case = cases.build_case(spec)
    case.sim.run(0.05, verbose=False)
    path = functions.write_vtk(case.sim, tmp_path / "f.vtk")
    raw = path.read_bytes()
    assert raw.startswith(b"# vtk DataFile Version 3.0")
    assert b"DIMENSIONS 89 18 1" in raw
    assert b"VECTORS U float" in raw and b"SCALARS T float 1" in raw
    i = raw.index(b"VECTORS U float\n") + len(b"VECTORS U float\n")
    vec = np.frombuffer(raw[i:i + 88 * 17 * 12], dtype=">f4").reshape(-1, 3)
    uc, _ = case.sim.cell_velocity()
    assert np.allclose(vec[:, 0], np.nan_to_num(uc).T.ravel(), atol=1e-5)


def test_case_json_roundtrip_with_function_objects(cuda_lib, tmp_path):
    # tests/test_functions.py:98-117 (without the matplotlib report)
    from cfd2d_b200 import cases, functions

    spec = {"fall": "cylinder", "parameter": {"re": 100, "nx": 88, "ny": 17, "t_end": 0.2},
            "function_objects": [{"typ": "sonden", "punkte": [[0.5, 0.2]]},
                                 {"typ": "mittelwerte", "t_start": 0.0},
                                 {"typ": "vtk", "intervall": 0.1},
                                 {"typ": "checkpoint", "intervall": 0.1}]}
    cases.save_case(spec, tmp_path / "case.json")
    loaded = cases.load_case(tmp_path / "case.json")
    assert loaded == spec
    case = cases.build_case(loaded)
    out = tmp_path / "out"
    out.mkdir()
    case.sim.function_objects = functions.build_function_objects(loaded["function_objects"], out)
    reason = case.sim.run(case.t_end, verbose=False)
    assert reason == "t_end"
    for fo in case.sim.function_objects:
        fo.write(out)
    for f in ("sonden.csv", "mittelwerte.npz", "checkpoint.npz", "vtk/feld.vtk.series", "vtk/feld_00000.vtk"):
        assert (out / f).exists(), f
    series = json.loads((out / "vtk/feld.vtk.series").read_text())
    assert len(series["files"]) >= 2
    assert len(case.sim.function_objects[0].t) == case.sim.n


def test_vof_fields_in_probes_and_vtk(cuda_lib, tmp_path):
    """alpha and rho of the VOF model through the device function objects."""
    import oracle as O
    from cfd2d_b200 import cases, functions

    sim = cases.dam_break(n=32).sim
    pts = [(0.1, 0.1), (0.3, 0.05), (0.2, 0.29), (0.29, 0.03)]
    pr = functions.Probes(pts, fields=("alpha", "rho", "pressure"))
    sim.function_objects.append(pr)
    sim.advance(10)
    xs, ys = [p[0] for p in pts], [p[1] for p in pts]
    for f in ("alpha", "rho", "pressure"):
        assert _eq(pr.data[f][-1], O.sample_field(sim, f, xs, ys)), f
    raw = functions.write_vtk(sim, tmp_path / "dam.vtk").read_bytes()
    assert raw == O.write_vtk_bytes(sim)
    assert b"SCALARS alpha float 1" in raw and b"SCALARS rho float 1" in raw

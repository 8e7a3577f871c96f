"""Pin the CPU oracle against outputs of the reference itself (CPU only).

The fixtures were produced by ``tests/golden/make_golden.py`` running the reference
(Numba kernels, scipy CG / SuperLU). Stencils and masks must agree bit for bit;
the time-stepping runs must agree to 1e-12 relative (bitwise on the machine that
made the fixtures, where the oracle calls the same BLAS dot as scipy's CG).
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from conftest import golden
from inputs import momentum_cases, scalar_cases

pytestmark = pytest.mark.filterwarnings("ignore::RuntimeWarning")


def rel(a, b):
    d = np.abs(np.asarray(a) - np.asarray(b)).max()
    s = np.abs(np.asarray(b)).max()
    return d / s if s > 0 else d


# ---------------------------------------------------------------- stencils
def test_momentum_and_obstacle_bc_bitwise():
    g = golden("golden_kernels")
    n = 0
    for k, c in enumerate(momentum_cases()):
        u, v = c["u"], c["v"]
        hu = np.full_like(u, 7.0)
        hv = np.full_like(v, 7.0)
        O.momentum_tendencies(u, v, c["fluid"], c["nx"], c["ny"], c["dx"], c["dy"], c["nu"],
                              c["variable"], c["gamma"], c["periodic"], hu, hv, c["rho"],
                              c["var_density"])
        assert np.array_equal(hu, g[f"m{k}_hu"]), k
        assert np.array_equal(hv, g[f"m{k}_hv"]), k
        uo, vo = u.copy(), v.copy()
        O.obstacle_bc(uo, vo, c["fluid"], c["nx"], c["ny"], c["periodic"])
        assert np.array_equal(uo, g[f"m{k}_u_obc"]), k
        assert np.array_equal(vo, g[f"m{k}_v_obc"]), k
        n += 1
    assert n == int(g["n_momentum"])


def test_scalar_transport_bitwise_all_limiters():
    g = golden("golden_kernels")
    n = 0
    for k, c in enumerate(scalar_cases()):
        o = np.full_like(c["phi"], 3.0)
        bt, bv = c["bt"], c["bv"]
        O.scalar_transport(c["phi"], c["u"], c["v"], c["fluid"], c["nx"], c["ny"], c["dx"], c["dy"],
                           c["diff"], c["limiter"], c["periodic"], bt["l"], bv["l"], bt["r"],
                           bv["r"], bt["b"], bv["b"], bt["t"], bv["t"], c["obs_t"], c["obs_v"], o)
        assert np.array_equal(o, g[f"s{k}_out"]), (k, c["limiter"], c["periodic"], c["obs_t"])
        n += 1
    assert n == int(g["n_scalar"])


# ---------------------------------------------------------------- geometry
def test_masks_and_finalize_bitwise():
    g = golden("golden_geometry")
    for k in range(int(g["n_shapes"])):
        nx, ny, lx, ly = g[f"g{k}_grid"]
        grid = O.OGrid(int(nx), int(ny), lx, ly)
        assert np.array_equal(O.circle_mask(grid, *g[f"g{k}_circle"]), g[f"g{k}_circle_mask"])
        assert np.array_equal(O.ellipse_mask(grid, *g[f"g{k}_ellipse"]), g[f"g{k}_ellipse_mask"])
        assert np.array_equal(O.rectangle_mask(grid, *g[f"g{k}_rect"]), g[f"g{k}_rect_mask"])
    grid = O.OGrid(440, 82, 2.2, 0.41)
    assert np.array_equal(O.circle_mask(grid, 0.2, 0.2, 0.1 / 2), g["cyl_mask"])
    grid = O.OGrid(60, 40, 1.5, 1.0)
    grid.fluid[:] = g["fin_before"]
    assert grid.finalize() == int(g["fin_removed"])
    assert np.array_equal(grid.fluid, g["fin_after"])


# ---------------------------------------------------------------- pressure
def _pressure_oracle(name, g):
    """Build the same simulation as the fixture generator and return its solver.

    Constructing the simulation matters: its initial projection (cfd2d/solver.py:195-204)
    runs whenever a boundary value makes u nonzero, and leaves the CG warm start x0 set.
    """
    if name == "cav":
        sim = O.cavity(re=100, n=24, pressure_solver="cg", tol=None)
    elif name == "cyl":
        sim = O.cylinder(re=20, nx=110, ny=21, pressure_solver="cg", tol=None)
    elif name == "per":
        grid = O.OGrid(32, 32, 1.0, 1.0)
        grid.add_obstacle(O.circle_mask(grid, 0.5, 0.5, 0.15))
        bcs = {"left": O.OBC("periodic"), "right": O.OBC("periodic"), "bottom": O.OBC("slip"),
               "top": O.OBC("slip")}
        sim = O.OSimulation(grid, bcs, nu=0.02, pressure_solver="cg")
    else:
        grid = O.OGrid(30, 20, 1.5, 1.0)
        grid.add_obstacle(O.rectangle_mask(grid, 0.7, -1.0, 0.8, 2.0))
        sim = O.OSimulation(grid, {s: O.OBC("noslip") for s in O.SIDES}, nu=0.02,
                            pressure_solver="cg")
    assert np.array_equal(sim.grid.fluid, g[name + "_fluid"])
    sim.pressure.tol = 1e-10
    return sim.pressure


@pytest.mark.parametrize("name", ["cav", "cyl", "per", "two"])
def test_pressure_operator_and_cg(name):
    g = golden("golden_pressure")
    ps = _pressure_oracle(name, g)
    assert np.array_equal(ps.diag[ps.fluid], g[name + "_diag"][ps.fluid])
    assert np.array_equal(ps.labels, g[name + "_labels"])
    assert np.array_equal(np.array(ps.pinned, dtype=np.int64).reshape(-1, 2), g[name + "_pinned"])
    assert list(ps.neumann_components) == list(g[name + "_neumann"])
    for s in O.SIDES:
        assert np.array_equal(ps.dirichlet[s], g[name + "_dir_" + s])
    # the stencil matvec equals the assembled CSR product bit for bit
    rng = np.random.default_rng(5)
    x = rng.standard_normal(ps.n)
    assert np.array_equal(ps.matvec(x), ps._assemble() @ x)
    p = ps.solve(g[name + "_rhs"])
    assert ps.last_iterations == int(g[name + "_its"])
    assert rel(p, g[name + "_p"]) < 1e-12
    p2 = ps.solve(g[name + "_rhs2"])
    assert ps.last_iterations == int(g[name + "_its2"])
    assert rel(p2, g[name + "_p2"]) < 1e-12


# ---------------------------------------------------------------- time stepping
def test_cavity_200_steps():
    g = golden("golden_cavity64")
    sim = O.cavity(re=100, n=64, gamma=0.1, tau=0.5, tol=1e-8)
    for n in range(1, 201):
        sim.step()
        if n in (1, 10, 200):
            for f in "uvp":
                assert rel(getattr(sim, f), g[f"cav_{f}_{n}"]) < 1e-12, (f, n)
    assert np.array_equal(np.array(sim.iterations), g["cav_its"][:200])
    assert np.array_equal(np.array(sim.hist["dt"]), g["cav_dt"][:200])


def test_cylinder_with_scalar_10_steps():
    g = golden("golden_cylinder440")
    sim = O.cylinder(re=100, nx=440, ny=82, tol=1e-8)
    O.add_scalar(sim, "c", 1e-3, inflow_band=(0.15, 0.25), limiter="vanleer")
    for n in range(1, 11):
        sim.step()
        if n in (1, 10):
            for f in "uvp":
                assert rel(getattr(sim, f), g[f"cyl_{f}_{n}"]) < 1e-12, (f, n)
            assert rel(sim.scalars["c"].phi, g[f"cyl_c_{n}"]) < 1e-12
    assert np.array_equal(np.array(sim.iterations), g["cyl_its"])
    assert rel(sim.hist["fx"], g["cyl_hist_fx"]) < 1e-12
    assert rel(sim.hist["fy"], g["cyl_hist_fy"]) < 1e-10


def test_sst_channel_20_steps():
    g = golden("golden_sst128x192")
    sim = O.sst_channel(128, 192, seed=0, tol=1e-8)
    for n in range(1, 21):
        sim.step()
        if n in (1, 20):
            for f in "uvp":
                assert rel(getattr(sim, f), g[f"sst_{f}_{n}"]) < 1e-12, (f, n)
            assert rel(sim.scalars["k"].phi, g[f"sst_k_{n}"]) < 1e-12
            assert rel(sim.scalars["omega"].phi, g[f"sst_w_{n}"]) < 1e-12
            assert rel(sim.nu_t, g[f"sst_nut_{n}"]) < 1e-12
    assert sim.flow_force == pytest.approx(float(g["sst_flow_force"]), rel=1e-12)


def test_misc_runs():
    g = golden("golden_misc")
    sim = O.heated_cavity(ra=1e5, n=32, tol=1e-8)
    for _ in range(100):
        sim.step()
    for f in "uvp":
        assert rel(getattr(sim, f), g[f"hot_{f}_100"]) < 1e-12
    assert rel(sim.scalars["T"].phi, g["hot_T_100"]) < 1e-12

    grid = O.OGrid(32, 32, 1.0, 1.0)
    grid.add_obstacle(O.circle_mask(grid, 0.5, 0.5, 0.15))
    bcs = {"left": O.OBC("periodic"), "right": O.OBC("periodic"), "bottom": O.OBC("slip"),
           "top": O.OBC("slip")}
    sim = O.OSimulation(grid, bcs, nu=0.02, flow_rate=1.0, pressure_solver="cg", tol=1e-8)
    for _ in range(50):
        sim.step()
    for f in "uvp":
        assert rel(getattr(sim, f), g[f"pob_{f}_50"]) < 1e-12
    assert sim.flow_force == pytest.approx(float(g["pob_flow_force"]), rel=1e-12)

    sim = O.cavity(re=100, n=16, scheme="euler", gamma=0.5, tol=1e-8)
    for _ in range(30):
        sim.step()
    for f in "uvp":
        assert rel(getattr(sim, f), g[f"eul_{f}_30"]) < 1e-12


def test_smagorinsky_runs():
    """LES Smagorinsky (cfd2d/turbulence.py:130-160): the reference's own test case
    (tests/test_models.py:116-122), a periodic channel around a cylinder with wall
    damping and the cylinder without it, carrying a scalar."""
    g = golden("golden_smagorinsky")
    sim = O.cavity(re=1000, n=32, tol=1e-8)
    sim.add_model(O.OSmagorinsky())
    for n in range(1, 101):
        sim.step()
        if n in (1, 100):
            for f in "uvp":
                assert rel(getattr(sim, f), g[f"smc_{f}_{n}"]) < 1e-12, (f, n)
            assert rel(sim.nu_t, g[f"smc_nut_{n}"]) < 1e-12
    assert np.array_equal(np.array(sim.iterations), g["smc_its"])
    assert sim.nu_t[1:-1, 1:-1].max() > 0  # the reference test's own check

    grid = O.OGrid(32, 32, 1.0, 1.0)
    grid.add_obstacle(O.circle_mask(grid, 0.5, 0.5, 0.15))
    bcs = {"left": O.OBC("periodic"), "right": O.OBC("periodic"), "bottom": O.OBC("noslip"),
           "top": O.OBC("noslip")}
    sim = O.OSimulation(grid, bcs, nu=0.002, flow_rate=1.0, models=[O.OSmagorinsky(cs=0.2)],
                        pressure_solver="cg", tol=1e-8)
    for _ in range(50):
        sim.step()
    for f in ("u", "v", "p", "nu_t"):
        key = "nut" if f == "nu_t" else f
        assert rel(getattr(sim, f), g[f"smp_{key}_50"]) < 1e-12, f
    assert sim.flow_force == pytest.approx(float(g["smp_flow_force"]), rel=1e-12)

    sim = O.cylinder(re=1000, nx=110, ny=21, tol=1e-8)
    sim.add_model(O.OSmagorinsky(cs=0.1, wall_damping=False))
    O.add_scalar(sim, "c", 1e-4, inflow_band=(0.15, 0.25))
    for _ in range(30):
        sim.step()
    for f in ("u", "v", "p", "nu_t"):
        key = "nut" if f == "nu_t" else f
        assert rel(getattr(sim, f), g[f"smy_{key}_30"]) < 1e-12, f
    assert rel(sim.scalars["c"].phi, g["smy_c_30"]) < 1e-12


# ---------------------------------------------------------------- function objects
FO_POINTS = [(0.5, 0.2), (0.2, 0.2), (0.0, 0.0), (2.2, 0.41), (1.0, 0.05), (-0.1, 0.5), (0.31, 0.1337),
             (0.15, 0.2), (2.5, -0.2)]
FO_FIELDS = ("u", "v", "pressure", "vorticity", "speed", "streamfunction", "c")


def _fo_case():
    sim = O.cylinder(re=100, nx=88, ny=17, tol=1e-8)
    O.add_scalar(sim, "c", 1e-3, inflow_band=(0.15, 0.25))
    return sim


def _eq(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(a, b, equal_nan=True)


def test_function_objects_on_the_reference_state_bitwise():
    """Sampling, line sample and the VTK bytes of the oracle on the reference's own
    final state equal the reference's outputs bit for bit (cfd2d/functions.py:24-287)."""
    g = golden("golden_functions")
    sim = _fo_case()
    sim.u, sim.v, sim.p = g["fo_u"], g["fo_v"], g["fo_p"]
    sim.scalars["c"].phi[:] = g["fo_c"]
    sim.t, sim.dt = float(g["fo_t"]), float(g["fo_dt"])
    xs, ys = [p[0] for p in FO_POINTS], [p[1] for p in FO_POINTS]
    for f in FO_FIELDS:
        assert _eq(O.sample_field(sim, f, xs, ys), g[f"fo_probe_{f}"][-1]), f
    s, x, y = O.line_points((0.0, 0.1), (2.2, 0.3), 37)
    assert _eq(s, g["fo_line_s"]) and _eq(x, g["fo_line_x"]) and _eq(y, g["fo_line_y"])
    for f in ("u", "v", "pressure", "c"):
        assert _eq(O.sample_field(sim, f, x, y), g[f"fo_line_{f}"]), f
    assert O.write_vtk_bytes(sim) == g["fo_vtk"].tobytes()


def test_probe_series_and_field_average_runs():
    """Probes and FieldAverage executed after each of 30 oracle steps match the
    reference's series and sums (cfd2d/functions.py:59-80, 180-204)."""
    g = golden("golden_functions")
    sim = _fo_case()
    fa = O.OFieldAverage(t_start=0.01)
    xs, ys = [p[0] for p in FO_POINTS], [p[1] for p in FO_POINTS]
    rows = {f: [] for f in FO_FIELDS}
    ts = []
    for _ in range(30):
        sim.step()
        ts.append(sim.t)
        for f in FO_FIELDS:
            rows[f].append(O.sample_field(sim, f, xs, ys))
        fa.execute(sim)
    assert rel(ts, g["fo_probe_t"]) < 1e-13
    for f in FO_FIELDS:
        a, b = np.array(rows[f]), g[f"fo_probe_{f}"]
        assert np.array_equal(np.isnan(a), np.isnan(b)), f
        assert rel(np.nan_to_num(a), np.nan_to_num(b)) < 1e-11, f
    assert fa.T == pytest.approx(float(g["fo_avg_T"]), rel=1e-13)
    for k in ("u", "v", "p"):
        for name, mine in (("sum", fa.sum[k]), ("sum2", fa.sum2[k])):
            ref = g[f"fo_avg_{name}_{k}"]
            assert np.array_equal(np.isnan(mine), np.isnan(ref))
            assert rel(np.nan_to_num(mine), np.nan_to_num(ref)) < 1e-11, (name, k)


# ---------------------------------------------------------------- VOF
def test_vof_advect_bitwise():
    """cfd2d/vof.py:36-137 on seeded inputs (periodic or not, with and without
    compression, random solids): bit for bit."""
    from inputs import vof_cases

    g = golden("golden_vof")
    k = 0
    for c in vof_cases():
        out = np.full_like(c["a"], 5.0)
        O.vof_advect(c["a"], c["u"], c["v"], c["fluid"], c["nx"], c["ny"], c["dx"], c["dy"], c["dt"],
                     c["c_alpha"], c["periodic"], c["a_in"], out)
        assert np.array_equal(out, g[f"adv{k}_out"]), k
        k += 1
    assert k == int(g["n_adv"])


def _vof_pressure_sims():
    sims = {}
    grid = O.OGrid(30, 20, 1.5, 1.0)
    grid.add_obstacle(O.rectangle_mask(grid, 0.7, -1.0, 0.8, 2.0))
    sims["two"] = O.OSimulation(grid, {s: O.OBC("noslip") for s in O.SIDES}, nu=0.02)
    grid = O.OGrid(32, 32, 0.584, 0.584)
    grid.add_obstacle(O.rectangle_mask(grid, 0.28, 0.0, 0.304, 0.048))
    sims["open"] = O.OSimulation(grid, {"left": O.OBC("noslip"), "right": O.OBC("noslip"),
                                        "bottom": O.OBC("noslip"), "top": O.OBC("outflow")}, nu=1e-6)
    grid = O.OGrid(32, 24, 1.0, 0.75)
    grid.add_obstacle(O.circle_mask(grid, 0.5, 0.4, 0.12))
    sims["per"] = O.OSimulation(grid, {"left": O.OBC("periodic"), "right": O.OBC("periodic"),
                                       "bottom": O.OBC("noslip"), "top": O.OBC("slip")}, nu=0.01)
    return sims


def face_coefficients(rho, nx, periodic):
    bx = 2.0 / (rho[:-1, :] + rho[1:, :])
    by = 2.0 / (rho[:, :-1] + rho[:, 1:])
    if periodic:
        bx[nx, :] = 2.0 / (rho[nx, :] + rho[1, :])
    return bx, by


def test_solve_variable():
    """cfd2d/pressure.py:187-244 (sparse direct) with a 1000:1 density interface:
    two Neumann components, an open top, periodic x."""
    g = golden("golden_vof")
    for name, sim in _vof_pressure_sims().items():
        rho = g[f"sv_{name}_rho"]
        bx, by = face_coefficients(rho, sim.grid.nx, sim.periodic)
        p = sim.pressure.solve_variable(g[f"sv_{name}_rhs"], bx[:, 1:-1], by[1:-1, :])
        assert rel(p, g[f"sv_{name}_p"]) < 1e-12, name


def test_dam_break_20_steps():
    """The reference's dam break (cfd2d/cases.py:294-320) on 32 x 32: VOF transport,
    surface tension, variable-density projection."""
    g = golden("golden_vof")
    sim = O.dam_break(n=32)
    vof = sim.model("multiphase")
    for n in range(1, 21):
        sim.step()
        if n in (1, 20):
            for f in "uvp":
                assert rel(getattr(sim, f), g[f"dam_{f}_{n}"]) < 1e-10, (f, n)
            assert rel(vof.alpha, g[f"dam_alpha_{n}"]) < 1e-10, n
    assert rel(sim.hist["dt"], g["dam_dt"]) < 1e-12
    assert vof.volume() == pytest.approx(float(g["dam_volume"]), rel=1e-12)


def test_vof_vtk_bytes_on_the_reference_state():
    """The VTK file of the reference's dam break after 20 steps (alpha, rho, no nu_t:
    cfd2d/visualization.py:86-88) from the oracle, byte for byte."""
    g = golden("golden_vof")
    sim = O.dam_break(n=32)
    vof = sim.model("multiphase")
    sim.u, sim.v, sim.p = g["dam_u_20"].copy(), g["dam_v_20"].copy(), g["dam_p_20"].copy()
    vof.alpha[:] = g["dam_alpha_20"]
    vof.update_properties()
    sim.t = float(g["dam_t"])
    assert O.write_vtk_bytes(sim) == g["dam_vtk"].tobytes()


# ---------------------------------------------------------------- polygon, NACA, image obstacles
def _shape_image(g, k, tmp_path):
    from PIL import Image

    name = str(g[f"img{k}_name"])
    path = tmp_path / f"{name}_{k}.png"
    Image.fromarray(g[f"pixels_{name}"]).save(path)
    kw = {}
    for item in g[f"img{k}_kw"]:
        a, b = str(item).split("=")
        kw[a] = b == "True" if b in ("True", "False") else float(b)
    return path, kw


def test_naca_outline_and_image_masks_bitwise(tmp_path):
    g = golden("golden_shapes")
    for k in range(int(g["n_naca"])):
        code, chord, n, closed = g[f"naca{k}_spec"]
        pts = O.naca4_coordinates(str(code), float(chord), int(n), bool(int(closed)))
        assert np.array_equal(pts, g[f"naca{k}_pts"]), k
    for k in range(int(g["n_img"])):
        nx, ny, lx, ly = g[f"img{k}_grid"]
        path, kw = _shape_image(g, k, tmp_path)
        og = O.OGrid(int(nx), int(ny), lx, ly)
        m = O.image_mask(og, path, **kw)
        assert np.array_equal(m, g[f"img{k}_mask"]), k


def _exact_inside(points, X, Y):
    """Crossing count in exact rational arithmetic for a point on no edge."""
    from fractions import Fraction as F

    pts = [(F(float(a)), F(float(b))) for a, b in points]
    X, Y = F(float(X)), F(float(Y))
    inside, on_edge = False, False
    for (x0, y0), (x1, y1) in zip(pts[-1:] + pts[:-1], pts):
        cross = (x1 - x0) * (Y - y0) - (y1 - y0) * (X - x0)
        if cross == 0 and min(x0, x1) <= X <= max(x0, x1) and min(y0, y1) <= Y <= max(y0, y1):
            on_edge = True
        if (y0 > Y) != (y1 > Y):
            xs = x0 + (Y - y0) * (x1 - x0) / (y1 - y0)
            if xs > X:
                inside = not inside
    return inside, on_edge


def test_polygon_crossing_test_against_exact_arithmetic():
    """The restated crossings test (matplotlib's Path.contains_points, which the
    reference calls, is not installed here) against an exact rational crossing count at
    every cell centre that lies on no edge, for star-shaped and self-intersecting
    polygons and NACA outlines."""
    rng = np.random.default_rng(5)
    og = O.OGrid(37, 29, 1.0, 0.8)
    X, Y = og.centres()
    polys = []
    for n in (3, 5, 9, 17):
        ang = np.sort(rng.uniform(0, 2 * np.pi, n))
        r = rng.uniform(0.1, 0.38, n)
        polys.append(np.column_stack([0.5 + r * np.cos(ang), 0.4 + r * np.sin(ang)]))
    polys.append(rng.uniform(0.05, 0.95, (7, 2)) * [1.0, 0.8])  # self-intersecting
    pts = O.naca4_coordinates("2412", 0.7)
    a = np.deg2rad(12.0)
    polys.append(np.column_stack([pts[:, 0] * np.cos(a) + pts[:, 1] * np.sin(a) + 0.15,
                                  -pts[:, 0] * np.sin(a) + pts[:, 1] * np.cos(a) + 0.45]))
    checked = 0
    for P in polys:
        m = O.polygon_mask(og, P)
        for i in range(og.nx):
            for j in range(og.ny):
                inside, on_edge = _exact_inside(P, X[i, j], Y[i, j])
                if not on_edge:
                    assert m[i, j] == inside, (i, j)
                    checked += 1
    assert checked > 5000


def test_reference_shape_tests_on_the_oracle(tmp_path):
    """tests/test_cfd2d.py:121-145 of the reference on the restated shapes."""
    from PIL import Image

    pts = O.naca4_coordinates("0012", chord=1.0)
    assert pts[:, 1].max() - pts[:, 1].min() == pytest.approx(0.12, rel=0.02)
    og = O.OGrid(200, 100, 2.0, 1.0)
    m = O.naca4_mask(og, "0012", 0.5, 0.5, 1.0, 0.0)
    assert m.sum() * og.dx * og.dy == pytest.approx(0.0822, rel=0.05)
    img = np.full((50, 100), 255, dtype=np.uint8)
    img[10:40, 20:40] = 0
    path = tmp_path / "hindernis.png"
    Image.fromarray(img).save(path)
    og = O.OGrid(100, 50, 2.0, 1.0)
    m = O.image_mask(og, path)
    assert m.sum() == pytest.approx(30 * 20, rel=0.05)
    yc = (np.arange(og.ny) + 0.5) * og.dy
    ys = yc[np.where(m.any(axis=0))[0]]
    assert ys.min() == pytest.approx(0.2, abs=0.03) and ys.max() == pytest.approx(0.8, abs=0.03)

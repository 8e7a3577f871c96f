"""Generate the golden fixtures in this folder by running the reference solver.

Run in a container that holds the reference checkout (default
``/root/reference``; override with ``CFD2D_REFERENCE``)::

    python tests/golden/make_golden.py [group ...]

Groups: kernels geometry pressure cavity cylinder sst misc checkpoint smagorinsky
functions vof validation shapes obstacles cylinder_long (default: all).
The reference imports matplotlib at module load; ``mplstub/`` stands in for it
(no fixture case needs plotting or polygon masks; NACA outlines and image
obstacles do not use it). Every pressure solve uses the
reference's own ``PressureSolver`` (scipy CG or SuperLU) with
``sim.pressure.tol`` set after construction, exactly as a user of the reference
would. Nothing at test time imports this script or the reference.
"""

from __future__ import annotations

import os
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF = os.environ.get("CFD2D_REFERENCE", "/root/reference")
sys.path.insert(0, str(HERE / "mplstub"))
sys.path.insert(0, REF)
sys.path.insert(0, str(HERE))

import numpy as np  # noqa: E402

from cfd2d import cases, geometry, kernels  # noqa: E402
from cfd2d.boundary import BoundaryCondition as BC  # noqa: E402
from cfd2d.grid import Grid  # noqa: E402
from cfd2d.models import PassiveScalar  # noqa: E402
from cfd2d.solver import Simulation  # noqa: E402
from cfd2d.turbulence import KOmegaSST  # noqa: E402

TOL = 1e-8


def _save(name, d):
    path = HERE / f"{name}.npz"
    np.savez_compressed(path, **d)
    print(f"wrote {path.name}: {path.stat().st_size / 1024:.0f} KiB", flush=True)


def gen_kernels():
    from inputs import momentum_cases, scalar_cases

    out = {}
    k = 0
    for c in momentum_cases():
        u, v = c["u"], c["v"]
        hu = np.full_like(u, 7.0)
        hv = np.full_like(v, 7.0)
        kernels.momentum_tendencies(u, v, c["fluid"], c["nx"], c["ny"], c["dx"], c["dy"], c["nu"],
                                    c["variable"], c["gamma"], c["periodic"], hu, hv, c["rho"],
                                    c["var_density"])
        uo, vo = u.copy(), v.copy()
        kernels.obstacle_bc(uo, vo, c["fluid"], c["nx"], c["ny"], c["periodic"])
        out.update({f"m{k}_hu": hu, f"m{k}_hv": hv, f"m{k}_u_obc": uo, f"m{k}_v_obc": vo})
        k += 1
    out["n_momentum"] = np.array(k)
    k = 0
    for c in scalar_cases():
        o = np.full_like(c["phi"], 3.0)
        bt, bv = c["bt"], c["bv"]
        kernels.scalar_transport(c["phi"], c["u"], c["v"], c["fluid"], c["nx"], c["ny"], c["dx"],
                                 c["dy"], c["diff"], c["limiter"], c["periodic"], bt["l"], bv["l"],
                                 bt["r"], bv["r"], bt["b"], bv["b"], bt["t"], bv["t"], c["obs_t"],
                                 c["obs_v"], o)
        out[f"s{k}_out"] = o
        k += 1
    out["n_scalar"] = np.array(k)
    _save("golden_kernels", out)


# --------------------------------------------------------------------------- #
def gen_geometry():
    rng = np.random.default_rng(77)
    out = {}
    k = 0
    for nx, ny, lx, ly in ((440, 82, 2.2, 0.41), (97, 61, 1.0, 0.7), (256, 128, 2.0, 1.0),
                           (1024, 512, 2.0, 1.0)):
        g = Grid(nx, ny, lx, ly)
        for _ in range(4):
            xc = float(rng.uniform(0.1, 0.9) * lx)
            yc = float(rng.uniform(0.1, 0.9) * ly)
            r = float(rng.uniform(0.02, 0.2) * ly)
            a = float(rng.uniform(0.02, 0.2) * ly)
            b = float(rng.uniform(0.02, 0.2) * ly)
            ang = float(rng.uniform(0, 180))
            out[f"g{k}_grid"] = np.array([nx, ny, lx, ly])
            out[f"g{k}_circle"] = np.array([xc, yc, r])
            out[f"g{k}_circle_mask"] = geometry.circle(g, xc, yc, r)
            out[f"g{k}_ellipse"] = np.array([xc, yc, a, b, ang])
            out[f"g{k}_ellipse_mask"] = geometry.ellipse(g, xc, yc, a, b, ang)
            rect = (xc - a, yc - b, xc + a, yc + b)
            out[f"g{k}_rect"] = np.array(rect)
            out[f"g{k}_rect_mask"] = geometry.rectangle(g, *rect)
            k += 1
    # the cylinder of the cylinder case exactly (cases.py:92-94)
    g = Grid(440, 82, 2.2, 0.41)
    out["cyl_mask"] = geometry.circle(g, 0.2, 0.2, 0.1 / 2)
    out["n_shapes"] = np.array(k)
    # finalize: a ring encloses fluid, and a second case with a single region
    g = Grid(60, 40, 1.5, 1.0)
    X, Y = g.cell_centers()
    ring = ((X - 0.7) ** 2 + (Y - 0.5) ** 2 <= 0.3 ** 2) & ((X - 0.7) ** 2 + (Y - 0.5) ** 2 > 0.2 ** 2)
    g.add_obstacle(ring)
    out["fin_before"] = g.fluid.copy()
    out["fin_removed"] = np.array(g.finalize())
    out["fin_after"] = g.fluid.copy()
    _save("golden_geometry", out)


# --------------------------------------------------------------------------- #
def _pressure_case(name, sim, rng, out):
    ps = sim.pressure
    nx, ny = sim.grid.nx, sim.grid.ny
    diag = np.zeros((nx, ny))
    diag[ps.fluid] = ps.A.diagonal()
    out[name + "_fluid"] = sim.grid.fluid.copy()
    out[name + "_diag"] = diag
    out[name + "_labels"] = ps.labels
    out[name + "_pinned"] = np.array(ps._pinned, dtype=np.int64).reshape(-1, 2)
    out[name + "_neumann"] = np.array(ps.neumann_components, dtype=np.int64)
    for s in ("left", "right", "bottom", "top"):
        out[name + "_dir_" + s] = np.asarray(ps.dirichlet[s])
    rhs = rng.standard_normal((nx, ny))
    rhs[~ps.fluid] = 0.0
    ps.tol = 1e-10
    p = ps.solve(rhs)
    out[name + "_rhs"] = rhs
    out[name + "_p"] = p
    out[name + "_its"] = np.array(ps.last_iterations)
    # second solve warm-started from the first (the CG keeps x0 between solves)
    rhs2 = rhs + 0.1 * rng.standard_normal((nx, ny))
    rhs2[~ps.fluid] = 0.0
    p2 = ps.solve(rhs2)
    out[name + "_rhs2"] = rhs2
    out[name + "_p2"] = p2
    out[name + "_its2"] = np.array(ps.last_iterations)


def gen_pressure():
    rng = np.random.default_rng(99)
    out = {}
    _pressure_case("cav", cases.lid_driven_cavity(re=100, n=24, pressure_solver="cg").sim, rng, out)
    _pressure_case("cyl", cases.cylinder_flow(re=20, nx=110, ny=21, pressure_solver="cg").sim, rng, out)
    g = Grid(32, 32, 1.0, 1.0)
    g.add_obstacle(geometry.circle(g, 0.5, 0.5, 0.15))
    bcs = dict(left=BC("periodic"), right=BC("periodic"), bottom=BC("slip"), top=BC("slip"))
    _pressure_case("per", Simulation(g, bcs, nu=0.02, pressure_solver="cg"), rng, out)
    # a wall across a closed box gives two Neumann components
    g = Grid(30, 20, 1.5, 1.0)
    g.add_obstacle(geometry.rectangle(g, 0.7, -1.0, 0.8, 2.0))
    bcs = {s: BC("noslip") for s in ("left", "right", "bottom", "top")}
    _pressure_case("two", Simulation(g, bcs, nu=0.02, pressure_solver="cg"), rng, out)
    _save("golden_pressure", out)


# --------------------------------------------------------------------------- #
def _run(sim, nsteps, keep_at, fields, out, prefix):
    its, dts = [], []
    hist_keys = ("divergence", "kinetic_energy", "fx", "fy")
    t0 = time.time()
    for n in range(1, nsteps + 1):
        sim.step()
        its.append(sim.pressure.last_iterations)
        dts.append(sim.dt)
        if n in keep_at:
            for name, getter in fields.items():
                out[f"{prefix}_{name}_{n}"] = np.array(getter(sim), copy=True)
    out[prefix + "_its"] = np.array(its)
    out[prefix + "_dt"] = np.array(dts)
    out[prefix + "_residual_last"] = np.array(sim.residual)
    out[prefix + "_t"] = np.array(sim.t)
    for k in hist_keys:
        val = getattr(sim.history, k)
        if val:
            out[prefix + "_hist_" + k] = np.array(val)
    if sim.flow_rate is not None:
        out[prefix + "_hist_flow_force"] = np.array(sim.history.extra["antriebskraft"])
    # the models' monitors, recorded after every step (cfd2d/solver.py:441-443)
    for k, vals in sim.history.extra.items():
        if k != "antriebskraft":
            out[prefix + "_extra_" + k] = np.array(vals, dtype=float)
    print(f"{prefix}: {nsteps} steps in {time.time() - t0:.1f}s, mean CG it {np.mean(its):.1f}",
          flush=True)


UVP = {"u": lambda s: s.u, "v": lambda s: s.v, "p": lambda s: s.p}


def gen_cavity():
    out = {}
    case = cases.lid_driven_cavity(re=100, n=64, scheme="ab2", gamma=0.1, tau=0.5,
                                   pressure_solver="cg")
    case.sim.pressure.tol = TOL
    _run(case.sim, 2000, {1, 10, 200, 2000}, UVP, out, "cav")
    _save("golden_cavity64", out)


def gen_cylinder():
    out = {}
    case = cases.build_case({"fall": "cylinder", "parameter": {"re": 100, "nx": 440, "ny": 82},
                             "numerik": {"pressure_solver": "cg"},
                             "skalar": {"name": "c", "diffusivity": 1e-3, "inflow_band": [0.15, 0.25],
                                        "limiter": "vanleer"}})
    case.sim.pressure.tol = TOL
    f = dict(UVP)
    f["c"] = lambda s: s.scalars["c"].phi
    _run(case.sim, 10, {1, 10}, f, out, "cyl")
    _save("golden_cylinder440", out)


def _sst_channel(nx, ny, seed):
    g = Grid(nx, ny, 2 * np.pi, 2.0)
    bcs = dict(left=BC("periodic"), right=BC("periodic"), bottom=BC("noslip"), top=BC("noslip"))
    nu = 2.0 / 1e4
    k0, w0 = 1e-3, 10.0
    sst = KOmegaSST(intensity=np.sqrt(k0 / 1.5), viscosity_ratio=k0 / (nu * w0), U_ref=1.0)
    sim = Simulation(g, bcs, nu=nu, flow_rate=1.0, models=[sst], pressure_solver="cg")
    sim.pressure.tol = TOL
    rng = np.random.default_rng(seed)
    y = (np.arange(ny) + 0.5) * g.dy
    prof = 1.5 * y * (2.0 - y)
    sim.u[1:nx + 1, 1:ny + 1] = prof[None, :] * (1.0 + 0.05 * rng.uniform(-1.0, 1.0, (nx, ny)))
    sim.v[1:nx + 1, 1:ny] = 0.05 * rng.uniform(-1.0, 1.0, (nx, ny - 1))
    sim.u[~sim.u_fluid] = 0.0
    sim.v[~sim.v_fluid] = 0.0
    sim._apply_bc()
    sim._project_initial()
    return sim


def gen_sst():
    out = {}
    sim = _sst_channel(128, 192, 0)
    f = dict(UVP)
    f["k"] = lambda s: s.scalars["k"].phi
    f["w"] = lambda s: s.scalars["omega"].phi
    f["nut"] = lambda s: s.nu_t
    _run(sim, 20, {1, 20}, f, out, "sst")
    out["sst_flow_force"] = np.array(sim.flow_force)
    _save("golden_sst128x192", out)


def gen_misc():
    out = {}
    # heated cavity (Boussinesq) 32x32
    case = cases.heated_cavity(ra=1e5, n=32, pressure_solver="cg")
    case.sim.pressure.tol = TOL
    f = dict(UVP)
    f["T"] = lambda s: s.scalars["T"].phi
    _run(case.sim, 100, {100}, f, out, "hot")
    # periodic channel with an obstacle, flow-rate control with re-projection
    g = Grid(32, 32, 1.0, 1.0)
    g.add_obstacle(geometry.circle(g, 0.5, 0.5, 0.15))
    bcs = dict(left=BC("periodic"), right=BC("periodic"), bottom=BC("slip"), top=BC("slip"))
    sim = Simulation(g, bcs, nu=0.02, flow_rate=1.0, pressure_solver="cg")
    sim.pressure.tol = TOL
    _run(sim, 50, {50}, UVP, out, "pob")
    out["pob_flow_force"] = np.array(sim.flow_force)
    # explicit Euler, fixed gamma (tests/test_cfd2d.py:97-102 setting)
    case = cases.lid_driven_cavity(re=100, n=16, scheme="euler", pressure_solver="cg", gamma=0.5)
    case.sim.pressure.tol = TOL
    _run(case.sim, 30, {30}, UVP, out, "eul")
    # obstacle flow of the learned-preconditioner family at reduced size
    obst = [{"typ": "kreis", "x": 0.5, "y": 0.45, "r": 0.06},
            {"typ": "ellipse", "x": 1.0, "y": 0.6, "a": 0.07, "b": 0.03, "winkel": 30.0},
            {"typ": "rechteck", "x0": 1.4, "y0": 0.2, "x1": 1.48, "y1": 0.3}]
    case = cases.custom_obstacles(obst, lx=2.0, ly=1.0, nx=256, ny=128, re=500.0,
                                  inflow_profile="uniform", walls="slip", pressure_solver="cg")
    case.sim.pressure.tol = TOL
    _run(case.sim, 5, {5}, UVP, out, "obs")
    # run() with the last step shortened to land on t_end (cfd2d/solver.py:466-480)
    case = cases.cylinder_flow(re=20, nx=110, ny=21, t_end=0.1, pressure_solver="cg")
    case.sim.pressure.tol = TOL
    reason = case.sim.run(0.1, verbose=False)
    out["run_u"] = case.sim.u.copy()
    out["run_n"] = np.array(case.sim.n)
    out["run_t"] = np.array(case.sim.t)
    out["run_dt_last"] = np.array(case.sim.dt)
    out["run_reason"] = np.array(reason)
    _save("golden_misc", out)


def gen_smagorinsky():
    """The Smagorinsky model (cfd2d/turbulence.py:130-160) on three cases: the
    reference's own test setting (tests/test_models.py:116-122, cavity Re 1000 on
    32 x 32, 100 steps), a periodic channel around a cylinder (periodic nu_t ghosts,
    interior solid, flow-rate control) and the 110 x 21 cylinder without wall
    damping carrying a scalar whose diffusivity takes nu_t / Sc_t."""
    out = {}
    f = dict(UVP)
    f["nut"] = lambda s: s.nu_t
    case = cases.add_turbulence(cases.lid_driven_cavity(re=1000, n=32, pressure_solver="cg"),
                                "Smagorinsky")
    case.sim.pressure.tol = TOL
    _run(case.sim, 100, {1, 100}, f, out, "smc")
    g = Grid(32, 32, 1.0, 1.0)
    g.add_obstacle(geometry.circle(g, 0.5, 0.5, 0.15))
    bcs = dict(left=BC("periodic"), right=BC("periodic"), bottom=BC("noslip"), top=BC("noslip"))
    from cfd2d.turbulence import Smagorinsky

    sim = Simulation(g, bcs, nu=0.002, flow_rate=1.0, models=[Smagorinsky(cs=0.2)],
                     pressure_solver="cg")
    sim.pressure.tol = TOL
    _run(sim, 50, {50}, f, out, "smp")
    out["smp_flow_force"] = np.array(sim.flow_force)
    case = cases.cylinder_flow(re=1000, nx=110, ny=21, pressure_solver="cg")
    cases.add_turbulence(case, "Smagorinsky", cs=0.1, wall_damping=False)
    cases.add_scalar(case, "c", 1e-4, inflow_band=(0.15, 0.25))
    case.sim.pressure.tol = TOL
    fc = dict(f)
    fc["c"] = lambda s: s.scalars["c"].phi
    _run(case.sim, 30, {30}, fc, out, "smy")
    _save("golden_smagorinsky", out)


FO_POINTS = [(0.5, 0.2), (0.2, 0.2), (0.0, 0.0), (2.2, 0.41), (1.0, 0.05), (-0.1, 0.5), (0.31, 0.1337),
             (0.15, 0.2), (2.5, -0.2)]
FO_FIELDS = ("u", "v", "pressure", "vorticity", "speed", "streamfunction", "c")


def gen_functions():
    """Function objects of the reference (cfd2d/functions.py) on the 88 x 17 cylinder
    with a passive scalar: probes of every field kind at points inside, on walls,
    in the obstacle and outside the domain, a time average started after the first
    steps, a slanted line sample and the VTK file after 30 steps."""
    import tempfile

    from cfd2d import functions

    case = cases.cylinder_flow(re=100, nx=88, ny=17, pressure_solver="cg")
    cases.add_scalar(case, "c", 1e-3, inflow_band=(0.15, 0.25))
    sim = case.sim
    sim.pressure.tol = TOL
    pr = functions.Probes(FO_POINTS, fields=FO_FIELDS)
    fa = functions.FieldAverage(t_start=0.01)
    sim.function_objects += [pr, fa]
    for _ in range(30):
        sim.step()
    out = {"fo_u": sim.u.copy(), "fo_v": sim.v.copy(), "fo_p": sim.p.copy(),
           "fo_c": sim.scalars["c"].phi.copy(), "fo_t": np.array(sim.t), "fo_dt": np.array(sim.dt),
           "fo_probe_t": np.array(pr.t)}
    for f in FO_FIELDS:
        out[f"fo_probe_{f}"] = np.array(pr.data[f])
    out["fo_avg_T"] = np.array(fa.T)
    for k in ("u", "v", "p"):
        out[f"fo_avg_sum_{k}"] = fa.sum[k]
        out[f"fo_avg_sum2_{k}"] = fa.sum2[k]
    ls = functions.LineSample((0.0, 0.1), (2.2, 0.3), n=37, fields=["u", "v", "pressure", "c"], label="schraeg")
    for k, v in ls.sample(sim).items():
        out[f"fo_line_{k}"] = np.asarray(v)
    with tempfile.TemporaryDirectory() as td:
        raw = functions.write_vtk(sim, Path(td) / "f.vtk").read_bytes()
    out["fo_vtk"] = np.frombuffer(raw, dtype=np.uint8)
    _save("golden_functions", out)


def _face_coefficients(rho, nx, periodic):
    # cfd2d/solver.py:267-271
    bx = 2.0 / (rho[:-1, :] + rho[1:, :])
    by = 2.0 / (rho[:, :-1] + rho[:, 1:])
    if periodic:
        bx[nx, :] = 2.0 / (rho[nx, :] + rho[1, :])
    return bx, by


def gen_vof():
    """The VOF path of the reference (cfd2d/vof.py, PressureSolver.solve_variable):
    vof_advect on seeded inputs, solve_variable (sparse direct) on three geometries
    with a 1000:1 density interface, and a 32 x 32 dam break over 20 steps."""
    import tempfile

    from inputs import rho_field, vof_cases

    from cfd2d import functions
    from cfd2d.vof import vof_advect

    out = {}
    k = 0
    for c in vof_cases():
        o = np.full_like(c["a"], 5.0)
        vof_advect(c["a"], c["u"], c["v"], c["fluid"], c["nx"], c["ny"], c["dx"], c["dy"], c["dt"],
                   c["c_alpha"], c["periodic"], c["a_in"], o)
        out[f"adv{k}_out"] = o
        k += 1
    out["n_adv"] = np.array(k)
    rng = np.random.default_rng(77)
    sims = {}
    g = Grid(30, 20, 1.5, 1.0)
    g.add_obstacle(geometry.rectangle(g, 0.7, -1.0, 0.8, 2.0))
    sims["two"] = Simulation(g, {s: BC("noslip") for s in ("left", "right", "bottom", "top")}, nu=0.02)
    g = Grid(32, 32, 0.584, 0.584)
    g.add_obstacle(geometry.rectangle(g, 0.28, 0.0, 0.304, 0.048))
    sims["open"] = Simulation(g, {"left": BC("noslip"), "right": BC("noslip"), "bottom": BC("noslip"),
                                  "top": BC("outflow")}, nu=1e-6)
    g = Grid(32, 24, 1.0, 0.75)
    g.add_obstacle(geometry.circle(g, 0.5, 0.4, 0.12))
    sims["per"] = Simulation(g, {"left": BC("periodic"), "right": BC("periodic"), "bottom": BC("noslip"),
                                 "top": BC("slip")}, nu=0.01)
    for name, sim in sims.items():
        nx, ny = sim.grid.nx, sim.grid.ny
        rho = rho_field(rng, nx, ny, sim.grid.fluid)
        bx, by = _face_coefficients(rho, nx, sim.periodic)
        rhs = rng.standard_normal((nx, ny))
        rhs[~sim.pressure.fluid] = 0.0
        p = sim.pressure.solve_variable(rhs, bx[:, 1:-1], by[1:-1, :])
        out[f"sv_{name}_rho"] = rho
        out[f"sv_{name}_rhs"] = rhs
        out[f"sv_{name}_p"] = p
    case = cases.dam_break(n=32)
    f = dict(UVP)
    vof = case.sim.model("multiphase")
    f["alpha"] = lambda s: vof.alpha
    _run(case.sim, 20, {1, 20}, f, out, "dam")
    out["dam_volume"] = np.array(vof.volume())
    out["dam_t"] = np.array(case.sim.t)
    with tempfile.TemporaryDirectory() as td:
        raw = functions.write_vtk(case.sim, Path(td) / "dam.vtk").read_bytes()
    out["dam_vtk"] = np.frombuffer(raw, dtype=np.uint8)
    # the reference's default size, 100 steps
    case = cases.dam_break(n=96)
    vof = case.sim.model("multiphase")
    f = dict(UVP)
    f["alpha"] = lambda s: vof.alpha
    _run(case.sim, 100, {100}, f, out, "d96")
    _save("golden_vof", out)


def gen_validation():
    """The reference's validation tests (tests/test_cfd2d.py:57-95, tests/test_models.py:
    69-84, 102-113) run by the reference itself: the physical figures each test checks,
    so the GPU runs can be compared with the reference's results rather than with the
    literature tables (which stay in the reference)."""
    from cfd2d import validation

    out = {}
    ys = np.linspace(0.0, 1.0, 33)
    case = cases.lid_driven_cavity(re=100, n=32)
    case.sim.run(40, steady_tol=1e-5, verbose=False)
    err = validation.cavity_centerline_errors(case.sim, 100)
    out["ghia_u_line"] = case.sim.sample_u(np.full_like(ys, 0.5), ys)
    out["ghia_v_line"] = case.sim.sample_v(ys, np.full_like(ys, 0.5))
    out["ghia_errors"] = np.array([err["u_max_fehler"], err["v_max_fehler"]])
    out["ghia_n"] = np.array(case.sim.n)
    case = cases.cylinder_flow(re=20, nx=220, ny=41, t_end=3.0)
    case.sim.run(case.t_end, verbose=False)
    fx, fy = case.sim.obstacle_forces()
    out["cyl20_cd_cl"] = np.array(validation.force_coefficients(fx, fy, 1.0, 0.1))
    out["cyl20_n"] = np.array(case.sim.n)
    case = cases.backward_facing_step(re=200, length=8, ny=16, t_end=30)
    case.sim.run(case.t_end, steady_tol=1e-4, verbose=False)
    out["step_xr"] = np.array(validation.reattachment_length(case.sim, case.info["x_stufe"]))
    out["step_n"] = np.array(case.sim.n)
    case = cases.heated_cavity(ra=1e4, n=32)
    case.sim.run(case.t_end, steady_tol=case.steady_tol, verbose=False)
    th = case.sim.model("thermal")
    out["dvd_nusselt"] = np.array([th.nusselt("left"), th.nusselt("right")])
    out["dvd_n"] = np.array(case.sim.n)
    for ra in (1200.0, 5000.0):
        case = cases.rayleigh_benard(ra=ra, ny=12, t_end=250)
        case.sim.run(case.t_end, steady_tol=1e-6, verbose=False)
        out[f"rb{int(ra)}_nusselt"] = np.array(case.sim.model("thermal").nusselt("bottom"))
        out[f"rb{int(ra)}_n"] = np.array(case.sim.n)
    case = cases.turbulent_channel(re_tau=120, y_plus_1=2.0, t_end=250)
    case.sim.run(case.t_end, steady_tol=1e-5, verbose=False)
    sim, g = case.sim, case.sim.grid
    u = sim.u[2, 1:-1]
    tau_w = sim.nu * 0.5 * (u[0] + u[-1]) / (0.5 * g.dy)  # as cfd2d/report.py:455-461
    utau = np.sqrt(max(tau_w, 1e-300))
    out["chan_cf_uplus"] = np.array([2 * tau_w / case.U_ref ** 2, u[g.ny // 2 - 1] / utau])
    out["chan_u"] = sim.u.copy()
    out["chan_n"] = np.array(sim.n)
    _save("golden_validation", out)


def gen_checkpoint():
    """A checkpoint written by the reference itself (cfd2d/functions.py:326) after 40
    steps of the 88 x 17 cylinder with a passive scalar, and the reference's state
    after 80 steps (tests/test_functions.py:48-70 setting, CG at 1e-12 so that the
    iterative GPU solve can be compared)."""
    import tempfile

    from cfd2d import functions

    spec = {"fall": "cylinder", "parameter": {"re": 100, "nx": 88, "ny": 17, "t_end": 0.2},
            "numerik": {"pressure_solver": "cg"},
            "skalar": {"name": "c", "diffusivity": 1e-3, "inflow_band": [0.15, 0.25]}}
    ref = cases.build_case(spec)
    ref.sim.pressure.tol = 1e-12
    for _ in range(80):
        ref.sim.step()
    a = cases.build_case(spec)
    a.sim.pressure.tol = 1e-12
    for _ in range(40):
        a.sim.step()
    with tempfile.TemporaryDirectory() as td:
        path = Path(td) / "cp.npz"
        functions.save_checkpoint(a.sim, path)
        cp = dict(np.load(path, allow_pickle=False))
    out = {f"cp_{k}": v for k, v in cp.items()}
    out["ref80_u"] = ref.sim.u.copy()
    out["ref80_v"] = ref.sim.v.copy()
    out["ref80_p"] = ref.sim.p.copy()
    out["ref80_c"] = ref.sim.scalars["c"].phi.copy()
    out["ref80_t"] = np.array(ref.sim.t)
    _save("golden_checkpoint", out)


def _images():
    """Synthetic obstacle images: grey, RGBA with transparency, RGBA fully opaque."""
    rng = np.random.default_rng(91)
    grey = np.full((50, 100), 255, dtype=np.uint8)
    grey[10:40, 20:40] = 0
    grey[5:12, 60:90] = 90
    rgba = np.zeros((37, 53, 4), dtype=np.uint8)
    rgba[..., :3] = rng.integers(0, 256, (37, 53, 3))
    rgba[8:30, 10:45, 3] = 255
    opaque = rng.integers(0, 256, (64, 48, 4)).astype(np.uint8)
    opaque[..., 3] = 255
    return {"grey": grey, "rgba": rgba, "opaque": opaque}


def gen_shapes():
    """NACA outlines and image obstacles from the reference (matplotlib is not
    needed by either; polygon masks themselves need it and are not here)."""
    import tempfile

    from PIL import Image

    out = {}
    for k, (code, chord, n, closed) in enumerate((("0012", 1.0, 200, True), ("2412", 0.6, 200, True),
                                                   ("4415", 1.3, 57, False), ("6409", 0.25, 200, True))):
        out[f"naca{k}_spec"] = np.array([code, str(chord), str(n), str(int(closed))])
        out[f"naca{k}_pts"] = geometry.naca4_coordinates(code, chord, n, closed)
    imgs = _images()
    cases_ = (("grey", (100, 50, 2.0, 1.0), {}),
              ("grey", (80, 40, 2.0, 1.0), {"x0": 0.3, "y0": 0.1, "width": 1.1, "threshold": 0.4}),
              ("grey", (61, 33, 1.0, 0.5), {"invert": True}),
              ("rgba", (90, 70, 1.5, 1.0), {"x0": 0.2, "y0": 0.15, "width": 1.0, "height": 0.7}),
              ("opaque", (64, 96, 1.0, 1.5), {"threshold": 0.6}))
    with tempfile.TemporaryDirectory() as td:
        for k, (name, (nx, ny, lx, ly), kw) in enumerate(cases_):
            path = Path(td) / f"{name}.png"
            Image.fromarray(imgs[name]).save(path)
            g = Grid(nx, ny, lx, ly)
            out[f"img{k}_name"] = np.array(name)
            out[f"img{k}_grid"] = np.array([nx, ny, lx, ly])
            out[f"img{k}_kw"] = np.array([f"{a}={b}" for a, b in kw.items()])
            out[f"img{k}_mask"] = geometry.from_image(g, path, **kw)
    out["n_naca"], out["n_img"] = np.array(4), np.array(len(cases_))
    for name, arr in imgs.items():
        out[f"pixels_{name}"] = arr
    _save("golden_shapes", out)


def _obstacle_spec(seed):
    """Obstacles and Re of the seeded obstacle flow (the package's generator, pure NumPy)."""
    sys.path.insert(0, str(HERE.parent.parent / "cfd-_b200"))
    from cfd2d_b200.cases import random_obstacle_spec

    return random_obstacle_spec(np.random.default_rng(seed))


def _digest(prefix, name, a, out, stride=8):
    """Size-bounded record of a large field: every stride-th entry in both directions,
    the sums of every row and every column, and the max-norm."""
    out[f"{prefix}_{name}_sub"] = np.ascontiguousarray(a[::stride, ::stride])
    out[f"{prefix}_{name}_rows"] = a.sum(axis=1)
    out[f"{prefix}_{name}_cols"] = a.sum(axis=0)
    out[f"{prefix}_{name}_max"] = np.array(np.abs(a).max())


def gen_obstacles():
    """The obstacle-flow benchmark case (seed 13, 1024 x 512, 2-12 obstacles, block
    inflow, outflow p = 0, slip walls; scipy CG at 1e-8) run for 3 steps from rest;
    fields stored as digests (_digest) at steps 1 and 3, the packed fluid flags
    in full."""
    out = {}
    obst, re = _obstacle_spec(13)
    out["obs1024_spec"] = np.array(repr((obst, re)))
    case = cases.custom_obstacles(obst, lx=2.0, ly=1.0, nx=1024, ny=512, re=re, inflow_profile="uniform",
                                  walls="slip", pressure_solver="cg")
    sim = case.sim
    sim.pressure.tol = TOL
    out["obs1024_fluid_bits"] = np.packbits(sim.grid.fluid.astype(np.uint8), axis=None)
    its, dts = [], []
    t0 = time.time()
    for n in range(1, 4):
        sim.step()
        its.append(sim.pressure.last_iterations)
        dts.append(sim.dt)
        if n in (1, 3):
            for name in ("u", "v", "p"):
                _digest(f"obs1024_{n}", name, getattr(sim, name), out)
        print(f"obs1024 step {n}: {time.time() - t0:.0f}s, CG it {its[-1]}", flush=True)
    out["obs1024_its"] = np.array(its)
    out["obs1024_dt"] = np.array(dts)
    out["obs1024_hist_fx"] = np.array(sim.history.fx)
    out["obs1024_hist_fy"] = np.array(sim.history.fy)
    _save("golden_obstacles1024", out)


def gen_cylinder_long():
    """The cylinder channel with the van Leer scalar (the side workload of the
    benchmark) over 2000 steps from rest with the reference's direct (SuperLU)
    pressure solver: field digests (_digest, every 2nd value) at steps 1000 and 2000,
    the force history and the drag/lift coefficients by the reference's
    validation.force_coefficients (U = 1, L = D = 0.1)."""
    from cfd2d import validation

    out = {}
    case = cases.build_case({"fall": "cylinder", "parameter": {"re": 100, "nx": 440, "ny": 82},
                             "numerik": {"pressure_solver": "direct"},
                             "skalar": {"name": "c", "diffusivity": 1e-3, "inflow_band": [0.15, 0.25],
                                        "limiter": "vanleer"}})
    sim = case.sim
    t0 = time.time()
    for n in range(1, 2001):
        sim.step()
        if n in (1000, 2000):
            for name, a in (("u", sim.u), ("v", sim.v), ("p", sim.p), ("c", sim.scalars["c"].phi)):
                _digest(f"cyl2k_{n}", name, a, out, stride=2)
            print(f"cyl2k step {n}: {time.time() - t0:.0f}s", flush=True)
    out["cyl2k_t"] = np.array(sim.history.t)
    out["cyl2k_fx"] = np.array(sim.history.fx)
    out["cyl2k_fy"] = np.array(sim.history.fy)
    cd, cl = validation.force_coefficients(sim.history.fx, sim.history.fy, U=1.0, L=0.1)
    out["cyl2k_cd"], out["cyl2k_cl"] = np.asarray(cd), np.asarray(cl)
    _save("golden_cylinder2000", out)


GROUPS = {"kernels": gen_kernels, "geometry": gen_geometry, "pressure": gen_pressure,
          "cavity": gen_cavity, "cylinder": gen_cylinder, "sst": gen_sst, "misc": gen_misc,
          "checkpoint": gen_checkpoint, "smagorinsky": gen_smagorinsky, "functions": gen_functions,
          "vof": gen_vof, "validation": gen_validation, "shapes": gen_shapes,
          "obstacles": gen_obstacles, "cylinder_long": gen_cylinder_long}

if __name__ == "__main__":
    import warnings

    warnings.simplefilter("ignore")
    for name in (sys.argv[1:] or list(GROUPS)):
        GROUPS[name]()

"""Incompressible 2-D projection solver on the GPU (drop-in for cfd2d/solver.py).

``Simulation`` keeps the reference's constructor, attributes and methods. All
fields live in device memory; ``step()`` replays one captured CUDA graph of the
whole projection step (boundary conditions, model hooks, time step, momentum,
predictor, pressure Poisson solve, correction, flow-rate control, scalar
transport, residual and history record) and then reads back a few scalars.
``run()`` replays multi-step graphs between the points where the host has to
look (print, callback, stop conditions), so the device runs ahead.

Host views: ``sim.u``, ``sim.v``, ``sim.p`` ... return numpy arrays that are
refreshed after every step once they have been requested; if the caller writes
into such an array, the change is uploaded before the next device operation.
"""

from __future__ import annotations

import ctypes as C
import math
import time
import warnings
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .boundary import BoundaryCondition, DomainBoundary
from .grid import Grid
from .pressure import PressureSolver

HIST_CAP = 4096


def _ring_rows(ring, first: int, n: int) -> np.ndarray:
    """Rows first..n-1 (step numbers, n - first <= capacity) of a device ring buffer,
    copied to the host as at most two contiguous slices."""
    cap = ring.shape[0]
    a, b = first % cap, n % cap
    if n - first == cap and a == b:
        parts = [ring[a:], ring[:a]]
    elif a < b:
        parts = [ring[a:b]]
    else:
        parts = [ring[a:], ring[:b]]
    return np.concatenate([t.cpu().numpy() for t in parts if t.shape[0] > 0], axis=0)
GRAPH_SIZES = (64, 8, 1)


class StopSimulation(Exception):
    """Raised to end a running simulation cleanly (cfd2d/solver.py:33)."""


@dataclass
class History:
    """Time series of monitor values (cfd2d/solver.py:37-55)."""

    step: list = field(default_factory=list)
    t: list = field(default_factory=list)
    dt: list = field(default_factory=list)
    residual: list = field(default_factory=list)
    divergence: list = field(default_factory=list)
    kinetic_energy: list = field(default_factory=list)
    fx: list = field(default_factory=list)
    fy: list = field(default_factory=list)
    extra: dict = field(default_factory=dict)

    def as_arrays(self) -> dict:
        out = {k: np.asarray(getattr(self, k)) for k in
               ("step", "t", "dt", "residual", "divergence", "kinetic_energy", "fx", "fy")}
        for k, v in self.extra.items():
            out[k] = np.asarray(v)
        return out


class _Mirror:
    __slots__ = ("t", "host", "snap")

    def __init__(self, tensor):
        self.t = tensor
        self.host = None
        self.snap = None


class Simulation:
    """2-D incompressible flow on a MAC grid, Chorin projection (cfd2d/solver.py:56-173)."""

    def __init__(self, grid: Grid, bcs: dict, nu: float, scheme: str = "ab2", gamma="auto",
                 tau: float = 0.5, dt: float | None = None, pressure_solver: str = "direct",
                 compute_forces: bool = False, initial_velocity: tuple = (0.0, 0.0),
                 models: list | None = None, body_force: tuple = (0.0, 0.0),
                 flow_rate: float | None = None):
        if nu <= 0:
            raise ValueError("Die Viskosität muss positiv sein.")
        if scheme not in ("ab2", "euler"):
            raise ValueError("scheme muss 'ab2' oder 'euler' sein.")
        if not (0 < tau <= 1):
            raise ValueError("tau muss in (0, 1] liegen.")
        if gamma != "auto" and not (0.0 <= float(gamma) <= 1.0):
            raise ValueError("gamma muss in [0, 1] liegen oder 'auto' sein.")
        t = _lib.torch()
        self._t = t
        self._stream = t.cuda.Stream()
        self.removed_cells = grid.finalize()
        self.grid = grid
        self.nu = float(nu)
        self.scheme = scheme
        self.gamma_setting = gamma
        self.tau = float(tau)
        self.compute_forces = compute_forces
        self.bcs = bcs
        self.body_force = (float(body_force[0]), float(body_force[1]))
        self.flow_rate = flow_rate
        self.variable_viscosity = False
        self.variable_density = False
        self.scalars: dict = {}
        self.function_objects: list = []
        self.models: list = []
        self._slots: list = []
        self._thermal = None
        self._sst = None
        self._smag = None
        self._vof = None
        self._graphs: dict = {}
        self._learned = None
        self._mirrors: dict = {}
        self._hist_seen = 0
        self.history = History()
        self.wall_time = 0.0
        nx, ny = grid.nx, grid.ny
        with self._on_stream():
            self.boundary = DomainBoundary(grid, bcs)
            self.periodic = self.boundary.periodic
            self.pressure = PressureSolver(grid, self.boundary, method=pressure_solver)
            self.pressure.on_change = self._invalidate
            dev = _lib.device()
            z = lambda *shape: t.zeros(shape, dtype=t.float64, device=dev)  # noqa: E731
            self._u, self._v, self._p = z(nx + 1, ny + 2), z(nx + 2, ny + 1), z(nx + 2, ny + 2)
            self._F, self._G = z(nx + 1, ny + 2), z(nx + 2, ny + 1)
            self._hu, self._hv = z(nx + 1, ny + 2), z(nx + 2, ny + 1)
            self._u_prev, self._v_prev = z(nx + 1, ny + 2), z(nx + 2, ny + 1)
            self._nu_t = z(nx + 2, ny + 2)
            self._nu_eff = t.full((nx + 2, ny + 2), self.nu, dtype=t.float64, device=dev)
            self._p_tmp = z(nx + 2, ny + 2)
            self._rho = t.ones((nx + 2, ny + 2), dtype=t.float64, device=dev)
            self.u_fluid = grid.u_fluid_faces()
            self.v_fluid = grid.v_fluid_faces()
            if self.periodic:
                self.u_fluid[0, :] = False
            self._fluid = _lib.to_dev(grid.fluid.astype(np.uint8))
            self._u_fluid_dev = _lib.to_dev(self.u_fluid)
            self._v_fluid_dev = _lib.to_dev(self.v_fluid)
            self._red = z(int(_lib.lib().cfd2d_sim_scratch_doubles(nx, ny)))
            self._hist = z(HIST_CAP * _lib.HIST_FIELDS)
            self._mon_ring = z(HIST_CAP * _lib.MAX_MONITORS)
            self._mon_part = z(_lib.MONITOR_SCRATCH)
            self._mon_keys: list = []
            st = _lib.State()
            st.t_end = math.inf
            st.max_steps = -1
            st.active = 1
            st.numin_bits = int(np.array(np.inf).view(np.uint64))
            st.dt_fixed = float(dt) if dt else 0.0
            self._st = st
            self._d_state = t.zeros(C.sizeof(_lib.State), dtype=t.uint8, device=dev)
            self._push()
            self._S = _lib.Sim()
            self._build_struct()
            for m in models or []:
                self.add_model(m)
            u0, v0 = initial_velocity
            if u0:
                self._u[self._u_fluid_dev.bool()] = float(u0)
            if v0:
                self._v[self._v_fluid_dev.bool()] = float(v0)
            self.gamma = 0.0 if gamma == "auto" else float(gamma)
            self._apply_bc()
            self._project_initial()

    # ================================================================ plumbing
    def _on_stream(self):
        return self._t.cuda.stream(self._stream)

    def _sync(self):
        self._stream.synchronize()

    def _push(self):
        buf = bytes(self._st)
        self._d_state.copy_(self._t.frombuffer(bytearray(buf), dtype=self._t.uint8), non_blocking=False)
        self._st_fresh = True

    def _pull(self):
        self._st = _lib.State.from_buffer_copy(bytes(self._d_state.cpu().numpy()))
        self._st_fresh = True
        return self._st

    def _invalidate(self):
        for g in self._graphs.values():
            _lib.lib().cfd2d_graph_destroy(C.c_void_p(g))
        self._graphs = {}
        if hasattr(self, "_S"):
            self._build_struct()

    def __del__(self):
        try:
            for g in self._graphs.values():
                _lib.lib().cfd2d_graph_destroy(C.c_void_p(g))
        except Exception:
            pass

    def _build_struct(self):
        g = self.grid
        S = self._S
        S.nx, S.ny, S.dx, S.dy = g.nx, g.ny, g.dx, g.dy
        S.periodic = int(self.periodic)
        S.scheme_ab2 = int(self.scheme == "ab2")
        S.gamma_auto = int(self.gamma_setting == "auto")
        S.gamma_fixed = 0.0 if self.gamma_setting == "auto" else float(self.gamma_setting)
        S.tau, S.nu = self.tau, self.nu
        S.body_fx, S.body_fy = self.body_force
        S.has_flow_rate = int(self.flow_rate is not None)
        S.flow_rate = float(self.flow_rate or 0.0)
        S.flow_count = float(self.u_fluid[1:g.nx + 1, 1:-1].sum())
        S.variable_viscosity = int(self.variable_viscosity)
        S.compute_forces = int(bool(self.compute_forces))
        S.has_solid = int(bool(g.solid.any()))
        self.boundary.fill_struct(S)
        S.fluid = self._fluid.data_ptr()
        for name in ("u", "v", "p", "F", "G", "hu", "hv", "u_prev", "v_prev", "nu_eff", "nu_t"):
            setattr(S, name, getattr(self, "_" + name).data_ptr())
        S.pcg = self.pressure.op
        S.cg_rtol = self.pressure.rtol
        S.cg_maxiter = self.pressure.maxiter
        S.nscalars = len(self._slots)
        for k, f in enumerate(self._slots):
            f.fill_struct(S.scalars[k])
            S.scalar_dtlim_const[k] = f.dt_limit_const()
        S.thermal_index = -1
        S.gx = S.gy = S.T_ref = 0.0
        if self._thermal is not None:
            S.thermal_index, (S.gx, S.gy), S.T_ref = self._thermal
        S.sst_on = int(self._sst is not None)
        if self._sst is not None:
            self._sst.fill_struct(S.sst)
        S.smag_on = int(self._smag is not None)
        S.smag.l2 = self._smag.l2_ptr() if self._smag is not None else None
        S.vof_on = int(self._vof is not None)
        if self._vof is not None:
            self._vof.fill_struct(S.vof)
        # model monitors recorded after every step (cfd2d/solver.py:441-443), in model order
        mons = []
        for m in self.models:
            dm = m.device_monitors(self) if hasattr(m, "device_monitors") else None
            mons += list(dm or [])
        if len(mons) > _lib.MAX_MONITORS:
            raise ValueError(f"höchstens {_lib.MAX_MONITORS} Monitore auf dem Gerät")
        self._mon_keys = [key for key, _ in mons]
        S.nmon = len(mons)
        for k, (_, mon) in enumerate(mons):
            S.mon[k] = mon
        S.mon_ring = self._mon_ring.data_ptr()
        S.mon_part = self._mon_part.data_ptr()
        S.state = self._d_state.data_ptr()
        S.red = self._red.data_ptr()
        S.hist = self._hist.data_ptr()
        S.hist_cap = HIST_CAP
        S.p_tmp = self._p_tmp.data_ptr()

    def _call(self, fn, *args):
        self._st_fresh = False
        rc = getattr(_lib.lib(), fn)(C.byref(self._S), *args, _lib.stream_ptr(self._stream))
        _lib.check(rc, fn)

    # hooks used by the models while they attach
    def _register_scalar(self, f) -> int:
        if len(self._slots) >= _lib.MAX_SCALARS:
            raise ValueError(f"höchstens {_lib.MAX_SCALARS} Skalarfelder auf dem Gerät")
        self._slots.append(f)
        self._invalidate()
        return len(self._slots) - 1

    def _set_thermal(self, slot, gravity, T_ref):
        self._thermal = (slot, gravity, T_ref)
        self._invalidate()

    def _set_sst(self, sst):
        self._sst = sst
        self._invalidate()

    def _set_smagorinsky(self, model):
        self._smag = model
        self._invalidate()

    def _set_vof(self, model):
        self._vof = model
        self._invalidate()

    def _vof_properties(self):
        with self._on_stream():
            self._flush_mirrors()
            self._call("cfd2d_sim_vof_properties")
            self._device_changed()

    def _smagorinsky_pre_momentum(self):
        with self._on_stream():
            self._flush_mirrors()
            self._call("cfd2d_sim_smagorinsky_pre_momentum")
            self._device_changed()

    def _scalar_fill_ghosts(self, slot):
        with self._on_stream():
            self._flush_mirrors()
            self._call("cfd2d_sim_scalar_fill_ghosts", int(slot))
            self._device_changed()

    def _sst_pre_momentum(self):
        with self._on_stream():
            self._flush_mirrors()
            self._call("cfd2d_sim_sst_pre_momentum")
            self._device_changed()

    # ---------------------------------------------------------------- host views
    def _mirror(self, name, tensor) -> np.ndarray:
        m = self._mirrors.get(name)
        if m is None:
            m = _Mirror(tensor)
            self._mirrors[name] = m
        if m.host is None:
            self._sync()
            m.host = tensor.cpu().numpy().copy()
            m.snap = m.host.copy()
        return m.host

    def _flush_mirrors(self):
        """Upload host views the caller has written into."""
        for m in self._mirrors.values():
            if m.host is not None and not np.array_equal(m.host, m.snap, equal_nan=True):
                m.t.copy_(self._t.from_numpy(np.ascontiguousarray(m.host)).to(m.t.device))
                m.snap[...] = m.host

    def _device_changed(self):
        """Refresh the host views that have been handed out."""
        live = [m for m in self._mirrors.values() if m.host is not None]
        if not live:
            return
        self._sync()
        for m in live:
            m.host[...] = m.t.cpu().numpy()
            m.snap[...] = m.host

    def _field(name):  # noqa: N805
        def get(self):
            return self._mirror(name, getattr(self, "_" + name))

        def set_(self, value):
            arr = np.asarray(value, dtype=np.float64)
            tensor = getattr(self, "_" + name)
            with self._on_stream():
                tensor.copy_(_lib.to_dev(arr))
            m = self._mirrors.get(name)
            if m is not None and m.host is not None:
                m.host[...] = arr
                m.snap[...] = arr

        return property(get, set_)

    u = _field("u")
    v = _field("v")
    p = _field("p")
    F = _field("F")
    G = _field("G")
    hu = _field("hu")
    hv = _field("hv")
    nu_t = _field("nu_t")
    nu_eff = _field("nu_eff")
    rho = _field("rho")

    @property
    def hu_old(self):
        return self.hu if (self.scheme == "ab2" and self._st.have_old) else None

    @property
    def hv_old(self):
        return self.hv if (self.scheme == "ab2" and self._st.have_old) else None

    @property
    def u_gpu(self):
        return self._u

    @property
    def v_gpu(self):
        return self._v

    @property
    def p_gpu(self):
        return self._p

    # scalar state (host copy of the device state, refreshed at every sync)
    def _state_prop(name, doc):  # noqa: N805
        def get(self):
            return float(getattr(self._st, name))

        def set_(self, value):
            with self._on_stream():
                self._sync()
                self._pull()
                setattr(self._st, name, float(value))
                self._push()

        return property(get, set_, doc=doc)

    t = _state_prop("t", "simulated time")
    dt = _state_prop("dt", "last time step")
    residual = _state_prop("residual", "max|du|/dt of the last step")
    flow_force = _state_prop("flow_force", "driving force of the flow-rate control")

    @property
    def n(self) -> int:
        return int(self._st.n)

    @n.setter
    def n(self, value: int) -> None:
        with self._on_stream():
            self._sync()
            self._pull()
            self._st.n = int(value)
            self._push()

    @property
    def dt_old(self):
        return float(self._st.dt_old) if self._st.n > 0 else None

    @property
    def dt_fixed(self):
        v = float(self._st.dt_fixed)
        return v if v != 0.0 else None

    @dt_fixed.setter
    def dt_fixed(self, value) -> None:
        with self._on_stream():
            self._sync()
            self._pull()
            self._st.dt_fixed = float(value) if value else 0.0
            self._push()

    @property
    def gamma(self) -> float:
        return float(self._st.gamma)

    @gamma.setter
    def gamma(self, value) -> None:
        with self._on_stream():
            self._sync()
            self._pull()
            self._st.gamma = float(value)
            self._push()

    # ================================================================ model hooks
    def add_model(self, model) -> None:
        """Attach a built-in model (cfd2d/solver.py:178-181)."""
        with self._on_stream():
            model.attach(self)
        self.models.append(model)
        self._invalidate()

    def model(self, kind: str):
        for m in self.models:
            if getattr(m, "kind", None) == kind:
                return m
        return None

    # ================================================================ step
    def _apply_bc(self) -> None:
        with self._on_stream():
            self._flush_mirrors()
            self._call("cfd2d_sim_apply_bc")
            self._device_changed()

    def _project_initial(self) -> None:
        """Make the initial field divergence-free (cfd2d/solver.py:195-204)."""
        with self._on_stream():
            self._flush_mirrors()
            if not (bool((self._u != 0).any()) or bool((self._v != 0).any())):
                return
            self._call("cfd2d_sim_project_initial")
            self._sync()
            if self._pull().status & _lib.S_BARRIER_TIMEOUT:
                raise RuntimeError("initial projection abandoned: a bounded inter-block wait timed out")
            self._device_changed()

    def _graph(self, nsteps: int):
        g = self._graphs.get(nsteps)
        if g is None:
            h = C.c_void_p(0)
            rc = _lib.lib().cfd2d_graph_capture_steps(C.byref(self._S), int(nsteps),
                                                      _lib.stream_ptr(self._stream), C.byref(h))
            _lib.check(rc, "cfd2d_graph_capture_steps")
            g = h.value
            self._graphs[nsteps] = g
        return g

    def _launch_steps(self, nsteps: int) -> None:
        self._st_fresh = False
        if self.function_objects:
            self._steps_with_functions(int(nsteps))
            return
        if self._learned is not None:
            for _ in range(int(nsteps)):
                self._learned_step()
            return
        left = int(nsteps)
        for size in GRAPH_SIZES:
            while left >= size:
                rc = _lib.lib().cfd2d_graph_launch(C.c_void_p(self._graph(size)),
                                                   _lib.stream_ptr(self._stream))
                _lib.check(rc, "cfd2d_graph_launch")
                left -= size

    def stage_times(self, nsteps: int = 10) -> dict:
        """Device time of the three parts of a step, in ms averaged over ``nsteps``
        steps that advance the simulation: before the pressure solve (boundary
        conditions, model hooks, dt, tendencies, predictor), the solve, and after it
        (correction, boundary conditions, flow-rate control, model post-steps,
        history and monitors). CUDA events recorded inside one captured step graph.
        The reference only accumulates wall time (cfd2d/solver.py:328, 393)."""
        if self.function_objects or self._learned is not None:
            raise ValueError("stage_times runs the plain step graph: detach function objects and the "
                             "learned preconditioner first")
        L = _lib.lib()
        ev = (C.c_void_p * 4)()
        _lib.check(L.cfd2d_events_create(4, ev), "cfd2d_events_create")
        graph, knodes = C.c_void_p(0), C.c_int(0)
        tot = [0.0, 0.0, 0.0]
        try:
            with self._on_stream():
                self._flush_mirrors()
                self._set_run_limits()
                s = _lib.stream_ptr(self._stream)
                _lib.check(L.cfd2d_graph_capture_steps_ex(C.byref(self._S), 1, s, ev, C.byref(graph),
                                                          C.byref(knodes)), "cfd2d_graph_capture_steps_ex")
                for _ in range(int(nsteps)):
                    self._st_fresh = False
                    _lib.check(L.cfd2d_graph_launch(graph, s), "cfd2d_graph_launch")
                    for k in range(3):
                        ms = C.c_float()
                        _lib.check(L.cfd2d_event_elapsed_ms(ev[k], ev[k + 1], C.byref(ms)), "elapsed")
                        tot[k] += ms.value
                self._sync()
                self._after_steps()
        finally:
            if graph.value:
                L.cfd2d_graph_destroy(graph)
            L.cfd2d_events_destroy(4, ev)
        n = max(int(nsteps), 1)
        return {"pre_solve_ms": tot[0] / n, "solve_ms": tot[1] / n, "post_solve_ms": tot[2] / n,
                "kernels_per_step": int(knodes.value)}

    def _steps_with_functions(self, nsteps: int) -> None:
        """Steps one at a time with the function objects after each (cfd2d/solver.py:401-403).
        Device function objects only queue kernels behind the step; host ones (and
        user-defined ones) run after a synchronisation, with the state read back,
        and only when the step ran."""
        fos = list(self.function_objects)
        host = [fo for fo in fos if not getattr(fo, "device", False)]
        saved, self.function_objects = self.function_objects, []
        try:
            for _ in range(nsteps):
                n0 = int(self._st.n)
                self._launch_steps(1)
                for fo in fos:
                    if getattr(fo, "device", False):
                        fo.execute(self)
                if host:
                    self._sync()
                    self._after_steps()
                    if int(self._st.n) == n0:
                        break
                    for fo in host:
                        fo.execute(self)
                    self._flush_mirrors()
        finally:
            self.function_objects = saved

    # ================================================================ learned pressure preconditioner
    def set_pressure_preconditioner(self, net=None, **kw) -> None:
        """Solve each step's pressure system by flexible CG with the learned
        preconditioner ``net`` (cfd2d_b200.learned; keyword arguments go to
        LearnedPCG), or with the plain Jacobi-PCG again when net is None. Needs an
        outflow (Dirichlet) boundary. No counterpart in the reference."""
        if self._learned is not None:
            self._learned.close()
            self._learned = None
        if net is not None:
            from .learned import LearnedPCG

            with self._on_stream():
                lp = LearnedPCG(self.pressure, net, **kw)
            lp.iters_out = self._d_state.data_ptr() + _lib.State.cg_iters_step.offset
            self._learned = lp

    def _learned_step(self) -> None:
        """step_begin, flexible CG on div(F, G)/dt inside one graph, the Jacobi-PCG
        fallback if it stalled, p scattered into the padded field, step_finish."""
        lp = self._learned
        L = _lib.lib()
        s = _lib.stream_ptr(self._stream)
        self._call("cfd2d_sim_step_begin")
        dt_ptr = C.c_void_p(self._d_state.data_ptr() + _lib.State.dt.offset)
        lp.solve_into_x(F=self._F, G=self._G, dx=self.grid.dx, dy=self.grid.dy, dt_ptr=dt_ptr, key="sim")
        if lp.last_reason in (_lib.FCG_STALLED, _lib.FCG_MAXITER):
            # the plain solver continues from the flexible CG's iterate
            self.pressure.solve((-lp.b).view(self.grid.nx, self.grid.ny))
        _lib.check(L.cfd2d_fcg_scatter_p(C.byref(self.pressure.op), _lib.ptr(self.pressure._d_x0),
                                         _lib.ptr(self._p), s), "fcg_scatter_p")
        self._call("cfd2d_sim_step_finish")

    def _set_run_limits(self, t_end=math.inf, max_steps=-1, steady_tol=0.0):
        # the host copy of the state is current unless device work ran since it was read
        st = self._st if getattr(self, "_st_fresh", False) else self._pull()
        changed = (st.t_end != t_end or st.max_steps != max_steps or st.steady_tol != steady_tol
                   or st.stop_reason != 0 or (st.status & _lib.S_NONFINITE))
        if changed:
            st.t_end, st.max_steps, st.steady_tol = t_end, max_steps, steady_tol
            st.stop_reason = 0
            st.status &= ~_lib.S_NONFINITE
            self._push()

    def _after_steps(self):
        """Read the state and new history records; report errors."""
        st = self._pull()
        self._pull_history()
        self._device_changed()
        if st.status & _lib.S_CG_MAXITER:
            warnings.warn(f"CG-Drucklöser nicht konvergiert ({self.pressure.maxiter} Iterationen)")
            st.status &= ~_lib.S_CG_MAXITER
            self._push()
        if st.status & _lib.S_BARRIER_TIMEOUT:
            raise RuntimeError("a bounded device wait timed out; the step was abandoned")
        if st.status & _lib.S_VOF_SUBSTEPS:
            st.status &= ~_lib.S_VOF_SUBSTEPS
            self._push()
            raise RuntimeError("der VOF-Transport brauchte mehr Unterschritte als vorgesehen "
                               "(VOF(nsub_max=...) erhöhen oder tau verkleinern)")
        if st.status & _lib.S_NONFINITE:
            n = st.error_step or st.n
            st.status &= ~_lib.S_NONFINITE
            st.error_step = 0
            self._push()
            raise FloatingPointError(
                f"Simulation instabil in Schritt {n} (t = {st.t:.4g}). "
                "Zeitschritt verkleinern (tau), Gitter verfeinern oder gamma erhöhen.")

    def step(self) -> None:
        """One projection time step (cfd2d/solver.py:326-403)."""
        t0 = time.perf_counter()
        with self._on_stream():
            self._flush_mirrors()
            self._set_run_limits()
            self._launch_steps(1)
            self._sync()
            self.wall_time += time.perf_counter() - t0
            self._after_steps()

    def launch_steps(self, nsteps: int) -> None:
        """Queue nsteps projection steps on this simulation's stream and return at
        once; finish_steps() waits for them and reads the results. Lets several
        simulations run side by side (cfd2d_b200.batch)."""
        with self._on_stream():
            self._flush_mirrors()
            self._set_run_limits()
            self._t_launch = time.perf_counter()
            self._launch_steps(nsteps)

    def finish_steps(self) -> None:
        """Wait for the steps queued by launch_steps() and report their results."""
        with self._on_stream():
            self._sync()
            self.wall_time += time.perf_counter() - getattr(self, "_t_launch", time.perf_counter())
            self._after_steps()

    @property
    def stream(self):
        """The CUDA stream (torch.cuda.Stream) this simulation's work runs on."""
        return self._stream

    def advance(self, nsteps: int) -> None:
        """nsteps projection steps with a single host synchronisation at the end."""
        t0 = time.perf_counter()
        with self._on_stream():
            self._flush_mirrors()
            self._set_run_limits()
            self._launch_steps(nsteps)
            self._sync()
            self.wall_time += time.perf_counter() - t0
            self._after_steps()

    def _pull_history(self):
        n = int(self._st.n)
        first = max(self._hist_seen, n - HIST_CAP)
        if n <= first:
            self._hist_seen = n
            return
        recs = _ring_rows(self._hist.view(HIST_CAP, _lib.HIST_FIELDS), first, n)
        nm = len(self._mon_keys)
        mrecs = (_ring_rows(self._mon_ring.view(HIST_CAP, _lib.MAX_MONITORS), first, n)[:, :nm] if nm
                 else np.zeros((n - first, 0)))
        h = self.history
        for k, r, rm in zip(range(first + 1, n + 1), recs, mrecs):
            h.step.append(k)
            h.t.append(float(r[0]))
            h.dt.append(float(r[1]))
            h.residual.append(float(r[2]))
            h.divergence.append(float(r[3]))
            h.kinetic_energy.append(float(r[4]))
            if self.compute_forces:
                h.fx.append(float(r[5]))
                h.fy.append(float(r[6]))
            if self.flow_rate is not None:
                h.extra.setdefault("antriebskraft", []).append(float(r[7]))
            for key, val in zip(self._mon_keys, rm):
                h.extra.setdefault(key, []).append(float(val))
            h.extra.setdefault("cg_iterationen", []).append(int(r[8]))
        self._hist_seen = n

    def run(self, t_end: float, max_steps: int | None = None, steady_tol: float | None = None,
            callback=None, callback_every: int = 50, verbose: bool = True,
            print_every: int = 200) -> str:
        """Run to t_end or convergence (cfd2d/solver.py:448-505).

        The device evaluates the stop conditions before every step; the host
        synchronises only at print and callback steps and every 256 steps.
        """
        reason = "t_end"
        t_start = time.perf_counter()
        t_ms = max_steps if max_steps is not None else -1
        try:
            with self._on_stream():
                self._flush_mirrors()
                self._set_run_limits(float(t_end), int(t_ms), float(steady_tol or 0.0))
                while self._st.t < t_end - 1e-12:
                    if max_steps is not None and self._st.n >= max_steps:
                        reason = "max_steps"
                        break
                    n0 = int(self._st.n)
                    chunk = 256
                    if verbose:
                        chunk = min(chunk, print_every - n0 % print_every)
                    if callback is not None:
                        chunk = min(chunk, callback_every - n0 % callback_every)
                    if max_steps is not None:
                        chunk = min(chunk, max_steps - n0)
                    t0 = time.perf_counter()
                    self._launch_steps(max(chunk, 1))
                    self._sync()
                    self.wall_time += time.perf_counter() - t0
                    prev = n0
                    self._after_steps()
                    n = int(self._st.n)
                    if verbose:
                        for k in range(prev + 1, n + 1):
                            if k % print_every == 0:
                                print(self._status_line_at(k))
                    if callback is not None and n > prev and n % callback_every == 0:
                        if callback(self) is False:
                            reason = "abgebrochen"
                            break
                        self._flush_mirrors()
                    if self._st.stop_reason == 3:
                        reason = "konvergiert"
                        break
                    if n == prev:
                        break
                self._set_run_limits()
        except (KeyboardInterrupt, StopSimulation):
            reason = "abgebrochen"
        if callback is not None:
            try:
                callback(self)
            except StopSimulation:
                pass
        if verbose:
            print(self.status_line())
            el = time.perf_counter() - t_start
            print(f"Ende: {reason}. {self.n} Schritte, Rechenzeit {el:.1f} s "
                  f"({1e3 * self.wall_time / max(self.n, 1):.2f} ms/Schritt)")
        return reason

    # ================================================================ diagnostics (host, on demand)
    def _status_line_at(self, k: int) -> str:
        h = self.history
        i = h.step.index(k) if k in h.step else -1
        s = (f"Schritt {k:7d} | t = {h.t[i]:9.4f} | dt = {h.dt[i]:.3e} | "
             f"Residuum = {h.residual[i]:.3e} | max|div u| = {h.divergence[i]:.2e}")
        if self.compute_forces and h.fx:
            s += f" | Fx = {h.fx[i]:+.4f} | Fy = {h.fy[i]:+.4f}"
        return s

    def status_line(self) -> str:
        s = (f"Schritt {self.n:7d} | t = {self.t:9.4f} | dt = {self.dt:.3e} | "
             f"Residuum = {self.residual:.3e} | max|div u| = {self.max_divergence():.2e}")
        if self.compute_forces and self.history.fx:
            s += f" | Fx = {self.history.fx[-1]:+.4f} | Fy = {self.history.fy[-1]:+.4f}"
        return s

    def compute_dt(self) -> float:
        """Time step for the current state (cfd2d/solver.py:209-231), on the host."""
        if self.dt_fixed:
            return float(self.dt_fixed)
        g = self.grid
        umax = max(np.abs(self.u).max(), 1e-12)
        vmax = max(np.abs(self.v).max(), 1e-12)
        if self.variable_density:
            nu_max = float((self.nu_eff / self.rho)[g.fluid].max())
        else:
            nu_max = float(self.nu_eff.max()) if self.variable_viscosity else self.nu
        dt_visc = 0.5 / (nu_max * (1.0 / g.dx ** 2 + 1.0 / g.dy ** 2))
        dt_conv = min(g.dx / umax, g.dy / vmax)
        if self.scheme == "ab2":
            dt_visc *= 0.5
            dt_conv *= 0.8
        dt = self.tau * min(dt_visc, dt_conv)
        for m in self.models:
            lim = m.dt_limit(self)
            if lim is not None:
                dt = min(dt, self.tau * lim)
        return dt

    def bulk_velocity(self) -> float:
        m = self.u_fluid[1:self.grid.nx + 1, 1:-1]
        return float(self.u[1:self.grid.nx + 1, 1:-1][m].mean())

    def divergence(self) -> np.ndarray:
        g = self.grid
        u, v = self.u, self.v
        div = (u[1:, 1:-1] - u[:-1, 1:-1]) / g.dx + (v[1:-1, 1:] - v[1:-1, :-1]) / g.dy
        return np.where(g.fluid_interior, div, 0.0)

    def max_divergence(self) -> float:
        return float(np.abs(self.divergence()).max())

    def cell_velocity(self):
        u, v = self.u, self.v
        uc = 0.5 * (u[:-1, 1:-1] + u[1:, 1:-1])
        vc = 0.5 * (v[1:-1, :-1] + v[1:-1, 1:])
        solid = self.grid.solid
        return np.where(solid, np.nan, uc), np.where(solid, np.nan, vc)

    def cell_pressure(self) -> np.ndarray:
        return np.where(self.grid.solid, np.nan, self.p[1:-1, 1:-1])

    def kinetic_energy(self) -> float:
        uc, vc = self.cell_velocity()
        return float(0.5 * np.nansum(uc ** 2 + vc ** 2) * self.grid.dx * self.grid.dy)

    def obstacle_forces(self):
        """Force of the fluid on the interior obstacles (cfd2d/solver.py:542-567)."""
        g = self.grid
        solid = g.interior_solid_padded()
        f = g.fluid[1:-1, 1:-1]
        east, west = f & solid[2:, 1:-1], f & solid[:-2, 1:-1]
        north, south = f & solid[1:-1, 2:], f & solid[1:-1, :-2]
        p = self.p[1:-1, 1:-1]
        u, v = self.u, self.v
        uc = 0.5 * (u[:-1, 1:-1] + u[1:, 1:-1])
        vc = 0.5 * (v[1:-1, :-1] + v[1:-1, 1:])
        mu = self.nu
        fx = (p[east].sum() - p[west].sum()) * g.dy
        fy = (p[north].sum() - p[south].sum()) * g.dx
        fx += mu * (uc[north].sum() + uc[south].sum()) / (0.5 * g.dy) * g.dx
        fy += mu * (vc[east].sum() + vc[west].sum()) / (0.5 * g.dx) * g.dy
        return float(fx), float(fy)

    def vorticity(self) -> np.ndarray:
        g = self.grid
        u, v = self.u, self.v
        return (v[1:, :] - v[:-1, :]) / g.dx - (u[:, 1:] - u[:, :-1]) / g.dy

    def cell_vorticity(self) -> np.ndarray:
        w = self.vorticity()
        wc = 0.25 * (w[:-1, :-1] + w[1:, :-1] + w[:-1, 1:] + w[1:, 1:])
        return np.where(self.grid.solid, np.nan, wc)

    def streamfunction(self) -> np.ndarray:
        g = self.grid
        fl = g.fluid
        u_open = fl[:-1, 1:-1] | fl[1:, 1:-1]
        v_open = fl[1:-1, 0] | fl[1:-1, 1]
        u = np.where(u_open, self.u[:, 1:-1], 0.0)
        v0 = np.where(v_open, self.v[1:-1, 0], 0.0)
        psi = np.zeros((g.nx + 1, g.ny + 1))
        psi[1:, 0] = -np.cumsum(v0) * g.dx
        psi[:, 1:] = psi[:, :1] + np.cumsum(u, axis=1) * g.dy
        return psi

    def sample_u(self, x, y) -> np.ndarray:
        """u interpolated bilinearly at arbitrary points, wall values through the ghost
        cells (cfd2d/solver.py:598-606); evaluated on the device."""
        from .functions import sample_field

        return sample_field(self, "u", x, y)

    def sample_v(self, x, y) -> np.ndarray:
        """v at arbitrary points (cfd2d/solver.py:608-615); evaluated on the device."""
        from .functions import sample_field

        return sample_field(self, "v", x, y)

    def summary(self) -> str:
        g = self.grid
        lines = [
            f"Gitter: {g.nx} x {g.ny} Zellen, Gebiet {g.lx:g} x {g.ly:g}, dx = {g.dx:.4g}, dy = {g.dy:.4g}",
            f"Fluidzellen: {g.fluid_interior.sum()} / {g.nx * g.ny}"
            + (f" ({self.removed_cells} eingeschlossene Zellen entfernt)" if self.removed_cells else ""),
            f"Viskosität nu = {self.nu:.4g}",
            f"Zeitschema: {'Adams-Bashforth 2' if self.scheme == 'ab2' else 'Euler explizit'}, "
            f"tau = {self.tau}, gamma = {self.gamma_setting}",
            f"Drucklöser: {'CG (Jacobi), rtol 1e-13' if self.pressure.method == 'direct' else 'CG (Jacobi)'}"
            " auf der GPU",
            "Randbedingungen:",
            self.boundary.describe(),
        ]
        return "\n".join(lines)

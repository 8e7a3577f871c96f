"""Function objects, VTK export and checkpoints (drop-in for cfd2d/functions.py).

The function objects read the device fields: ``Probes`` and ``FieldAverage`` queue
one small kernel after each step on the simulation's stream (they read t, dt and n
on the device, so the steps keep running without a host synchronisation);
``LineSample``, ``sample_field`` and ``write_vtk`` evaluate or pack the fields on the
device and copy only the samples or the finished VTK payload to the host. Files
have the reference's names and formats; the PNG plots the reference draws beside
them need matplotlib, which this package does not depend on, and are not written.
``VTKWriter``, ``Checkpoint`` and user-defined function objects run on the host
after every step, which synchronises each step as in the reference.

Checkpoints use the reference's schema (``np.savez_compressed``): u, v, p, t, n, dt,
flow_force, dt_old, the fluid flags, hu_old/hv_old after an AB2 step, one
``skalar_<name>`` array per scalar field, per-model state and the history as JSON,
so a checkpoint written here loads in the reference and the other way round. One key
is added: ``pressure_x0``, the warm start of the iterative pressure solve, which makes
a restart continue bit-identically (the reference ignores keys it does not read).
"""

from __future__ import annotations

import csv
import ctypes as C
import json
from pathlib import Path

import numpy as np

from . import _lib
from .visualization import available_fields, device_field, streamfunction_device


def _field_array(descs):
    arr = (_lib.Field * len(descs))()
    for k, (kind, data) in enumerate(descs):
        arr[k].kind = kind
        arr[k].data = data.data_ptr() if data is not None else None
    return arr


def sample_field(sim, field: str, x, y) -> np.ndarray:
    """Field interpolated at arbitrary points (cfd2d/functions.py:24-39): u and v on
    their staggered grids (extrapolated), cell fields bilinear between the cell
    centres with the points clipped to them. Evaluated on the device."""
    t = _lib.torch()
    x = np.atleast_1d(np.asarray(x, dtype=float)).ravel()
    y = np.atleast_1d(np.asarray(y, dtype=float)).ravel()
    if x.shape != y.shape:
        raise ValueError("x und y brauchen gleich viele Punkte")
    with sim._on_stream():
        sim._flush_mirrors()
        kind, data = device_field(sim, field, faces=True)
        fields = _field_array([(kind, data)])
        px, py = _lib.to_dev(x, t.float64), _lib.to_dev(y, t.float64)
        out = t.empty(len(x), dtype=t.float64, device=_lib.device())
        sim._call("cfd2d_sample", fields, 1, _lib.ptr(px), _lib.ptr(py), len(x), _lib.ptr(out))
        return out.cpu().numpy()


class FunctionObject:
    """Base class (cfd2d/functions.py:42-56). ``device = True`` marks objects whose
    execute() only queues work on the simulation's stream."""

    name = "function"
    device = False

    def execute(self, sim) -> None:
        pass

    def write(self, outdir: Path) -> list[Path]:
        return []

    def describe(self) -> str:
        return self.name

    def spec(self) -> dict:
        return {}


class Probes(FunctionObject):
    """Time series of fields at fixed points (cfd2d/functions.py:59-114).

    Each execute() queues one single-block kernel that samples every (field, point)
    pair and appends the row with the step's time to a device buffer; ``t`` and
    ``data`` copy the rows to the host when they are read."""

    device = True

    def __init__(self, points, fields=("u", "v", "pressure"), every: int = 1):
        self.points = [tuple(map(float, p)) for p in points]
        self.fields = list(fields)
        self.every = max(1, int(every))
        self.name = "probes"
        self._sim = None
        self._cache = None

    def _bind(self, sim) -> None:
        t = _lib.torch()
        dev = _lib.device()
        self._sim = sim
        self._px = _lib.to_dev(np.array([p[0] for p in self.points], dtype=float), t.float64)
        self._py = _lib.to_dev(np.array([p[1] for p in self.points], dtype=float), t.float64)
        g = sim.grid
        self._psi = (t.empty((g.nx + 1, g.ny + 1), dtype=t.float64, device=dev)
                     if "streamfunction" in self.fields else None)
        descs = []
        for f in self.fields:
            if f == "streamfunction":
                descs.append((_lib.FIELD_NODE, self._psi))
            else:
                descs.append(device_field(sim, f, faces=True))
        self._descs = descs
        self._farr = _field_array(descs)
        self._cap = 0
        self._t = self._vals = None
        self._count = t.tensor([0, int(sim.n), 0], dtype=t.int64, device=dev)
        self._queued = 0
        self._grow(256)

    def _grow(self, cap: int) -> None:
        t = _lib.torch()
        dev = _lib.device()
        width = len(self.fields) * len(self.points)
        new_t = t.zeros(cap, dtype=t.float64, device=dev)
        new_v = t.zeros((cap, width), dtype=t.float64, device=dev)
        if self._t is not None:
            new_t[:self._cap].copy_(self._t)
            new_v[:self._cap].copy_(self._vals)
        self._t, self._vals, self._cap = new_t, new_v, cap
        self._series = _lib.ProbeSeries(self._t.data_ptr(), self._vals.data_ptr(), self._count.data_ptr(),
                                        cap, self.every)

    def execute(self, sim) -> None:
        if not self.points or not self.fields:
            return
        with sim._on_stream():
            if self._sim is not sim:
                self._bind(sim)
            if self._queued >= self._cap:  # every queued call may add a row
                self._grow(2 * self._cap)
            if self._psi is not None:
                streamfunction_device(sim, self._psi)
            sim._call("cfd2d_probe_record", self._farr, len(self.fields), _lib.ptr(self._px),
                      _lib.ptr(self._py), len(self.points), C.byref(self._series))
            self._queued += 1
            self._cache = None

    def _rows(self):
        if self._sim is None:
            return np.zeros(0), np.zeros((0, len(self.fields), len(self.points)))
        if self._cache is None:
            sim = self._sim
            with sim._on_stream():
                sim._sync()
                cnt = self._count.cpu().numpy()
                if cnt[2]:
                    raise RuntimeError("Sonden-Zeitreihe übergelaufen")
                n = int(cnt[0])
                tt = self._t[:n].cpu().numpy()
                vals = self._vals[:n].cpu().numpy().reshape(n, len(self.fields), len(self.points))
            self._cache = (tt, vals)
        return self._cache

    @property
    def t(self) -> list:
        return [float(v) for v in self._rows()[0]]

    @property
    def data(self) -> dict:
        vals = self._rows()[1]
        return {f: [vals[r, k] for r in range(vals.shape[0])] for k, f in enumerate(self.fields)}

    def write(self, outdir: Path) -> list[Path]:
        tt, vals = self._rows()
        if len(tt) == 0:
            return []
        outdir = Path(outdir)
        path = outdir / "sonden.csv"
        with open(path, "w", newline="", encoding="utf-8") as fh:
            w = csv.writer(fh, delimiter=";")
            w.writerow(["t"] + [f"{f}@({x:g},{y:g})" for f in self.fields for (x, y) in self.points])
            for r, tv in enumerate(tt):
                w.writerow([f"{tv:.6g}"] + [f"{vals[r, k, i]:.6g}" for k in range(len(self.fields))
                                            for i in range(len(self.points))])
        return [path]

    def describe(self) -> str:
        return f"Sonden an {len(self.points)} Punkten: {', '.join(self.fields)}"

    def spec(self) -> dict:
        return {"typ": "sonden", "punkte": self.points, "felder": self.fields, "alle": self.every}


class LineSample(FunctionObject):
    """Profile along the segment p0 -> p1 at the end of the run
    (cfd2d/functions.py:117-177); sampled on the device."""

    device = True

    def __init__(self, p0, p1, n: int = 100, fields=("u", "v", "pressure"), label: str = "linie"):
        self.p0 = tuple(map(float, p0))
        self.p1 = tuple(map(float, p1))
        self.n = int(n)
        self.fields = list(fields)
        self.label = label
        self.name = "linie"
        self.result = None
        self.sim = None

    def execute(self, sim) -> None:
        self.sim = sim

    def sample(self, sim) -> dict:
        s = np.linspace(0, 1, self.n)
        x = self.p0[0] + s * (self.p1[0] - self.p0[0])
        y = self.p0[1] + s * (self.p1[1] - self.p0[1])
        dist = s * np.hypot(self.p1[0] - self.p0[0], self.p1[1] - self.p0[1])
        out = {"s": dist, "x": x, "y": y}
        for f in self.fields:
            out[f] = sample_field(sim, f, x, y)
        return out

    def write(self, outdir: Path) -> list[Path]:
        if self.sim is None:
            return []
        outdir = Path(outdir)
        d = self.sample(self.sim)
        self.result = d
        path = outdir / f"linie_{self.label}.csv"
        keys = ["s", "x", "y"] + self.fields
        with open(path, "w", newline="", encoding="utf-8") as fh:
            w = csv.writer(fh, delimiter=";")
            w.writerow(keys)
            for k in range(self.n):
                w.writerow([f"{d[c][k]:.6g}" for c in keys])
        return [path]

    def describe(self) -> str:
        return f"Linienprobe {self.p0} → {self.p1} ({self.n} Punkte): {', '.join(self.fields)}"

    def spec(self) -> dict:
        return {"typ": "linie", "p0": self.p0, "p1": self.p1, "n": self.n, "felder": self.fields,
                "name": self.label}


class FieldAverage(FunctionObject):
    """Time means and RMS of u, v, p from t_start on (cfd2d/functions.py:180-241).
    The sums live on the device; mean() and rms() copy them when called."""

    device = True
    KEYS = ("u", "v", "p")

    def __init__(self, t_start: float = 0.0):
        self.t_start = float(t_start)
        self.name = "mittelwerte"
        self.sim = None
        self._avg = None

    def _bind(self, sim) -> None:
        t = _lib.torch()
        dev = _lib.device()
        g = sim.grid
        self.sim = sim
        self._sum = t.zeros((3, g.nx, g.ny), dtype=t.float64, device=dev)
        self._sum2 = t.zeros((3, g.nx, g.ny), dtype=t.float64, device=dev)
        self._n0 = float(sim.n)
        self._T = t.tensor([0.0, self._n0], dtype=t.float64, device=dev)
        self._avg = _lib.FieldAverage(self.t_start, self._sum.data_ptr(), self._sum2.data_ptr(),
                                      self._T.data_ptr())

    def execute(self, sim) -> None:
        with sim._on_stream():
            if self.sim is not sim or self._avg is None:
                self._bind(sim)
            sim._call("cfd2d_field_average_accumulate", C.byref(self._avg))

    def _host(self):
        if self._avg is None:
            return None
        with self.sim._on_stream():
            self.sim._sync()
            T = self._T.cpu().numpy()
            if T[1] == self._n0:  # nothing accumulated yet
                return None
            s1, s2 = self._sum.cpu().numpy(), self._sum2.cpu().numpy()
        return float(T[0]), {k: s1[i] for i, k in enumerate(self.KEYS)}, {k: s2[i] for i, k in enumerate(self.KEYS)}

    @property
    def T(self) -> float:
        h = self._host()
        return h[0] if h else 0.0

    @property
    def sum(self):
        h = self._host()
        return h[1] if h else None

    @property
    def sum2(self):
        h = self._host()
        return h[2] if h else None

    def mean(self, k: str) -> np.ndarray:
        T, s1, _ = self._host()
        return s1[k] / max(T, 1e-300)

    def rms(self, k: str) -> np.ndarray:
        T, s1, s2 = self._host()
        m = s1[k] / max(T, 1e-300)
        return np.sqrt(np.maximum(s2[k] / max(T, 1e-300) - m * m, 0.0))

    def write(self, outdir: Path) -> list[Path]:
        h = self._host()
        if h is None or h[0] <= 0:
            return []
        outdir = Path(outdir)
        np.savez_compressed(outdir / "mittelwerte.npz", T=h[0],
                            **{f"{k}_mittel": self.mean(k) for k in self.KEYS},
                            **{f"{k}_rms": self.rms(k) for k in self.KEYS})
        return [outdir / "mittelwerte.npz"]

    def describe(self) -> str:
        return f"Zeitmittelung ab t = {self.t_start:g}"

    def spec(self) -> dict:
        return {"typ": "mittelwerte", "t_start": self.t_start}


def write_vtk(sim, path) -> Path:
    """All fields as a legacy binary VTK file (RECTILINEAR_GRID) for ParaView
    (cfd2d/functions.py:244-287). The payload (big-endian float32, VTK cell order)
    is packed on the device; the host adds the header lines."""
    t = _lib.torch()
    g = sim.grid
    path = Path(path)
    nx, ny = g.nx, g.ny
    N = nx * ny
    names = [k for k in available_fields(sim) if k not in ("u", "v")] + ["fluid"]
    with sim._on_stream():
        sim._flush_mirrors()
        descs = [(_lib.FIELD_FLUID, None) if k == "fluid" else device_field(sim, k) for k in names]
        blocks = []
        vec = None
        for start in range(0, len(descs), _lib.MAX_FIELDS):
            chunk = descs[start:start + _lib.MAX_FIELDS]
            buf = t.empty(4 * N * (3 + len(chunk)), dtype=t.uint8, device=_lib.device())
            sim._call("cfd2d_vtk_pack", _field_array(chunk), len(chunk), _lib.ptr(buf))
            host = buf.cpu().numpy().tobytes()
            if vec is None:
                vec = host[:12 * N]
            blocks += [host[12 * N + 4 * N * k: 12 * N + 4 * N * (k + 1)] for k in range(len(chunk))]
    with open(path, "wb") as fh:
        def line(s):
            fh.write((s + "\n").encode("ascii"))

        line("# vtk DataFile Version 3.0")
        line(f"cfd2d t={sim.t:.8g}")
        line("BINARY")
        line("DATASET RECTILINEAR_GRID")
        line(f"DIMENSIONS {nx + 1} {ny + 1} 1")
        line(f"X_COORDINATES {nx + 1} float")
        fh.write(g.xn.astype(">f4").tobytes())
        line("")
        line(f"Y_COORDINATES {ny + 1} float")
        fh.write(g.yn.astype(">f4").tobytes())
        line("")
        line("Z_COORDINATES 1 float")
        fh.write(np.zeros(1, ">f4").tobytes())
        line("")
        line(f"CELL_DATA {N}")
        line("VECTORS U float")
        fh.write(vec)
        line("")
        for k, blk in zip(names, blocks):
            line(f"SCALARS {k.replace(' ', '_')} float 1")
            line("LOOKUP_TABLE default")
            fh.write(blk)
            line("")
    return path


class VTKWriter(FunctionObject):
    """VTK files at fixed time intervals plus a ParaView series (cfd2d/functions.py:290-322)."""

    def __init__(self, interval: float, outdir):
        self.interval = float(interval)
        self.outdir = Path(outdir) / "vtk"
        self.next_t = 0.0
        self.files: list = []
        self.name = "vtk"

    def execute(self, sim) -> None:
        if sim.t + 1e-12 >= self.next_t:
            self.outdir.mkdir(parents=True, exist_ok=True)
            f = write_vtk(sim, self.outdir / f"feld_{len(self.files):05d}.vtk")
            self.files.append((sim.t, f.name))
            self.next_t = sim.t + self.interval

    def write(self, outdir: Path) -> list[Path]:
        if not self.files:
            return []
        series = {"file-series-version": "1.0",
                  "files": [{"name": n, "time": t} for t, n in self.files]}
        p = self.outdir / "feld.vtk.series"
        p.write_text(json.dumps(series, indent=1), encoding="utf-8")
        return [p]

    def describe(self) -> str:
        return f"VTK-Export alle Δt = {self.interval:g} nach {self.outdir}"

    def spec(self) -> dict:
        return {"typ": "vtk", "intervall": self.interval}


def save_checkpoint(sim, path) -> Path:
    """Write the complete state of ``sim`` to ``path`` (cfd2d/functions.py:326-346)."""
    path = Path(path)
    data = {"u": sim.u, "v": sim.v, "p": sim.p, "t": sim.t, "n": sim.n, "dt": sim.dt,
            "flow_force": sim.flow_force, "dt_old": sim.dt_old if sim.dt_old else 0.0,
            "fluid": sim.grid.fluid}
    if sim.hu_old is not None:
        data["hu_old"] = sim.hu_old
        data["hv_old"] = sim.hv_old
    for name, f in sim.scalars.items():
        data[f"skalar_{name}"] = f.phi
    for k, m in enumerate(sim.models):
        for key, arr in (m.state() if hasattr(m, "state") else {}).items():
            data[f"modell{k}_{key}"] = arr
    hist = sim.history
    data["history_json"] = json.dumps({k: list(map(float, v)) for k, v in hist.__dict__.items()
                                       if k != "extra"} | {"extra": {k: list(map(float, v))
                                                                    for k, v in hist.extra.items()}})
    data["pressure_x0"] = sim.pressure._d_x0.cpu().numpy()
    np.savez_compressed(path, **data)
    return path


def load_checkpoint(sim, path) -> None:
    """Load a checkpoint into a simulation built the same way (cfd2d/functions.py:349-380).
    Raises ValueError when the grid or the geometry differ."""
    d = np.load(Path(path), allow_pickle=False)
    if d["u"].shape != sim.u.shape or not np.array_equal(d["fluid"], sim.grid.fluid):
        raise ValueError("Der Speicherstand passt nicht zum Gitter bzw. zur Geometrie dieses Falls.")
    sim.u = d["u"]
    sim.v = d["v"]
    sim.p = d["p"]
    ab2_old = "hu_old" in d and sim.scheme == "ab2"
    if ab2_old:
        # the device keeps the last tendency in hu/hv; it is the AB2 old term of the next step
        sim.hu = d["hu_old"]
        sim.hv = d["hv_old"]
    with sim._on_stream():
        sim._sync()
        st = sim._pull()
        st.t = float(d["t"])
        st.n = int(d["n"])
        st.dt = float(d["dt"])
        st.flow_force = float(d["flow_force"])
        st.dt_old = float(d["dt_old"])
        st.have_old = 1 if ab2_old else 0
        sim._push()
    for name, f in sim.scalars.items():
        key = f"skalar_{name}"
        if key in d:
            f.phi[:] = d[key]
            f.fill_ghosts()
    for k, m in enumerate(sim.models):
        if hasattr(m, "set_state"):
            st_m = {key.split("_", 1)[1]: d[key] for key in d.files if key.startswith(f"modell{k}_")}
            if st_m:
                m.set_state(sim, st_m)
    h = json.loads(str(d["history_json"]))
    extra = h.pop("extra", {})
    for k, v in h.items():
        setattr(sim.history, k, v)
    sim.history.extra = extra
    sim._hist_seen = int(d["n"])
    ps = sim.pressure
    if "pressure_x0" in d and d["pressure_x0"].shape == tuple(ps._d_x0.shape):
        x0 = d["pressure_x0"]
    else:
        # a checkpoint of the reference: start the next solve from the saved pressure
        x0 = np.where(ps.fluid, np.asarray(d["p"])[1:-1, 1:-1], 0.0)
    with sim._on_stream():
        ps._d_x0.copy_(sim._t.from_numpy(np.ascontiguousarray(x0, dtype=np.float64)).to(ps._d_x0.device))
    sim._apply_bc()


class Checkpoint(FunctionObject):
    """A checkpoint (``checkpoint.npz``, overwritten) at fixed time intervals
    (cfd2d/functions.py:382-410)."""

    def __init__(self, interval: float, outdir):
        self.interval = float(interval)
        self.path = Path(outdir) / "checkpoint.npz"
        self.next_t = self.interval
        self.name = "checkpoint"
        self.sim = None

    def execute(self, sim) -> None:
        self.sim = sim
        if sim.t + 1e-12 >= self.next_t:
            self.path.parent.mkdir(parents=True, exist_ok=True)
            save_checkpoint(sim, self.path)
            self.next_t = sim.t + self.interval

    def write(self, outdir: Path) -> list[Path]:
        if self.sim is not None:
            self.path.parent.mkdir(parents=True, exist_ok=True)
            save_checkpoint(self.sim, self.path)
            return [self.path]
        return []

    def describe(self) -> str:
        return f"Speicherstand alle Δt = {self.interval:g}"

    def spec(self) -> dict:
        return {"typ": "checkpoint", "intervall": self.interval}


def build_function_objects(specs: list[dict], outdir) -> list[FunctionObject]:
    """Function objects from their case-file specs (cfd2d/functions.py:413-430)."""
    out = []
    for s in specs or []:
        t = s["typ"]
        if t == "sonden":
            out.append(Probes(s["punkte"], s.get("felder", ("u", "v", "pressure")), s.get("alle", 1)))
        elif t == "linie":
            out.append(LineSample(s["p0"], s["p1"], s.get("n", 100), s.get("felder", ("u", "v")),
                                  s.get("name", "linie")))
        elif t == "mittelwerte":
            out.append(FieldAverage(s.get("t_start", 0.0)))
        elif t == "vtk":
            out.append(VTKWriter(s["intervall"], outdir))
        elif t == "checkpoint":
            out.append(Checkpoint(s["intervall"], outdir))
        else:
            raise ValueError(f"Unbekanntes Function Object {t!r}")
    return out

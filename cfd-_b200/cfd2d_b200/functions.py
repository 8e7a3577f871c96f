"""Checkpoint and restart of a simulation from its device state (cfd2d/functions.py:326-380).

The file is the reference's schema (``np.savez_compressed``): u, v, p, t, n, dt,
flow_force, dt_old, the fluid flags, hu_old/hv_old after an AB2 step, one
``skalar_<name>`` array per scalar field, per-model state and the history as JSON,
so a checkpoint written here loads in the reference and the other way round. One key
is added: ``pressure_x0``, the warm start of the iterative pressure solve, which makes
a restart continue bit-identically (the reference ignores keys it does not read).
"""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np


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

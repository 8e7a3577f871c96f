"""Field catalogue of a simulation (cfd2d/visualization.py:41-93, without plotting).

``available_fields`` and ``field_data`` keep the reference's names, labels and
order; the function objects (cfd2d_b200.functions) use ``device_field`` to read
the same fields on the device. Live plots and animations are not part of this
package (it does not depend on matplotlib).
"""

from __future__ import annotations

import numpy as np

from . import _lib

FIELDS = {
    "speed": "Geschwindigkeitsbetrag |u|",
    "vorticity": "Wirbelstärke ω",
    "pressure": "Druck p",
    "u": "Geschwindigkeit u (x-Richtung)",
    "v": "Geschwindigkeit v (y-Richtung)",
    "streamfunction": "Stromfunktion ψ",
}


def _model_fields(sim):
    """[(key, label, kind, tensor or host cell array)] of the models, in model order."""
    out = []
    for m in getattr(sim, "models", []):
        dev = m.device_fields(sim) if hasattr(m, "device_fields") else None
        if dev is not None:
            out += [(k, label, kind, t) for k, (label, kind, t) in dev.items()]
        else:
            out += [(k, label, None, data) for k, (label, data) in m.fields(sim).items()]
    return out


def available_fields(sim) -> dict:
    """All named fields: the base fields plus the models' (visualization.py:80-89)."""
    out = dict(FIELDS)
    for k, label, _, _ in _model_fields(sim):
        out[k] = label
    if (getattr(sim, "variable_viscosity", False) and not getattr(sim, "variable_density", False)
            and "nu_t" not in out):
        out["nu_t"] = "Turbulente Viskosität ν_t"
    return out


_BASE_KINDS = {"speed": _lib.FIELD_SPEED, "vorticity": _lib.FIELD_VORTICITY, "pressure": _lib.FIELD_PRESSURE}


def device_field(sim, field: str, faces: bool = False):
    """(CFD2D_FIELD_* kind, device tensor or None) of a named field
    (visualization.py:50-73 order). ``faces``: u and v on their own staggered
    grids (sampling, cfd2d/solver.py:598-615) instead of cell means."""
    t = _lib.torch()
    if field in ("u", "v"):
        if faces:
            return (_lib.FIELD_U if field == "u" else _lib.FIELD_V), None
        return (_lib.FIELD_UC if field == "u" else _lib.FIELD_VC), None
    if field in _BASE_KINDS:
        return _BASE_KINDS[field], None
    if field == "streamfunction":
        return _lib.FIELD_NODE, streamfunction_device(sim)
    for k, _, kind, data in _model_fields(sim):
        if k != field:
            continue
        if kind is not None:
            return kind, data
        # a model with host fields only: its (nx, ny) cell array, padded
        g = sim.grid
        pad = np.full((g.nx + 2, g.ny + 2), np.nan)
        pad[1:-1, 1:-1] = np.asarray(data, dtype=np.float64)
        return _lib.FIELD_CELL, _lib.to_dev(pad, t.float64)
    if field == "nu_t" and getattr(sim, "variable_viscosity", False):
        return _lib.FIELD_CELL, sim._nu_t
    raise ValueError(f"Unbekanntes Feld {field!r}, erlaubt: {list(available_fields(sim))}")


def streamfunction_device(sim, out=None):
    """Stream function psi (nx+1, ny+1) on the device (cfd2d/solver.py:580-596)."""
    t = _lib.torch()
    g = sim.grid
    if out is None:
        out = t.empty((g.nx + 1, g.ny + 1), dtype=t.float64, device=_lib.device())
    with sim._on_stream():
        sim._flush_mirrors()
        sim._call("cfd2d_streamfunction", _lib.ptr(out))
    return out


def field_data(sim, field: str) -> np.ndarray:
    """Field at the cell centres, (nx, ny), NaN on solids (visualization.py:50-73),
    evaluated on the device."""
    t = _lib.torch()
    kind, data = device_field(sim, field)
    g = sim.grid
    f = (_lib.Field * 1)(_lib.Field(kind, 0, data.data_ptr() if data is not None else None))
    with sim._on_stream():
        sim._flush_mirrors()
        out = t.empty((g.nx, g.ny), dtype=t.float64, device=_lib.device())
        sim._call("cfd2d_cell_values", f, _lib.ptr(out))
        return out.cpu().numpy()

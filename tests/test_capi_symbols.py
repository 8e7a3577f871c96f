"""The C-ABI library loads without a GPU and exports every declared entry point."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

from conftest import ROOT

HEADER = ROOT / "include" / "cfd2d_b200.h"
LIB = ROOT / "cfd-_b200" / "cfd2d_b200" / "lib" / "libcfd2d_b200.so"


def declared():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cfd2d_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared()
    assert "cfd2d_sim_step" in names and "cfd2d_pressure_solve" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol():
    assert LIB.exists(), f"{LIB} not built"
    lib = ctypes.CDLL(str(LIB))
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    lib.cfd2d_version.restype = ctypes.c_char_p
    assert lib.cfd2d_version().startswith(b"cfd2d_b200")


def test_python_binding_covers_header():
    from cfd2d_b200 import _lib

    assert sorted(_lib.exported_symbols()) == declared()


def test_struct_sizes_match_the_header():
    # the library computes its scratch needs from these structs; a mismatch in the
    # ctypes mirror would shift every field after it
    from cfd2d_b200 import _lib

    assert ctypes.sizeof(_lib.State) % 8 == 0
    assert _lib.Sim.state.offset > _lib.Sim.sst.offset


STRUCTS = {"State": "cfd2d_state", "Poisson": "cfd2d_poisson", "Scalar": "cfd2d_scalar", "SST": "cfd2d_sst",
           "Smagorinsky": "cfd2d_smagorinsky", "Vof": "cfd2d_vof", "Monitor": "cfd2d_monitor", "Sim": "cfd2d_sim",
           "FcgScalars": "cfd2d_fcg_scalars", "FcgControl": "cfd2d_fcg_control", "Field": "cfd2d_field",
           "ProbeSeries": "cfd2d_probe_series", "FieldAverage": "cfd2d_field_average"}


def test_ctypes_layout_equals_the_c_header(tmp_path):
    """Every ctypes mirror has the C struct's size and every field its offset: a C
    program compiled against include/cfd2d_b200.h prints them."""
    import shutil
    import subprocess

    from cfd2d_b200 import _lib

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ["#include <stddef.h>", "#include <stdio.h>", f'#include "{HEADER}"', "int main(void) {"]
    expect = []
    for py, cname in STRUCTS.items():
        cls = getattr(_lib, py)
        lines.append(f'printf("%zu\\n", sizeof({cname}));')
        expect.append(ctypes.sizeof(cls))
        for name, _ in cls._fields_:
            lines.append(f'printf("%zu\\n", offsetof({cname}, {name}));')
            expect.append(getattr(cls, name).offset)
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c11", str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert got == expect


def test_entry_points_reject_invalid_arguments_before_any_device_work():
    """The C ABI checks its arguments first and answers CFD2D_E_ARG (-1) without
    touching the device (runs without a GPU)."""
    from cfd2d_b200 import _lib

    lib = _lib.lib()
    E_ARG = _lib.E_ARG
    null = None
    sim = _lib.Sim()  # nx = ny = 0, no state
    assert lib.cfd2d_sim_step(null, null) == E_ARG
    assert lib.cfd2d_sim_step(ctypes.byref(sim), null) == E_ARG
    assert lib.cfd2d_sim_smagorinsky_pre_momentum(ctypes.byref(sim), null) == E_ARG
    assert lib.cfd2d_sim_sst_pre_momentum(ctypes.byref(sim), null) == E_ARG
    assert lib.cfd2d_sim_vof_properties(ctypes.byref(sim), null) == E_ARG
    assert lib.cfd2d_sim_wall_distance(ctypes.byref(sim), null, null, 0, null) == E_ARG
    assert lib.cfd2d_sample(ctypes.byref(sim), null, 0, null, null, 0, null, null) == E_ARG
    assert lib.cfd2d_probe_record(ctypes.byref(sim), null, 0, null, null, 0, null, null) == E_ARG
    assert lib.cfd2d_field_average_accumulate(ctypes.byref(sim), null, null) == E_ARG
    assert lib.cfd2d_streamfunction(ctypes.byref(sim), null, null) == E_ARG
    assert lib.cfd2d_vtk_pack(ctypes.byref(sim), null, 0, null, null) == E_ARG
    assert lib.cfd2d_cell_values(ctypes.byref(sim), null, null, null) == E_ARG
    assert lib.cfd2d_vof_advect(null, null, null, null, 4, 4, 0.1, 0.1, 0.01, 1.0, 0, 0.0, null, null) == E_ARG
    assert lib.cfd2d_pressure_solve(null, null, null, 1e-8, 10, null, null, null) == E_ARG
    op = _lib.Poisson()
    assert lib.cfd2d_pressure_solve_static(ctypes.byref(op), null, null, 1e-8, 10, null, null, null) == E_ARG
    assert lib.cfd2d_wall_distance_workspace_bytes(0, 4) == 0

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

"""The C-ABI library loads without a GPU and exports every declared entry point."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

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

"""Shared test setup: import paths, the ``gpu`` marker and fixture loading."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
for p in (ROOT, ROOT / "cfd-_b200", GOLDEN):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def golden(name: str) -> dict:
    """Load ``tests/golden/<name>.npz`` as a dict of arrays."""
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def cuda_lib():
    """The built CUDA library; skips nothing: a GPU test without it must fail loudly."""
    from cfd2d_b200 import _lib

    return _lib.lib()

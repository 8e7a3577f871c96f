"""How far two correct runs of the reference's CG drift apart at 1024 x 512.

Runs the oracle's scipy-form CG (the reference's iteration, same stop test) on
step 1 of the obstacle-flow benchmark case with its dot products summed
pairwise (``np.sum(a * b)``) instead of by BLAS ``ddot``, and prints the
iteration count and the relative max-norm difference of u, v, p (every 8th
value) from the reference's own run stored in golden_obstacles1024.npz. Only
the rounding of the dot products differs; the printed p difference is the
spread any FP64 implementation of the reference's solve must be allowed.

    python tests/golden/sensitivity_obstacles1024.py     (about 4 minutes)

Measured here: 3847 iterations (the reference's count), u 8.7e-13, v 7.3e-13,
p 5.4e-10.
"""

from __future__ import annotations

import ast
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
for p in (str(ROOT), str(ROOT / "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

import oracle as O  # noqa: E402
import oracle.cfd2d_oracle as OC  # noqa: E402
from conftest import golden  # noqa: E402


def main():
    g = golden("golden_obstacles1024")
    obst, re = ast.literal_eval(str(g["obs1024_spec"]))
    blas_dot = np.dot

    def pairwise_dot(a, b):
        if isinstance(a, np.ndarray) and a.ndim == 1 and isinstance(b, np.ndarray) and b.ndim == 1:
            return float(np.sum(a * b))
        return blas_dot(a, b)

    OC.np.dot = pairwise_dot
    try:
        t0 = time.time()
        sim = O.custom_obstacles(obst, lx=2.0, ly=1.0, nx=1024, ny=512, re=re, tol=1e-8)
        sim.step()
    finally:
        OC.np.dot = blas_dot
    print(f"{time.time() - t0:.0f}s; iterations {sim.iterations[-1]} (reference {int(g['obs1024_its'][0])})")
    for name in ("u", "v", "p"):
        a = getattr(sim, name)
        d = np.abs(a[::8, ::8] - g[f"obs1024_1_{name}_sub"]).max() / float(g[f"obs1024_1_{name}_max"])
        print(f"{name}: {d:.2e}")


if __name__ == "__main__":
    main()

"""CPU oracle for the cfd2d projection time step.

TEST INFRASTRUCTURE ONLY. This package restates, in NumPy, the arithmetic of the
reference solver (kaeptnzursee1910/CFD-, package ``cfd2d``) so that the CUDA
implementation in ``cfd-_b200/`` can be checked against it. Only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference`` legs of
``bench.py`` may import it, and only to check results or as the timed CPU baseline;
the product never calls into it.

Parity is pinned: ``tests/golden/make_golden.py`` runs the reference itself (in
the container that has it) and stores its outputs as fixtures, and the CPU tests
check this oracle against them (bitwise for the stencils and masks, to the last
bit for the scipy-trajectory CG on the same machine).
"""

from .cfd2d_oracle import *  # noqa: F401,F403

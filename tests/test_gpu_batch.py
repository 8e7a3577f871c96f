"""Independent cases stepped side by side on one GPU (cfd2d_b200.batch) (GPU).

Concurrency must not change any case: every member of a batch ends bit-identical to
the same case stepped on its own.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu]


def test_batched_steps_equal_single_case_steps(cuda_lib):
    from cfd2d_b200 import batch

    sizes = (32, 64, 96)
    together = batch.uneven_cavities(n_cases=6, seed=5, sizes=sizes)
    alone = batch.uneven_cavities(n_cases=6, seed=5, sizes=sizes)
    b = batch.Batch([c.sim for c in together])
    b.advance(10)
    ms = b.timed_advance(5)
    assert ms > 0.0
    for c in alone:
        c.sim.advance(15)
    for a, s in zip(together, alone):
        assert a.sim.n == s.sim.n == 15
        for name in ("u", "v", "p"):
            assert np.array_equal(getattr(a.sim, name), getattr(s.sim, name)), name
    # the heated members carry their temperature along
    for a, s in zip(together[1::2], alone[1::2]):
        ta = next(iter(a.sim.scalars.values())).phi
        ts = next(iter(s.sim.scalars.values())).phi
        assert np.array_equal(ta, ts)

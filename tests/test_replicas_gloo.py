"""The replica harness of bench.py across two ranks on the CPU (gloo).

The path does not partition: ``bench.py --gpus N`` runs N independent replicas and
reports the whole-job rate from the slowest rank's device time. What crosses ranks
is the max-over-ranks timing and the barriers around the timed region; the
reference arm runs on rank 0 only.
"""

from __future__ import annotations

import io
import os
import socket
from contextlib import redirect_stdout

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, q) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    dist, r, w = bench._dist()
    try:
        assert (r, w) == (rank, world)
        # each rank times its own replica; the job is as slow as its slowest rank
        slowest = bench._max_over_ranks(dist, 1.0 + rank)
        bench._barrier(dist)

        class Args:
            steps, warmup = 1, 0

        buf = io.StringIO()
        if rank != 0:
            with redirect_stdout(buf):
                bench.run_reference(Args, dist, r, w)  # returns at once on ranks > 0
        q.put((rank, slowest, buf.getvalue()))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_rank0_only_reference_arm():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
            pytest.fail("a gloo rank did not finish")
        assert p.exitcode == 0
    out = sorted(q.get(timeout=5) for _ in range(2))
    assert [o[1] for o in out] == [2.0, 2.0]
    assert out[1][2] == ""  # rank 1 printed no reference line

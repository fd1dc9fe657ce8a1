"""The benchmark's multi-rank plumbing on CPU: two gloo ranks (127.0.0.1) take the barrier and the max over ranks
that the timing uses (the GPU run uses the same class over NCCL, one process per GPU)."""

from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest

torch = pytest.importorskip("torch")
ROOT = Path(__file__).resolve().parents[1]


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.dist_env() == (rank, world, rank)
    d = bench.Dist(world, "gloo")
    d.barrier()
    got = d.max(10.0 * (rank + 1))  # each rank's time; the step time is the slowest
    d.barrier()
    d.close()
    q.put((rank, got))


def test_two_gloo_ranks_take_the_max():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=10) for _ in procs)
    assert got == [(0, 20.0), (1, 20.0)]


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    d = bench.Dist(1, "gloo")
    d.barrier()
    assert d.max(3.5) == 3.5
    d.close()

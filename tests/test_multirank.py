"""Replica plumbing of bench.py at world size 2 on CPU (gloo): every rank
runs its own replica, the job time is the max over ranks, and the reported
value is the units of all ranks over that time."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(dist)
        local_ms = 10.0 * (rank + 1)  # rank 1 is the slow one
        ms = bench.max_over_ranks(dist, local_ms)
        out[rank] = (ms, bench.replica_value(1e9, world, ms))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_use_the_slowest_rank():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0][0] == res[1][0] == 20.0
    assert res[0][1] == pytest.approx(2e9 / 0.020)

"""The multi-GPU path of bench.py runs N independent replicas (one process per
GPU, no data-path collective): each rank times its own steps on its device,
and the job throughput is all ranks' work over the slowest rank's time. This
checks that reduction with two gloo ranks on the CPU (rendezvous on
127.0.0.1), the only cross-rank step the replicas take."""

from __future__ import annotations

import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q) -> None:
    import datetime
    import sys

    import torch.distributed as dist

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = [2.0, 5.0][rank]
        value, ms_max = bench.job_throughput(1000, local_ms, dist)
        q.put((rank, value, ms_max))
    finally:
        dist.destroy_process_group()


def test_replica_throughput_is_all_work_over_slowest_rank():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, value, ms_max in got:
        assert ms_max == 5.0
        assert value == pytest.approx(1000 * 2 / 5e-3)


def test_single_process_throughput():
    import bench

    value, ms = bench.job_throughput(500, 4.0)
    assert ms == 4.0 and value == pytest.approx(500 / 4e-3)

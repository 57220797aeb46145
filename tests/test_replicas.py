"""The multi-rank host path of the benchmark, on CPU with two gloo ranks."""

from __future__ import annotations

import os
import socket

import pytest

from conftest import pkg


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        m = pkg("replicas").max_over_ranks(1.5 + rank, dist, "cpu")
        out.put((rank, m))
    finally:
        dist.destroy_process_group()


def test_two_ranks_agree_on_the_slowest_time():
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
    got = dict(q.get(timeout=10) for _ in range(2))
    assert got == {0: 2.5, 1: 2.5}
    rep = pkg("replicas")
    assert rep.whole_job_rate(38, 2, 20.0) == pytest.approx(3.8)
    assert rep.max_over_ranks(4.0) == 4.0

"""The multi-rank host path of the benchmark, on CPU with two gloo ranks: a sweep partitioned over ranks."""

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
        rep = pkg("replicas")
        sweep = pkg("sweep")
        dist.barrier()
        m = rep.max_over_ranks(1.5 + rank, dist, "cpu")
        # this rank's share of one 2 x 8-point sweep, and the tallies summed over ranks
        mine = rep.partition(sweep.sample_points(8 * world, 0), rank, world)
        tally = rep.sum_over_ranks([len(mine), sum(p.order for p in mine)], dist, "cpu")
        out.put((rank, m, [(p.area_ratio, p.back_pressure_ratio, p.order, p.refine, p.element) for p in mine], tally))
    finally:
        dist.destroy_process_group()


def test_two_ranks_partition_one_sweep():
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
    got = {r: (m, pts, tally) for r, m, pts, tally in (q.get(timeout=10) for _ in range(2))}
    assert got[0][0] == got[1][0] == 2.5
    # the ranks' shares are disjoint and together are the single-rank sweep of 16 points, point for point
    whole = [(p.area_ratio, p.back_pressure_ratio, p.order, p.refine, p.element)
             for p in pkg("sweep").sample_points(16, 0)]
    assert got[0][1] == whole[0::2] and got[1][1] == whole[1::2]
    assert sorted(got[0][1] + got[1][1]) == sorted(whole)
    assert got[0][2] == got[1][2] == [16.0, float(sum(p[2] for p in whole))]


def test_partition_and_rates():
    rep = pkg("replicas")
    assert rep.partition(range(7), 0, 3) == [0, 3, 6]
    assert rep.partition(range(7), 2, 3) == [2, 5]
    assert sorted(sum((rep.partition(range(11), r, 4) for r in range(4)), [])) == list(range(11))
    assert rep.partition(range(5), 0, 1) == list(range(5))
    with pytest.raises(ValueError):
        rep.partition(range(5), 2, 2)
    assert rep.whole_job_rate(76, 20.0) == pytest.approx(3.8)
    assert rep.max_over_ranks(4.0) == 4.0
    assert rep.sum_over_ranks([1, 2.5]) == [1.0, 2.5]

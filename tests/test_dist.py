"""Multi-rank plumbing of bench.py on CPU (gloo, world_size 2): the timed region's length is
the max over ranks and the job throughput counts every rank's replica products."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as tdist
    import bench
    tdist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                             timeout=datetime.timedelta(seconds=60))
    try:
        m = bench.max_over_ranks(1.5 + rank)       # rank 0: 1.5, rank 1: 2.5
        q.put((rank, m, bench.job_throughput(world, 20, m)))
    finally:
        tdist.destroy_process_group()


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [2.5, 2.5]
    assert all(abs(r[2] - 2 * 20 / 2.5) < 1e-9 for r in res)
    assert all(p.exitcode == 0 for p in procs)


def test_single_process_has_no_group():
    import bench
    assert bench.max_over_ranks(3.25) == 3.25
    assert bench.job_throughput(1, 10, 2.0) == 5.0

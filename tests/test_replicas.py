"""The multi-GPU path is N independent replicas (the form factor needs no exchange): the
bench's slowest-rank time and whole-job throughput, run as two gloo ranks on the CPU."""
import os
import socket
import sys

import pytest

from conftest import ROOT

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import datetime

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(100.0 + 50.0 * rank, dist, "cpu")  # rank 1 is slower
        value = bench.job_throughput(world, 8.0e11, ms * 1e-3)
        out.put((rank, ms, value))
    finally:
        dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, value in res:
        assert ms == 150.0                       # the max over ranks, on every rank
        assert value == pytest.approx(2 * 8.0e11 / 0.150)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(12.5, None, "cpu") == 12.5
    assert bench.job_throughput(1, 10.0, 2.0) == 5.0

"""Replica-parallel aggregation (bench.py --gpus N) with two gloo ranks on
CPU: the job's time is the slowest rank's, its work the sum over ranks, and
every rank sees the same result."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from openludwig_b200 import replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        # rank r did (r + 1) * 1e6 units in (r + 1) * 10 ms
        rate, ms = replicas.job_rate((rank + 1) * 1e6, (rank + 1) * 10.0)
        out.put((rank, replicas.world(), rate, ms))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_slowest_time_summed_work():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, (r, n), rate, ms in res:
        assert (r, n) == (rank, 2)
        assert ms == pytest.approx(20.0)               # slowest rank
        assert rate == pytest.approx(3e6 / 0.020)      # (1 + 2) e6 units in 20 ms


def test_single_process_is_identity():
    assert replicas.world() == (0, 1)
    rate, ms = replicas.job_rate(5e6, 25.0)
    assert ms == 25.0 and rate == pytest.approx(2e8)

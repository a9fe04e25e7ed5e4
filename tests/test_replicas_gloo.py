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


def test_bench_gpus_flag_starts_the_ranks_itself():
    """`python bench.py --gpus 2` without torchrun starts two ranks (here its
    CPU self-test of the launcher: gloo barrier and max over ranks) and
    reports n_gpus = 2 from rank 0."""
    import json
    import os
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    env = {k: v for k, v in os.environ.items()
           if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    r = subprocess.run([sys.executable, str(root / "bench.py"), "--gpus", "2", "--steps", "2",
                        "--warmup", "3", "--launcher-selftest"], capture_output=True, text=True,
                       timeout=300, env=env, cwd=str(root))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    assert lines[0]["n_gpus"] == 2 and lines[0]["selftest"]
    assert lines[0]["max_rank_ms"] == 1.5      # the slower rank's time wins

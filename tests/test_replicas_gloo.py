"""bench.py's multi-GPU bookkeeping (replicas only: every rank advances its own field, no data
exchange) on two gloo ranks on the CPU: the slowest rank's time is taken, the whole-job rate
counts every replica's steps, and the reference arm runs on rank 0 only."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, REPO)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = 10.0 + 5.0 * rank  # rank 1 is the slower replica
    ms_max = bench.max_over_ranks(ms, world)
    q.put((rank, ms_max, bench.replica_throughput(100, ms_max, world)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=5) for _ in range(2))
    for rank, ms_max, value in res:
        assert ms_max == 15.0
        assert abs(value - 2 * 100 / 0.015) < 1e-6


def test_reference_arm_prints_only_on_rank_zero(monkeypatch):
    sys.path.insert(0, REPO)
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference"])
    args = bench.parse()
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.main_reference(args)
    assert buf.getvalue() == ""

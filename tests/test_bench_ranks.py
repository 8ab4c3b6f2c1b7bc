"""Multi-process host logic of bench.py on the CPU (gloo, world size 2): the
max-over-ranks timing reduction, and the reference arm doing no work on
ranks other than 0."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        got = bench.max_over_ranks([1.0 + rank, 10.0 - rank, 3.5], dist, "cpu")
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(2))
    assert res[0] == res[1] == [2.0, 10.0, 3.5]


def test_max_over_ranks_single():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([1.5, 2.5], None, "cpu") == [1.5, 2.5]


def test_reference_arm_other_ranks_idle(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import argparse

    import bench
    monkeypatch.setenv("RANK", "1")
    called = []
    monkeypatch.setattr(bench, "run_cpu_baseline", lambda *a, **k: called.append(1))
    args = argparse.Namespace(gpus=2, steps=1, warmup=1)
    assert bench.reference_arm(args, "dense32") == 0
    assert not called and capsys.readouterr().out == ""

"""Multi-process logic of bench.py, on CPU with the gloo backend (world size 2): every rank runs its
own replica and reports its own time; the job time is the max over ranks and the whole-job rate
counts every replica; the reference arm runs on rank 0 alone (other ranks exit without work)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, ws, port, q):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    import bench
    try:
        dist.barrier()
        t = bench.max_over_ranks(0.5 + rank, ws, "cpu")   # rank 1 is the slow one
        rate = bench.whole_job_rate(ws, 1000, 4, t)
        q.put((rank, t, rate))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, t, rate in got:
        assert t == pytest.approx(1.5)
        assert rate == pytest.approx(2 * 1000 * 3 * 4 / 1.5)


def test_single_rank_is_identity():
    import bench
    assert bench.max_over_ranks(0.25, 1, "cpu") == 0.25


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    import argparse
    import bench
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    args = argparse.Namespace(steps=2, warmup=1)
    assert bench.run_reference(args) == 0
    assert capsys.readouterr().out == ""

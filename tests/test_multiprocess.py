"""The N>1 plumbing of the benchmark on CPU (gloo, world size 2): replicas report the slowest
rank's time, and only rank 0 of the reference arm does work."""
import datetime
import os
import socket
import types

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        q.put((rank, bench.max_over_ranks(1.5 + rank, dist, device="cpu")))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == {0: 2.5, 1: 2.5}


def test_max_over_ranks_single_process():
    import bench
    assert bench.max_over_ranks(3.25, None) == 3.25


def test_reference_arm_other_ranks_exit_without_work(monkeypatch, capsys):
    import bench
    monkeypatch.setenv("RANK", "1")
    args = types.SimpleNamespace(size=100, steps=10, warmup=3)
    assert bench.run_reference(args) == 0
    assert capsys.readouterr().out == ""

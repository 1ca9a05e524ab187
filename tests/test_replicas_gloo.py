"""The multi-GPU bench runs independent replicas (one solve per rank, no
data-path collective); its only collectives are the barriers around the timed
region and the maximum of the timed totals over the ranks. These run here
with two gloo ranks on the CPU, and the reference arm's non-zero ranks exit
at once without work."""
import multiprocessing as mp
import os
import socket
import types

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        got = bench.max_over_ranks(100.0 + 7.5 * rank, dist, device="cpu")
        dist.barrier()
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    results = dict(q.get(timeout=10) for _ in range(2))
    assert results == {0: 107.5, 1: 107.5}


def test_max_over_ranks_without_group():
    import bench
    assert bench.max_over_ranks(3.25) == 3.25


def test_reference_arm_other_ranks_exit(monkeypatch, capsys):
    import bench
    monkeypatch.setenv("RANK", "1")
    args = types.SimpleNamespace(cpu_threads=1, grid=4, tiles=1, sigma=1.5, gpus=2, steps=1, warmup=0,
                                 inner_maxit=10, inner_tol=1e-4)
    assert bench.reference_arm(args) == 0
    assert capsys.readouterr().out == ""

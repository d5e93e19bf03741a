"""bench.py's multi-rank plumbing with two gloo ranks on the host: replicas
report the job's time as the slowest rank's and its work as the sum over
ranks, and every rank takes the same collective steps."""

import os
import socket

import pytest

torch = pytest.importorskip("torch")
mp = pytest.importorskip("torch.multiprocessing")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      LOCAL_RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist

    import bench

    w, r, local = bench.dist_setup(backend="gloo")
    try:
        assert (w, r, local) == (world, rank, rank)
        bench.barrier(w)
        ms = 10.0 + 5.0 * rank  # rank 1 is the slowest replica
        cells = 1000.0 * (rank + 1)  # uneven work per replica
        slowest = bench.reduce_max(ms, w)
        total = bench.reduce_sum(cells, w)
        bench.barrier(w)
        out.put((rank, slowest, total, total / (slowest / 1e3) / 1e9))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_time_and_work():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    results = sorted(out.get(timeout=10) for _ in procs)
    for rank, slowest, total, value in results:
        assert slowest == 15.0 and total == 3000.0
        assert value == pytest.approx(3000.0 / 0.015 / 1e9)


def test_single_rank_needs_no_process_group(monkeypatch):
    import bench

    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert bench.dist_setup(backend="gloo") == (1, 0, 0)
    assert bench.reduce_max(3.5, 1) == 3.5 and bench.reduce_sum(2.0, 1) == 2.0

"""The multi-GPU path of the benchmark is independent replicas, one per rank, with no collective on
the data path: the ranks meet only to time the job (the slowest rank's elapsed time) and to report
one line. These tests run that host logic as two gloo ranks on the CPU."""
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


def _rank(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    try:
        dist.barrier()
        slowest = bench.max_over_ranks(1.0 + 0.5 * rank)          # the timed region's elapsed seconds
        e2e = 1.0 / bench.max_over_ranks(1.0 / (4.0 - rank))     # per-step time, the slowest rank's
        q.put((rank, slowest, e2e, bench.replica_rate(world, 10, slowest)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, slowest, e2e, rate in got:
        assert slowest == 1.5          # max over ranks of 1.0, 1.5
        assert e2e == 3.0              # the slower rank's e2e rate
        assert rate == pytest.approx(2 * 10 / 1.5)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(2.5) == 2.5
    assert bench.replica_rate(1, 10, 2.0) == 5.0


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    assert bench.reference(None) is None   # rank 1 returns before any work (args is never read)

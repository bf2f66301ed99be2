"""Multi-GPU is replicas only: each rank relaxes its own specimen with no
data-path collective, and bench.py reports every rank's work over the
slowest rank's time. These tests run that reduction on a world-size-2
`gloo` group on the CPU (the GPUs use NCCL through the same function), and
check that the reference arm does its work on rank 0 alone."""

import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    import sys
    from datetime import timedelta

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        assert bench.dist_env() == (rank, world, rank)
        # Rank r took 1 + r seconds for 100 (r + 1) node-iterations.
        value, seconds, work = bench.replica_throughput(1.0 + rank, 100.0 * (rank + 1), world, device="cpu")
        out.put((rank, value, seconds, work))
    finally:
        dist.destroy_process_group()


def test_replica_throughput_is_total_work_over_the_slowest_rank():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    results = sorted(out.get(timeout=10) for _ in range(2))
    for rank, value, seconds, work in results:
        assert seconds == 2.0 and work == 300.0 and value == 150.0, (rank, value, seconds, work)


def test_single_rank_needs_no_process_group():
    import sys

    sys.path.insert(0, ROOT)
    import bench

    assert bench.replica_throughput(2.0, 10.0, 1) == (5.0, 2.0, 10.0)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    import sys

    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    # run_reference returns at once on a rank other than 0 (no work, no line).
    assert bench.run_reference(None) == 0

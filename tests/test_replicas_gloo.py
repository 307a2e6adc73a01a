"""The multi-GPU form of the bench is independent replicas (a full-tensor call needs no
exchange between GPUs): each rank times the same workload, the job's time is the slowest
rank's, and throughput aggregates over ranks.  This runs that host logic as two ``gloo``
ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(1.5 + rank, dist, torch.device("cpu"))  # rank 1 is slower
        e2e = bench.max_over_ranks(10.0 - rank, dist, torch.device("cpu"))  # rank 0 is slower
        dist.barrier()
        q.put((rank, ms, e2e, bench.replica_throughput(world, 1000, ms)))
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank_and_aggregate():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, ms, e2e, value in got:
        assert ms == pytest.approx(2.5)
        assert e2e == pytest.approx(10.0)
        assert value == pytest.approx(world * 1000 / 2.5e-3)


def test_single_process_needs_no_group():
    assert bench.max_over_ranks(3.25, None, None) == 3.25
    assert bench.replica_throughput(1, 500, 2.0) == pytest.approx(250000.0)


def test_reference_arm_runs_on_rank_zero_only():
    class Args:
        steps, warmup = 1, 0
    assert bench.run_reference(Args(), rank=1, world=2) is None

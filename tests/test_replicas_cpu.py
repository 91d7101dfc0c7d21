"""Multi-process plumbing of bench.py's replica mode on the CPU: two gloo
ranks (world size 2, rendezvous on 127.0.0.1) exercise the barrier, the
max-over-ranks time and the whole-job value, as `bench.py --gpus 2` under
torchrun does with NCCL (each rank an independent 512^3 replica, no
data-path collective)."""
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
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        w, r, local = bench.dist_setup()
        assert (w, r, local) == (world, rank, rank)
        bench.barrier(w)
        t = 1.0 + rank  # rank 1 is the slow replica
        tmax = bench.reduce_max(t, w)
        v = bench.job_value(100.0e9, w, tmax)
        bench.barrier(w)
        q.put((rank, tmax, v))
    finally:
        dist.destroy_process_group()


def test_two_gloo_replicas_report_max_time_and_job_value():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=5) for _ in range(world))
    for rank, tmax, v in got:
        assert tmax == 2.0                         # the slowest rank's time
        assert v == pytest.approx(100.0 * 2 / 2.0)  # all ranks' updates / max time


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_max(3.5, 1) == 3.5
    assert bench.job_value(10e9, 1, 2.0) == pytest.approx(5.0)

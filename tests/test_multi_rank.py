"""The multi-GPU bench path on CPU: two gloo ranks (replicas, weak scaling).

Every rank scores its own copy of the workload; the job's time is the
slowest rank's (an all-reduce MAX of the per-rank device times) and the
job's throughput is the units of all ranks over that time.
"""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        ms = 10.0 + 5.0 * rank          # rank 1 is the slow one
        ms_max = bench.max_over_ranks(ms, dist, "cpu")
        out[rank] = (ms_max, bench.job_rate(1000, world, ms_max))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_rank_and_the_whole_job():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        ms_max, rate = res[r]
        assert ms_max == 15.0
        assert abs(rate - 1000 * 2 / 0.015) < 1e-6


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(7.5, None, "cpu") == 7.5
    assert bench.job_rate(384000, 1, 150.0) == pytest.approx(2.56e6)

"""The multi-GPU bench paths on CPU: two gloo ranks.

Replicas (weak scaling): every rank scores its own copy of the workload; the
job's time is the slowest rank's (an all-reduce MAX of the per-rank device
times) and the job's throughput is the units of all ranks over that time.
Partitioned (``bench.py --partition``, strong scaling): the complexes are
split over the ranks by estimated work, each rank scores its share, and the
scores are gathered on every rank afterwards.
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


def _shard_rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        import oracle
        items = _small_items()
        mine = bench.shard_items(items, world)[rank]
        # each rank scores only its complexes (the oracle stands in for a GPU
        # here), then every rank holds all scores
        local = {i: oracle.Model(items[i]["family"], items[i]["rec"], items[i]["lig"])
                 .batch_energy_grid(items[i]["poses"], threads=1) for i in mine}
        merged = bench.gather_scores(local, dist)
        total = bench.sum_over_ranks(sum(len(items[i]["poses"]) for i in mine), dist, "cpu")
        out[rank] = (mine, {k: v.tolist() for k, v in merged.items()}, total)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _small_items():
    import importlib
    synth = importlib.import_module("lklight-gpu_b200.synth")
    items = []
    for k, (nr, bp, fam) in enumerate(((600, 2, "dna"), (900, 4, "pydock"), (400, 3, "dna"), (700, 2, "vdw"),
                                        (500, 5, "pydock"))):
        rec, lig = synth.globule(nr, 50 + k), synth.duplex(bp, 60 + k)
        poses = synth.to_kernel_poses(synth.setup_poses(rec["coords"], 2, 3 + k, 70 + k))
        items.append(dict(rec=rec, lig=lig, family=fam, poses=poses))
    return items


def test_partitioned_run_gathers_every_complex_once_with_single_process_scores():
    # the partitioned (strong-scaling) path: complexes spread over 2 gloo
    # ranks by estimated work, each scored on its rank only, all scores
    # gathered on every rank; equal to one process scoring everything
    import bench
    import numpy as np
    import oracle
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_shard_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    shards = [res[r][0] for r in range(world)]
    assert sorted(shards[0] + shards[1]) == list(range(5)) and not set(shards[0]) & set(shards[1])
    items = _small_items()
    for r in range(world):
        merged = res[r][1]
        assert sorted(merged) == list(range(5))
        assert res[r][2] == sum(len(it["poses"]) for it in _small_items())
        for i, it in enumerate(items):
            ref = oracle.Model(it["family"], it["rec"], it["lig"]).batch_energy_grid(it["poses"], threads=1)
            assert np.array_equal(np.array(merged[i]), ref)
    # the greedy split balances the estimated work within the largest item
    w = [len(it["poses"]) * len(it["lig"]["coords"]) for it in items]
    loads = [sum(w[i] for i in s) for s in shards]
    assert abs(loads[0] - loads[1]) <= max(w)

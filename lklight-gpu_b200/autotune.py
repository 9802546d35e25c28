"""Tile-shape autotuner for the batched scorer.

The warp kernel's shape is four numbers fixed when complexes are added to a
context: ligand atoms per work unit (``tile``), ligand atoms per
candidate-search group (``group``), the receptor cell edge (``cell``, in A)
and the x sub-cells per cell edge (``xsub``).  The best shape depends on the
receptor density and the ligand sizes of the batch, so it is measured: a
sample of the batch's complexes (spread over their size range) is built
once per candidate shape, one launch group over a sample of each complex's
poses is captured in a CUDA graph and replayed, and the fastest shape wins.
Results are cached per device name and batch signature in a JSON file.
"""
import hashlib
import importlib
import json
import os

import numpy as np

CANDIDATES = [
    (128, 8, 4.0, 8), (128, 8, 5.0, 8), (128, 8, 6.0, 8), (128, 8, 7.0, 8),
    (128, 16, 4.0, 8), (128, 16, 5.0, 8), (128, 16, 6.0, 8), (128, 16, 7.0, 8),
    (128, 16, 8.0, 8), (256, 16, 6.0, 8), (256, 16, 7.0, 8), (256, 16, 8.0, 8), (128, 32, 6.0, 8), (256, 32, 7.0, 8),
    (128, 4, 4.0, 8), (64, 8, 4.0, 8), (256, 8, 6.0, 8),
]
DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "lkg", "tuning.json")


def signature(items, device_name):
    """Batch signature: device, then (family, receptor atoms, ligand atoms,
    poses) of every complex: the best shape for 200 poses of a complex is
    not the best for 10,000."""
    h = hashlib.sha1(device_name.encode())
    for it in items:
        n = len(it["poses"]) if "poses" in it else 0
        h.update(("%s:%d:%d:%d;" % (it["family"], len(it["rec"]["coords"]), len(it["lig"]["coords"]), n)).encode())
    return h.hexdigest()


def _sample(items, k):
    """k complexes that stand for the batch's work: a pose's cost grows
    with its ligand's atom count, so the picks sit at evenly spaced
    quantiles of the cumulative ligand atoms (large-ligand complexes, which
    dominate the step, are picked more often than by count)."""
    order = sorted(range(len(items)), key=lambda i: len(items[i]["lig"]["coords"]))
    if len(order) <= k:
        return order
    w = np.cumsum([len(items[i]["lig"]["coords"]) for i in order], dtype=float)
    w /= w[-1]
    picks = []
    for j in range(k):
        q = (j + 0.5) / k
        i = order[int(np.searchsorted(w, q))]
        if i not in picks:
            picks.append(i)
    return picks


def autotune(items, device=0, candidates=CANDIDATES, sample=12, poses_per_complex=3000, reps=3,
             cache_path=DEFAULT_CACHE, verbose=False):
    """Returns dict(tile, group, cell, xsub, ms, source) for a batch given as
    a list of dicts with ``family``, ``rec``, ``lig`` and ``poses`` (N x 7,
    kernel layout).  ``source`` is "cache" or "measured"."""
    import torch
    lkg = importlib.import_module("lklight-gpu_b200")
    name = torch.cuda.get_device_name(device)
    key = signature(items, name)
    cache = {}
    if cache_path and os.path.exists(cache_path):
        try:
            with open(cache_path) as f:
                cache = json.load(f)
        except (OSError, ValueError):
            cache = {}
    if key in cache:
        r = dict(cache[key])
        r["source"] = "cache"
        return r
    pick = _sample(items, sample)
    sub = [items[i] for i in pick]
    counts = [min(poses_per_complex, len(it["poses"])) for it in sub]
    poses = np.vstack([it["poses"][:n] for it, n in zip(sub, counts)])
    with torch.cuda.device(device):
        d_poses = torch.tensor(poses, dtype=torch.float64, device="cuda")
        d_scores = torch.zeros(len(poses), dtype=torch.float64, device="cuda")
        results = []
        for tile, group, cell, xsub in candidates:
            ctx = lkg.Context(device=device, tile=tile, group=group, cell=cell, xsub=xsub)
            try:
                ids = [ctx.add_complex(it["family"], it["rec"], it["lig"]) for it in sub]
                plan = lkg.Plan(ctx, ids, counts)
                plan.capture(d_poses.data_ptr(), d_scores.data_ptr(), n_launches=1)
                stream = torch.cuda.ExternalStream(ctx.stream)
                plan.replay()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(reps):
                    plan.replay()
                e1.record(stream)
                e1.synchronize()
                plan.sync()
                ms = e0.elapsed_time(e1) / reps
                plan.close()
            finally:
                ctx.close()
            results.append((ms, tile, group, cell, xsub))
            if verbose:
                print("autotune tile %d group %d cell %.2f xsub %d: %.3f ms" % (tile, group, cell, xsub, ms), flush=True)
    ms, tile, group, cell, xsub = min(results)
    best = dict(tile=tile, group=group, cell=cell, xsub=xsub, ms=ms, device=name,
                sample=dict(complexes=pick, poses=int(sum(counts))))
    if cache_path:
        cache[key] = best
        os.makedirs(os.path.dirname(cache_path), exist_ok=True)
        tmp = cache_path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1)
        os.replace(tmp, cache_path)
    r = dict(best)
    r["source"] = "measured"
    return r

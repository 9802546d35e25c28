"""Parity at the benchmark's full sizes, through properties that do not need
the oracle to score everything:
* the batched workload (64 complexes, 384,000 poses in one launch group):
  bitwise reproducible, equal to one launch per complex, a sample of poses
  from every complex against the exact path, and samples of the four
  smallest complexes against the oracle (1e-5 relative; the oracle's CPU
  far-field builds for all 64 receptors would take about ten minutes);
* the config-4 cpydock complex (101k-atom receptor, 12k-atom ligand,
  25,000 poses): bitwise reproducible, and a sample against the exact path
  (the oracle's CPU far-field build for this receptor alone takes minutes;
  the exact path is pinned to the oracle on the smaller complexes).
"""
import numpy as np
import pytest

import oracle
from tests.lkg_helpers import config2_items, lkg, rel_err, synth

pytestmark = pytest.mark.gpu

FAST_TOL = 1e-5


def _device_scores(ctx, ids, counts, allp):
    import torch
    d_p = torch.tensor(allp, dtype=torch.float64, device="cuda")
    d_s = torch.zeros(len(allp), dtype=torch.float64, device="cuda")
    ctx.score_multi_device(ids, counts, d_p.data_ptr(), d_s.data_ptr())
    ctx.sync()
    return d_s.cpu().numpy()


def test_batched_workload_full_size():
    items = config2_items()
    ctx = lkg.Context()
    try:
        ids = [ctx.add_complex(it["family"], it["rec"], it["lig"]) for it in items]
        counts = [len(it["poses"]) for it in items]
        allp = np.vstack([it["poses"] for it in items])
        assert len(allp) == 384000
        a = _device_scores(ctx, ids, counts, allp)
        b = _device_scores(ctx, ids, counts, allp)
        assert np.array_equal(a, b)                       # deterministic
        off = np.concatenate([[0], np.cumsum(counts)])
        for k in (0, 17, 31, 32, 50, 63):                 # one launch per complex gives the same bits
            assert np.array_equal(ctx.score(ids[k], items[k]["poses"]), a[off[k]:off[k + 1]])
        rng = np.random.default_rng(5)
        sel = [rng.choice(n, 4, replace=False) for n in counts]
        ctx_x = lkg.Context(precision="exact")
        try:
            xids = [ctx_x.add_complex(it["family"], it["rec"], it["lig"]) for it in items]
            ref = ctx_x.score_multi(xids, [4] * len(items), np.vstack([it["poses"][s] for it, s in zip(items, sel)]))
        finally:
            ctx_x.close()
        got = np.concatenate([a[off[k] + s] for k, s in enumerate(sel)])
        assert rel_err(got, ref).max() < FAST_TOL        # every complex against the exact path
        small = np.argsort([len(it["rec"]["coords"]) for it in items])[:4]
        for k in small:                                   # and the smallest ones against the oracle
            it = items[k]
            o = oracle.Model(it["family"], it["rec"], it["lig"]).batch_energy_grid(it["poses"][sel[k]])
            assert rel_err(a[off[k] + sel[k]], o).max() < FAST_TOL, k
            assert rel_err(ref[4 * k:4 * k + 4], o).max() < 1e-11, k
    finally:
        ctx.close()


def test_cpydock_large_complex_full_size():
    c4 = synth.config4()
    poses = synth.to_kernel_poses(synth.setup_poses(c4["rec"]["coords"], 50, 500, 19))
    ctx = lkg.Context()
    ctx_x = lkg.Context(precision="exact")
    try:
        cid = ctx.add_complex("cpydock", c4["rec"], c4["lig"])
        a = _device_scores(ctx, [cid], [len(poses)], poses)
        b = _device_scores(ctx, [cid], [len(poses)], poses)
        assert np.array_equal(a, b)
        sel = np.random.default_rng(7).choice(len(poses), 48, replace=False)
        ref = ctx_x.score(ctx_x.add_complex("cpydock", c4["rec"], c4["lig"]), poses[sel])
        assert rel_err(a[sel], ref).max() < FAST_TOL
    finally:
        ctx.close()
        ctx_x.close()

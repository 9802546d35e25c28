"""Restraints and membrane in the batch kernels, against the oracle.

The reference scores restraint / membrane runs on its CPU path only
(dna.rs:885-897, 1047-1056 and the other families' supports_batch); here the
kernels collect per-pose interface bits in the near scan and apply the
restraint fractions and the membrane penalty on the device.  The fractions
are counts over counts and must equal the oracle's exactly, except for poses
with a tagged pair within 1e-6 A^2 of the 3.9 A cutoff (the fast path's
transform may differ in the last place); scores follow the plain parity
tolerances (fast 1e-5, exact 1e-11, relative, denominator max(|E|, 1)) times
the restraint factor 1 + pr + pl that multiplies the plain score.
"""
import numpy as np
import pytest

import oracle
from tests.lkg_helpers import (azp_model, azp_residues, config0, config0_cpydock, lkg, random_poses, rel_err,
                               restraint_tags, synth, tagged_border)

pytestmark = pytest.mark.gpu

FAST_TOL = 1e-5
EXACT_TOL = 1e-11
BORDER = 1e-6


def _azp_restraints(seed=11):
    rresid, _, lresid, _ = azp_residues()
    rng = np.random.default_rng(seed)
    ract = rng.choice(rresid.max() + 1, 9, replace=False)
    lact = rng.choice(lresid.max() + 1, 4, replace=False)
    mem = np.sort(rng.choice(len(rresid), 40, replace=False)).astype(np.int32)
    return restraint_tags(rresid, ract), restraint_tags(lresid, lact), mem


def _compare(rec, lig, rr, lr, mem, poses, got, gf, ref, rf, tol):
    rmask = rr >= 0
    rmask[mem] = True
    lmask = lr >= 0
    checked = 0
    for k in range(len(poses)):
        if not np.array_equal(gf[k], rf[k]):
            assert tagged_border(rec["coords"], lig["coords"], poses[k], rmask, lmask) < BORDER, (k, gf[k], rf[k])
            continue
        # s (1 + pr + pl) - pen carries the plain score's error times (1 + pr + pl)
        assert rel_err(got[k], ref[k]) < tol * (1.0 + rf[k, 0] + rf[k, 1]), (k, got[k], ref[k])
        checked += 1
    assert checked >= len(poses) - 2
    assert (rf > 0).any(axis=0).all()   # every term exercised


def _set(ctx, m, cid, rr, lr, mem):
    ctx.set_restraints(cid, rr, lr, mem)
    m.set_restraints(rr, int(rr.max()) + 1, lr, int(lr.max()) + 1, mem)


@pytest.mark.parametrize("exact", [False, True])
@pytest.mark.parametrize("family", ["dna", "pydock", "vdw", "cpydock"])
def test_restraints_1azp_match_oracle(family, exact):
    rec, lig = azp_model(family)
    rr, lr, mem = _azp_restraints()
    m = oracle.Model(family, rec, lig)
    ctx = lkg.Context(precision="exact" if exact else "fast")
    try:
        cid = ctx.add_complex(family, rec, lig)
        _set(ctx, m, cid, rr, lr, mem)
        poses = random_poses(48, [0, 0, 0], 16.0, 21)
        got, gf = ctx.score_interface(cid, poses)
        ref, rf = m.batch_energy_grid_iface(poses)
        _compare(rec, lig, rr, lr, mem, poses, got, gf, ref, rf, EXACT_TOL if exact else FAST_TOL)
        if exact:   # the exact path decides every pair in f64 in the reference's order
            assert np.array_equal(gf, rf)
    finally:
        ctx.close()


def _config0_restraints(c, poses, seed):
    """Restraint residues (blocks of 10 receptor atoms, 30 ligand atoms)
    drawn near the poses, and membrane beads among receptor atoms near them,
    so that every term varies over the poses."""
    rc, lc = c["rec"]["coords"], c["lig"]["coords"]
    rng = np.random.default_rng(seed)
    centre = poses[:, 4:7].mean(axis=0)
    near = np.nonzero(np.linalg.norm(rc - centre, axis=1) < 30.0)[0]
    rres = rc.shape[0] // 10
    ract = rng.choice(np.unique(near // 10), 12, replace=False)
    rr = restraint_tags(np.minimum(np.arange(len(rc)) // 10, rres - 1), ract)
    lres = np.arange(len(lc)) // 30
    lr = restraint_tags(lres, rng.choice(lres.max() + 1, 8, replace=False))
    mem = np.sort(rng.choice(near, 60, replace=False)).astype(np.int32)
    return rr, lr, mem


def _swarm_poses(c, n, seed):
    pos = synth.setup_poses(c["rec"]["coords"], 1, n, seed)
    return np.hstack([pos[:, 3:7], pos[:, 0:3]])


@pytest.mark.parametrize("group", [4, 8, 16, 32])
def test_restraints_config0_warp_groups(group):
    c = config0()
    poses = _swarm_poses(c, 24, 5)
    rr, lr, mem = _config0_restraints(c, poses, 3)
    m = oracle.Model("dna", c["rec"], c["lig"])
    ctx = lkg.Context(group=group)
    try:
        cid = ctx.add_complex("dna", c["rec"], c["lig"])
        _set(ctx, m, cid, rr, lr, mem)
        got, gf = ctx.score_interface(cid, poses)
        ref, rf = m.batch_energy_grid_iface(poses)
        _compare(c["rec"], c["lig"], rr, lr, mem, poses, got, gf, ref, rf, FAST_TOL)
    finally:
        ctx.close()


@pytest.mark.parametrize("group", [8, 16, 32])
def test_restraints_config0_cpydock(group):
    c = config0_cpydock()
    poses = _swarm_poses(c, 16, 7)
    rr, lr, mem = _config0_restraints(c, poses, 4)
    m = oracle.Model("cpydock", c["rec"], c["lig"])
    ctx = lkg.Context(group=group)
    try:
        cid = ctx.add_complex("cpydock", c["rec"], c["lig"])
        _set(ctx, m, cid, rr, lr, mem)
        got, gf = ctx.score_interface(cid, poses)
        ref, rf = m.batch_energy_grid_iface(poses)
        _compare(c["rec"], c["lig"], rr, lr, mem, poses, got, gf, ref, rf, FAST_TOL)
    finally:
        ctx.close()


def test_restrained_and_plain_complexes_in_one_launch():
    rec, lig = azp_model("dna")
    prec, plig = azp_model("pydock")
    rr, lr, mem = _azp_restraints(13)
    m = oracle.Model("dna", rec, lig)
    m.set_restraints(rr, int(rr.max()) + 1, lr, int(lr.max()) + 1, mem)
    mp = oracle.Model("pydock", prec, plig)
    ctx = lkg.Context()
    try:
        a = ctx.add_complex("dna", rec, lig)
        b = ctx.add_complex("pydock", prec, plig)
        ctx.set_restraints(a, rr, lr, mem)
        pa, pb = random_poses(20, [0, 0, 0], 14.0, 1), random_poses(30, [0, 0, 0], 14.0, 2)
        got = ctx.score_multi([a, b], [20, 30], np.vstack([pa, pb]))
        assert rel_err(got[20:], mp.batch_energy_grid(pb)).max() < FAST_TOL
        alone, gf = ctx.score_interface(a, pa)
        assert np.array_equal(got[:20], alone)   # same kernel, per-pose sums in the same order
        ref, rf = m.batch_energy_grid_iface(pa)
        _compare(rec, lig, rr, lr, mem, pa, alone, gf, ref, rf, FAST_TOL)
    finally:
        ctx.close()


def test_clearing_restraints_restores_plain_scores():
    rec, lig = azp_model("pydock")
    rr, lr, mem = _azp_restraints(17)
    ctx = lkg.Context()
    try:
        cid = ctx.add_complex("pydock", rec, lig)
        poses = random_poses(16, [0, 0, 0], 12.0, 4)
        plain = ctx.score(cid, poses)
        ctx.set_restraints(cid, rr, lr, mem)
        restrained = ctx.score(cid, poses)
        assert not np.array_equal(plain, restrained)
        ctx.set_restraints(cid)
        assert np.array_equal(ctx.score(cid, poses), plain)
    finally:
        ctx.close()


def test_plans_made_before_restraints_are_refused():
    import torch
    rec, lig = azp_model("dna")
    rr, lr, mem = _azp_restraints(19)
    ctx = lkg.Context()
    try:
        cid = ctx.add_complex("dna", rec, lig)
        poses = torch.tensor(random_poses(32, [0, 0, 0], 12.0, 6), dtype=torch.float64, device="cuda")
        scores = torch.zeros(32, dtype=torch.float64, device="cuda")
        plan = lkg.Plan(ctx, [cid], [32])
        plan.capture(poses.data_ptr(), scores.data_ptr(), n_launches=1)
        ctx.set_restraints(cid, rr, lr, mem)
        with pytest.raises(lkg.LkgError):
            plan.replay()        # the graph was captured without room for the bits
        with pytest.raises(lkg.LkgError):
            plan.launch(poses.data_ptr(), scores.data_ptr())
        plan.close()
        plan = lkg.Plan(ctx, [cid], [32])   # a plan made now carries them
        plan.capture(poses.data_ptr(), scores.data_ptr(), n_launches=1)
        plan.replay()
        plan.sync()
        want, _ = ctx.score_interface(cid, poses.cpu().numpy())
        assert np.array_equal(scores.cpu().numpy(), want)
        plan.close()
    finally:
        ctx.close()


def test_gso_with_restraints_host_and_device_agree():
    # the GSO drivers score restrained complexes through the same launches:
    # a few device steps follow the host steps (up to the slerp's last place)
    c = config0()
    pos = synth.setup_poses(c["rec"]["coords"], 2, 150, 13)
    rr, lr, mem = _config0_restraints(c, synth.to_kernel_poses(pos), 6)
    ctx = lkg.Context()
    try:
        cid = ctx.add_complex("dna", c["rec"], c["lig"])
        ctx.set_restraints(cid, rr, lr, mem)
        out = []
        for dev in (False, True):
            g = lkg.GSO(ctx, [(cid, 2, 150)], pos, [13])
            g.run(4, device=dev)
            out.append(g.state())
            del g
        a, b = out
        for k in ("translation", "luciferin", "scoring"):
            d = np.abs(a[k] - b[k]) / np.maximum(np.abs(a[k]), 1.0)
            assert d.max() < 1e-9, (k, d.max())
        assert np.array_equal(a["neighbors"], b["neighbors"])
        # and the restraint terms took part: the scores differ from plain ones
        ctx.set_restraints(cid)
        g = lkg.GSO(ctx, [(cid, 2, 150)], pos, [13])
        g.run(1)
        plain = g.state()["scoring"]
        del g
        g = lkg.GSO(ctx, [(cid, 2, 150)], pos, [13])
        ctx.set_restraints(cid, rr, lr, mem)
        g.run(1)
        assert not np.array_equal(g.state()["scoring"], plain)
        del g
    finally:
        ctx.close()

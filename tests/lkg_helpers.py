"""Shared helpers for the lkg tests: package import, model dictionaries and
the parity metric (relative error with denominator max(|E|, 1), as the
reference's own grid-vs-exact test uses it, src/dna.rs:1176)."""
import functools
import importlib
import os
import re

import numpy as np

lkg = importlib.import_module("lklight-gpu_b200")
synth = importlib.import_module("lklight-gpu_b200.synth")
compat = importlib.import_module("lklight-gpu_b200.compat")

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def rel_err(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.abs(a - b) / np.maximum(np.abs(b), 1.0)


def header_symbols():
    """Every function declared in include/lkg.h."""
    with open(os.path.join(REPO, "include", "lkg.h")) as f:
        src = f.read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b((?:cuda|lkg)_\w+)\s*\(", src)))


def random_poses(n, center, spread, seed):
    """n x 7 kernel-layout poses: random unit quaternions, translations
    uniform in center +- spread."""
    rng = np.random.default_rng(seed)
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    t = np.asarray(center, float) + rng.uniform(-spread, spread, size=(n, 3))
    return np.hstack([q, t])


def azp_model(family):
    """1AZP receptor/ligand dicts typed for `family` (golden fixture), with
    cpydock desolvation arrays derived like the synthetic ones."""
    from tests.golden_models import azp
    rec, lig = azp(family)
    if family == "cpydock":
        for m in (rec, lig):
            heavy = 1 - m["is_h"].astype(np.int32)
            m["hyd"] = heavy
            m["des"] = np.where(heavy == 1, 0.02, 0.0)
            m["asa"] = np.where(heavy == 1, 30.0, -1.0)
    return rec, lig


@functools.lru_cache(maxsize=2)
def config0():
    return synth.config0()


@functools.lru_cache(maxsize=1)
def config2_items():
    """The batched workload: 64 complexes (dna, then pydock) with their
    20 x 300 kernel-layout poses each (seed 11)."""
    items = synth.config2()
    for it in items:
        it["poses"] = synth.to_kernel_poses(synth.setup_poses(it["rec"]["coords"], it["swarms"], it["glowworms"],
                                                              it["seed"]))
    return items


@functools.lru_cache(maxsize=2)
def config0_cpydock():
    return synth.config1("cpydock", base=config0())


def azp_residues():
    """Per-atom residue index and residue ids ("chain.resname.serial") of the
    1AZP receptor and ligand (golden fixture)."""
    from tests.golden_models import GOLDEN
    d = np.load(os.path.join(GOLDEN, "1azp_models.npz"))
    return d["rec_resid"], d["rec_residues"], d["lig_resid"], d["lig_residues"]


def restraint_tags(resid, active):
    """Per-atom restraint residue index (position in `active`, -1 = none) for
    atoms whose residue index is in `active`: the flattened form of the
    reference's active_restraints map."""
    pos = {int(r): k for k, r in enumerate(active)}
    return np.array([pos.get(int(r), -1) for r in resid], np.int32)


def pose_matrix(p):
    """Rotation of kernel-layout pose p (w, x, y, z, ...): qt.rs:67-74."""
    w, x, y, z = p[:4]
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def brute_interface(rec_c, lig_c, pose, cutoff=3.9):
    """Interface flags of one pose by all pairs (f64): receptor flags,
    ligand flags and the smallest |d^2 - cutoff^2| (pairs that close to the
    cutoff can flip with last-place rounding of the transform)."""
    L = lig_c @ pose_matrix(pose).T + np.asarray(pose[4:7])
    d2 = ((L[:, None, :] - rec_c[None, :, :]) ** 2).sum(-1)
    hit = d2 <= cutoff * cutoff
    return hit.any(axis=0), hit.any(axis=1), float(np.abs(d2 - cutoff * cutoff).min())


def combine_restraints(family, s, pr, pl, m):
    """Restraint fractions and membrane penalty applied to score s in the
    family's operation order (dna.rs:989-995, pydock.rs:440-445,
    vdw.rs:146-149, cpydock.rs:670-675)."""
    pen = 999.0 * m if m > 0.0 else 0.0
    if family == "dna":
        return s + ((pr * s + pl * s) - pen)
    if family == "vdw":
        return s + pr * s + pl * s
    return s + pr * s + pl * s - pen


def tagged_border(rec_c, lig_c, pose, rmask, lmask, cutoff=3.9):
    """Smallest |d^2 - cutoff^2| over the pairs that involve a tagged atom
    (receptor atoms where rmask, ligand atoms where lmask): only those
    pairs move a restraint fraction or the membrane count."""
    L = lig_c @ pose_matrix(pose).T + np.asarray(pose[4:7])
    c2 = cutoff * cutoff
    best = np.inf
    if rmask.any():
        d2 = ((L[:, None, :] - rec_c[rmask][None, :, :]) ** 2).sum(-1)
        best = min(best, float(np.abs(d2 - c2).min()))
    if lmask.any():
        d2 = ((L[lmask][:, None, :] - rec_c[None, :, :]) ** 2).sum(-1)
        best = min(best, float(np.abs(d2 - c2).min()))
    return best

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


@functools.lru_cache(maxsize=2)
def config0_cpydock():
    return synth.config1("cpydock", base=config0())

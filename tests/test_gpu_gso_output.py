"""GSO output files: lkg_gso_save writes each swarm as gso_<step>.out in the
reference's format (swarm.rs:232-271), restated here with Python's
correctly rounded fixed-point formatting (Rust's {:.N} rounds the same
way), and the ranking lists read them back (lightdock.rs:123-148,863-903)."""
import importlib

import numpy as np
import pytest

from tests.lkg_helpers import config0, lkg, synth

pytestmark = pytest.mark.gpu

SWARMS, GLOW, STEPS = 2, 60, 3


def _expected(st, rows):
    out = ["#Coordinates  RecID  LigID  Luciferin  Neighbor's number  Vision Range  Scoring\n"]
    for i in rows:
        v = list(st["translation"][i]) + list(st["rotation"][i])
        out.append("(" + ", ".join("%.7f" % x for x in v) + ")    0    0   %.8f  %d %.3f %.8f\n" % (
            st["luciferin"][i], st["neighbors"][i], st["vision"][i], st["scoring"][i]))
    return "".join(out)


def test_gso_files_and_rankings(tmp_path):
    rank = importlib.import_module("lklight-gpu_b200.rank")
    c0 = config0()
    ctx = lkg.Context()
    try:
        cid = ctx.add_complex("dna", c0["rec"], c0["lig"])
        pos = synth.setup_poses(c0["rec"]["coords"], SWARMS, GLOW, 9)
        g = lkg.GSO(ctx, [(cid, SWARMS, GLOW)], pos, [9])
        g.run(STEPS)
        st = g.state()
        for sw in range(SWARMS):
            d = tmp_path / ("swarm_%d" % sw)
            d.mkdir()
            g.save(sw, STEPS, str(d))
            text = (d / ("gso_%d.out" % STEPS)).read_text()
            assert text == _expected(st, range(sw * GLOW, (sw + 1) * GLOW))
        with pytest.raises(lkg.LkgError):
            g.save(SWARMS, STEPS, str(tmp_path))
        del g
    finally:
        ctx.close()
    ranked = rank.rank(SWARMS, STEPS, str(tmp_path))
    assert len(ranked) == SWARMS * GLOW
    best = int(np.argmax(st["scoring"]))
    assert (ranked[0]["swarm"], ranked[0]["glowworm"]) == (best // GLOW, best % GLOW)
    assert abs(ranked[0]["scoring"] - st["scoring"][best]) <= 5e-9

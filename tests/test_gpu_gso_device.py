"""Device-resident GSO steps against the host GSO (the reference GSO).

Both run the same plain GSO from the same start.  The device path draws the
swarms' StdRng streams on the GPU and does the f64 arithmetic of the host
path without FMA contraction; only the slerp's acos / sin come from another
math library (last-place differences), so a few steps agree to ~1e-9 and the
neighbour counts exactly.  Switching between the two in one run keeps the
random streams aligned.
"""
import numpy as np
import pytest

from tests.lkg_helpers import config0, lkg, synth

pytestmark = pytest.mark.gpu

SWARMS, GLOW = 3, 200


@pytest.fixture(scope="module")
def setup():
    c0 = config0()
    ctx = lkg.Context()
    cid = ctx.add_complex("dna", c0["rec"], c0["lig"])
    pos = synth.setup_poses(c0["rec"]["coords"], SWARMS, GLOW, 17)
    yield ctx, cid, pos
    ctx.close()


def _run(setup, plan):
    ctx, cid, pos = setup
    g = lkg.GSO(ctx, [(cid, SWARMS, GLOW)], pos, [17])
    for steps, dev in plan:
        g.run(steps, device=dev)
    st = g.state()
    st["scored"] = g.scored
    del g
    return st


def _close(a, b, tol):
    for k in ("translation", "rotation", "luciferin", "scoring", "vision"):
        d = np.abs(a[k] - b[k]) / np.maximum(np.abs(b[k]), 1.0)
        assert d.max() < tol, (k, d.max())
    assert np.array_equal(a["neighbors"], b["neighbors"])


def test_device_steps_match_host_steps(setup):
    host = _run(setup, [(4, False)])
    dev = _run(setup, [(4, True)])
    _close(dev, host, 1e-9)


def test_switching_between_host_and_device_keeps_the_random_streams(setup):
    host = _run(setup, [(5, False)])
    mixed = _run(setup, [(2, False), (2, True), (1, False)])
    _close(mixed, host, 1e-9)


def test_device_run_is_reproducible(setup):
    a = _run(setup, [(12, True)])
    b = _run(setup, [(12, True)])
    for k in ("translation", "rotation", "luciferin", "scoring"):
        assert np.array_equal(a[k], b[k])

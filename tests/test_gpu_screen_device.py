"""Device-resident screened GSO against the host screened GSO.

The device run does whole GSO steps on the GPU: the training steps (plain
steps whose exact pairs train the surrogate), then screened steps with K
selections per glowworm from the swarm's stream, candidate poses, surrogate
predictions, the per-swarm choice of the moves scored exactly, the move, and
a full rescoring with fine-tuning every `rescore_every` steps.  Training is bitwise reproducible (fixed-order
reductions), so host screened runs repeat exactly; the device run agrees
with the host run up to the slerp's acos / sin (device library vs glibc):
a last-place difference in a candidate pose can move a BF16 feature and
flip a choice, so agreement is checked per glowworm over a few steps.
"""
import numpy as np
import pytest

from tests.lkg_helpers import config0, lkg, synth

pytestmark = pytest.mark.gpu

SWARMS, GLOW, SEED = 3, 240, 11
SCREEN = dict(candidates=4, exact_fraction=0.25, rescore_every=3, train_steps=4, train_epochs=10, finetune_epochs=1,
              lr=1e-3, seed=7, batch=256)


@pytest.fixture(scope="module")
def setup():
    c0 = config0()
    ctx = lkg.Context()
    cid = ctx.add_complex("dna", c0["rec"], c0["lig"])
    pos = synth.setup_poses(c0["rec"]["coords"], SWARMS, GLOW, SEED)
    yield ctx, cid, pos
    ctx.close()


def _run(setup, plan, **extra):
    ctx, cid, pos = setup
    g = lkg.GSO(ctx, [(cid, SWARMS, GLOW)], pos, [SEED])
    g.set_screen(**SCREEN, **extra)
    for steps, dev in plan:
        g.run(steps, device=dev)
    st = g.state()
    st["scored"], st["predicted"] = g.scored, g.predicted
    del g
    return st


def test_host_screened_runs_repeat_exactly(setup):
    a = _run(setup, [(9, False)])
    b = _run(setup, [(9, False)])
    for k in ("translation", "rotation", "luciferin", "scoring", "vision"):
        assert np.array_equal(a[k], b[k]), k
    assert a["scored"] == b["scored"]


@pytest.mark.parametrize("carry", [False, True])
@pytest.mark.parametrize("plan", [[(9, True)], [(4, False), (5, True)]])
def test_device_screened_steps_follow_the_host(setup, plan, carry):
    # all on the device (training steps 0-3 too), or the training steps on
    # the host; a full rescoring at step 7 in both; unscored moves keep
    # their last exact score, or (carry) take the predicted gain
    host = _run(setup, [(9, False)], carry_prediction=carry)
    dev = _run(setup, plan, carry_prediction=carry)
    close = np.all(np.abs(dev["translation"] - host["translation"]) <= 1e-6 * np.maximum(1.0, np.abs(host["translation"])),
                   axis=1)
    assert close.mean() >= 0.9, close.mean()
    both = close & (np.abs(host["scoring"]) > 0)
    rel = np.abs(dev["scoring"][both] - host["scoring"][both]) / np.maximum(1.0, np.abs(host["scoring"][both]))
    assert np.median(rel) < 1e-6
    assert abs(dev["scored"] - host["scored"]) <= 0.02 * host["scored"]


def test_device_screened_run_is_reproducible_and_mixable(setup):
    a = _run(setup, [(10, True)])
    b = _run(setup, [(10, True)])
    for k in ("translation", "rotation", "luciferin", "scoring"):
        assert np.array_equal(a[k], b[k]), k
    mixed = _run(setup, [(6, True), (2, False), (2, True)])   # host and device steps share the state
    assert np.isfinite(mixed["scoring"]).all()
    assert mixed["scored"] < 0.7 * SWARMS * GLOW * 10


def test_device_screening_refuses_the_ablation(setup):
    ctx, cid, pos = setup
    g = lkg.GSO(ctx, [(cid, SWARMS, GLOW)], pos, [SEED])
    g.set_screen(**dict(SCREEN, random_rank=True))
    g.run(4)
    with pytest.raises(lkg.LkgError):
        g.run(1, device=True)
    del g

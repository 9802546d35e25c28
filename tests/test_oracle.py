"""Pins the oracle against the reference's own known-answer tests.

Each test restates one reference test (file:line cited) on the committed
1AZP fixture; the oracle is trusted by the GPU parity tests only because
these pass.
"""
import numpy as np
import pytest

import oracle
from tests.golden_models import azp

ID = [1.0, 0.0, 0.0, 0.0]


def model(family):
    rec, lig = azp(family)
    if family == "cpydock":
        for m in (rec, lig):
            heavy = 1 - m["is_h"].astype(np.int32)
            m["hyd"] = heavy
            m["des"] = np.where(heavy == 1, 0.02, 0.0)
            m["asa"] = np.where(heavy == 1, 30.0, -1.0)
    return oracle.Model(family, rec, lig)


def test_random_quaternion_kat():
    # src/qt.rs:474-488: seed_from_u64(324324324) -> Quaternion::random
    q = oracle.Rng(324324324).quat()
    exp = [0.31924330894562036, -0.5980633213833059, 0.5444724265858514, 0.49391674399349367]
    assert np.all(np.abs(q - exp) < 2.3e-16)


def test_slerp_kats():
    # src/qt.rs:424-471
    e0 = [0.4472135954999579, 0.0, 0.0, 0.8944271909999159]
    e1 = [0.50709255283711, -0.1690308509457033, 0.6761234037828132, 0.50709255283711]
    assert np.all(np.abs(oracle.slerp([1, 0, 0, 2], [3, -1, 4, 3], 0.0) - e0) < 2.3e-16)
    assert np.all(np.abs(oracle.slerp([1, 0, 0, 2], [3, -1, 4, 3], 1.0) - e1) < 2.3e-16)
    h = 0.7071067811865475
    assert np.all(np.abs(oracle.slerp([1, 0, 0, 0], [0, 0, 1, 0], 0.5) - [h, 0, h, 0]) < 2.3e-16)
    assert np.all(np.abs(oracle.slerp([h, 0, 0, h], [0, h, h, 0], 0.5) - [0.5] * 4) < 2.3e-16)
    s = 0.7071067811865476
    assert np.all(oracle.slerp([s, 0, 0, s], [s, 0, 0, s], 0.1) == [s, 0, 0, s])


def test_field_unit_charge():
    # src/grid_dna.rs:217-233
    f = oracle.Field(np.zeros((1, 3)), np.ones(1))
    at12, atn12 = f.sample(12, 0, 0), f.sample(-12, 0, 0)
    assert abs(at12 - atn12) < 1e-6
    assert abs(at12 - 1 / 144) < 1e-4
    assert abs(f.sample(5, 0, 0)) < 1e-9
    assert abs(f.sample(28, 0, 0) - 1 / 784) < 1e-5
    assert abs(f.sample(35, 0, 0)) < 1e-9


@pytest.mark.parametrize("fp64", [False, True])
def test_field_brick_order_equals_atom_scatter(fp64):
    # grid_dna.rs:71-149 scatters atom by atom; the oracle builds the grid in
    # parallel bricks (and AVX2 rows where the host has them) that keep each
    # point's atom order: the bits must equal the plain scalar scatter
    import importlib
    synth = importlib.import_module("lklight-gpu_b200.synth")
    rec, _ = azp("dna")
    glob = synth.globule(1200, 31)
    for c, q in ((rec["coords"], rec["ele"]), (glob["coords"], glob["ele"])):
        a = oracle.Field(c, q, fp64=fp64)
        b = oracle.Field(c, q, fp64=fp64, scatter=True)
        view = np.uint64 if fp64 else np.uint32
        assert np.array_equal(a.dims, b.dims) and np.array_equal(a.origin, b.origin)
        assert np.array_equal(a.phi.view(view), b.phi.view(view))


def test_lr_sasa_analytic_spheres():
    # Lee & Richards (src/lr_sasa.rs, probe 1.4 A, 20 slices): an isolated
    # sphere's slices sum to 4 pi R^2 exactly; two overlapping spheres side
    # by side (slices cut both) approach the analytic exposed areas
    # 4 pi R^2 - 2 pi R h (h: height of the cap inside the other sphere)
    # within the 20-slice discretisation; a sphere inside another is buried
    a = oracle.lr_sasa(np.zeros((1, 3)), [1.6])
    assert abs(a[0] - 4 * np.pi * 3.0 ** 2) < 1e-9
    for r1, r2, d in ((1.6, 1.9, 3.0), (1.8, 1.8, 4.5), (1.4, 2.0, 2.2)):
        got = oracle.lr_sasa(np.array([[0.0, 0, 0], [d, 0, 0]]), [r1, r2])
        p1, p2 = r1 + 1.4, r2 + 1.4
        h1 = p1 - (d * d + p1 * p1 - p2 * p2) / (2 * d)
        h2 = p2 - (d * d + p2 * p2 - p1 * p1) / (2 * d)
        exact = [4 * np.pi * p1 * p1 - 2 * np.pi * p1 * h1, 4 * np.pi * p2 * p2 - 2 * np.pi * p2 * h2]
        assert np.all(np.abs(got - exact) / exact < 0.01)
    b = oracle.lr_sasa(np.array([[0.0, 0, 0], [0.1, 0, 0]]), [0.5, 4.0])
    assert b[0] == 0.0 and b[1] > 0


def test_nearcell_matches_allpairs():
    # src/nearcell.rs:120-160: xorshift coordinates, 300 atoms, cell 5
    state = 7
    vals = []
    for _ in range(900):
        state ^= (state << 13) & 0xFFFFFFFFFFFFFFFF
        state ^= state >> 7
        state ^= (state << 17) & 0xFFFFFFFFFFFFFFFF
        vals.append((state % 200) / 10.0 - 10.0)
    c = np.array(vals).reshape(300, 3)
    assert oracle.lib().orc_nearcell_pair_count(oracle._p(c), 300, 5.0) == \
        oracle.lib().orc_allpairs_count(oracle._p(c), 300, 5.0)


def test_pydock_1azp_exact():
    # src/pydock.rs:546-594
    m = model("pydock")
    exact0 = m.energy_exact([0, 0, 0], ID)
    assert abs(exact0 - (-364.88126358158974)) < 1e-8
    g = m.energy_grid([0, 0, 0], ID)
    assert abs(g - exact0) / abs(exact0) < 0.05
    for t in ([2, 0, 0], [0, 3, 0], [-4, 2, 5], [1, -2, 6]):
        g, e = m.energy_grid(t, ID), m.energy_exact(t, ID)
        r = abs(g - e) / abs(e) if abs(e) > 1 else abs(g - e)
        assert r < 0.05


def test_dna_1azp_grid():
    # src/dna.rs:1113-1152: the pinned value is the grid path's own output;
    # the restatement reproduces it bit for bit.
    m = model("dna")
    assert m.energy_grid([0, 0, 0], ID) == -1211.6718762645426


def test_dna_1azp_grid_matches_exact():
    # src/dna.rs:1155-1179
    m = model("dna")
    for t in ([0, 0, 0], [1, 2, 3], [-2, 1, -4], [5, -3, 2]):
        e, g = m.energy_exact(t, ID), m.energy_grid(t, ID)
        assert abs(e - g) / max(abs(e), 1.0) < 0.02


def test_vdw_1azp_grid_equals_exact():
    # src/vdw.rs:351-378
    m = model("vdw")
    for t in ([0, 0, 0], [2, 0, 0], [0, 3, 0], [-4, 2, 5], [1, -2, 6]):
        assert abs(m.energy_grid(t, ID) - m.energy_exact(t, ID)) < 1e-9


def test_cpydock_1azp_grid_matches_exact():
    # src/cpydock.rs:861-876
    m = model("cpydock")
    for t in ([0, 0, 0], [2, 3, 1], [-4, 5, 2], [0, -6, 8], [3, 3, -3]):
        assert abs(m.energy_grid(t, ID) - m.energy_exact(t, ID)) < 12.0


def test_fp64_variant_close_to_f32_field():
    m = model("pydock")
    for t in ([0, 0, 0], [3, -2, 4]):
        a, b = m.energy_grid(t, ID), m.energy_grid(t, ID, fp64=True)
        assert abs(a - b) / abs(a) < 1e-4


@pytest.mark.parametrize("family", ["dna", "pydock", "vdw", "cpydock"])
def test_batch_matches_single(family):
    m = model(family)
    rng = np.random.default_rng(5)
    poses = np.zeros((6, 7))
    q = rng.normal(size=(6, 4))
    poses[:, :4] = q / np.linalg.norm(q, axis=1, keepdims=True)
    poses[:, 4:] = rng.uniform(-4, 4, size=(6, 3))
    b = m.batch_energy_grid(poses)
    for k in range(6):
        assert b[k] == m.energy_grid(poses[k, 4:], poses[k, :4])


def test_gso_deterministic():
    m = model("dna")
    rng = oracle.Rng(42)
    pos = np.array([[rng.f64() * 2 - 1 + 20, rng.f64() * 2 - 1, rng.f64() * 2 - 1] + list(rng.quat())
                    for _ in range(20)])
    runs = []
    for _ in range(2):
        g = oracle.GSO(m, pos, 42)
        g.run(5)
        runs.append(g.state())
    assert np.array_equal(runs[0]["scoring"], runs[1]["scoring"])
    assert np.array_equal(runs[0]["translation"], runs[1]["translation"])


@pytest.mark.parametrize("family", ["dna", "pydock", "vdw", "cpydock"])
def test_restraints_match_all_pairs_interface(family):
    """Interface flags collected in the near scan (dna.rs:970-973 and the
    other families' grid paths) against an all-pairs numpy scan, and the
    restraint / membrane combination against a restatement in Python
    floats (scoring.rs:83-108)."""
    from tests.lkg_helpers import azp_residues, brute_interface, combine_restraints, restraint_tags
    rec, lig = azp(family)
    rresid, _, lresid, _ = azp_residues()
    base, m = model(family), model(family)
    rng = np.random.default_rng(11)
    ract = rng.choice(rresid.max() + 1, 9, replace=False)
    lact = rng.choice(lresid.max() + 1, 4, replace=False)
    rr, lr = restraint_tags(rresid, ract), restraint_tags(lresid, lact)
    mem = np.sort(rng.choice(len(rresid), 40, replace=False)).astype(np.int32)
    m.set_restraints(rr, len(ract), lr, len(lact), mem)
    poses = np.zeros((12, 7))
    q = rng.normal(size=(12, 4))
    poses[:, :4] = q / np.linalg.norm(q, axis=1, keepdims=True)
    poses[:, 4:] = rng.uniform(-18, 18, size=(12, 3))
    got, frac = m.batch_energy_grid_iface(poses)
    plain = base.batch_energy_grid(poses)
    seen = np.zeros(3)
    for k in range(len(poses)):
        ir, il, border = brute_interface(rec["coords"], lig["coords"], poses[k])
        if border < 1e-9:
            continue
        pr = len({int(rr[i]) for i in np.nonzero(ir)[0] if rr[i] >= 0}) / len(ract)
        pl = len({int(lr[j]) for j in np.nonzero(il)[0] if lr[j] >= 0}) / len(lact)
        mi = float(ir[mem].sum()) / len(mem)
        assert (frac[k] == [pr, pl, mi]).all(), (k, frac[k], (pr, pl, mi))
        assert got[k] == combine_restraints(family, plain[k], pr, pl, mi)
        seen += np.array([pr, pl, mi]) > 0
    assert (seen > 0).all()   # every term was exercised


def test_restraints_cleared_score_equals_plain():
    from tests.lkg_helpers import azp_residues
    m, base = model("pydock"), model("pydock")
    rresid = azp_residues()[0]
    m.set_restraints(np.zeros(len(rresid), np.int32), 1, None, 0, None)
    m.set_restraints(None, 0, None, 0, None)
    poses = np.array([[1, 0, 0, 0, 3.0, -2.0, 1.0], [0.6, 0.8, 0, 0, -5.0, 4.0, 2.0]])
    assert (m.batch_energy_grid(poses) == base.batch_energy_grid(poses)).all()

"""CPU-side tests of the product library: it loads, exports every symbol
include/lkg.h declares, and its host logic (RNG, setup poses, cell-list
packing, field geometry, SASA, synthetic inputs) behaves; no GPU calls."""
import ctypes
import importlib

import numpy as np
import pytest

import oracle
from tests.lkg_helpers import compat, header_symbols, lkg, synth


def test_library_exports_header_symbols():
    lib = ctypes.CDLL(lkg.LIB_PATH)
    syms = header_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_status_strings_and_no_device_error():
    L = lkg.lib()
    assert L.lkg_status_string(0) == b"ok"
    assert L.lkg_status_string(6) == b"device capacity exceeded"
    if not lkg.device_available():
        with pytest.raises(lkg.LkgError) as e:
            lkg.Context()
        assert e.value.status == 7


def test_product_rng_matches_reference_kat():
    # src/qt.rs:474-488 through the product's StdRng
    r = lkg.Rng(324324324)
    u1, u2, u3 = r.f64(), r.f64(), r.f64()
    q = [np.sqrt(1 - u1) * np.sin(2 * np.pi * u2), np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
         np.sqrt(u1) * np.sin(2 * np.pi * u3), np.sqrt(u1) * np.cos(2 * np.pi * u3)]
    exp = [0.31924330894562036, -0.5980633213833059, 0.5444724265858514, 0.49391674399349367]
    assert np.all(np.abs(np.array(q) - exp) < 2.3e-16)


def test_product_rng_matches_oracle_stream():
    a, b = lkg.Rng(42), oracle.Rng(42)
    assert [a.f64() for _ in range(1000)] == [b.f64() for _ in range(1000)]


def test_setup_poses_are_unit_quaternions_near_sphere():
    c = synth.globule(800, 3)["coords"]
    pos = synth.setup_poses(c, 3, 10, 5)
    assert pos.shape == (30, 7)
    assert np.allclose(np.linalg.norm(pos[:, 3:], axis=1), 1.0, atol=5e-6)
    avg_r = np.mean(np.linalg.norm(c, axis=1))
    r = np.linalg.norm(pos[:, :3], axis=1)
    assert np.all(np.abs(r - (avg_r + 3.0)) < 1.8)
    assert np.array_equal(pos, synth.setup_poses(c, 3, 10, 5))


def test_compat_cell_list_packing_matches_oracle():
    c = synth.globule(1500, 9)["coords"]
    cr = compat.CudaReceptor(c, np.zeros(len(c)), np.ones(len(c)), np.ones(len(c)))
    o = oracle.crec_build(c)
    assert np.array_equal(cr.cell_start, o["cell_start"])
    assert np.array_equal(cr.cell_atoms, o["cell_atoms"])
    assert [cr.ncx, cr.ncy, cr.ncz] == list(o["nc"])
    assert np.allclose(cr.c_o, o["origin"])


def test_field_geometry_matches_oracle():
    g = synth.globule(700, 4)
    L = lkg.lib()
    o, d, s = np.zeros(3), np.zeros(3, np.int32), ctypes.c_double()
    c = np.ascontiguousarray(g["coords"])
    q = np.ascontiguousarray(g["ele"])
    assert L.lkg_field_build(lkg.ptr(c), lkg.ptr(q), len(q), lkg.ptr(o), lkg.ptr(d), ctypes.byref(s), None) == 0
    f = oracle.Field(np.zeros((2, 3)) + c[:2], q[:2])  # geometry only depends on the bbox
    f2 = oracle.Field(c, np.zeros(len(q)))
    assert np.array_equal(d, f2.dims) and np.array_equal(o, f2.origin) and s.value == f2.spacing
    del f


def test_lr_sasa_isolated_and_buried():
    # one isolated sphere: 4 pi (r + 1.4)^2 up to slice discretisation
    a = lkg.lr_sasa(np.zeros((1, 3)), np.array([1.6]))
    assert abs(a[0] - 4 * np.pi * 3.0 ** 2) / (4 * np.pi * 9.0) < 0.02
    # a sphere inside a larger one is fully buried
    b = lkg.lr_sasa(np.array([[0, 0, 0], [0.1, 0, 0]]), np.array([0.5, 4.0]))
    assert b[0] == 0.0 and b[1] > 0


def test_lr_sasa_equals_the_oracle_restatement():
    # liblkg's Lee & Richards areas (the cpydock reference ASA) against the
    # oracle's own restatement of src/lr_sasa.rs, atom by atom: the 1AZP
    # heavy atoms, the config-0 duplex ligand and a 3000-atom globule with
    # the radius_per_asp radii cpydock uses (cpydock.rs:59-70, 269-332)
    from tests.golden_models import azp
    rec, _ = azp("pydock")
    heavy = rec["is_h"] == 0
    cases = [(rec["coords"][heavy], rec["radius"][heavy])]
    for m in (synth.duplex(20, 42), synth.globule(3000, 5)):
        h = np.asarray(m["heavy"]).astype(bool)
        cases.append((np.asarray(m["coords"])[h], np.array([synth._RASP.get(t, 0.0)
                                                            for t, k in zip(m["types"], h) if k])))
    for c, r in cases:
        assert np.array_equal(lkg.lr_sasa(c, r), oracle.lr_sasa(c, r))
    # and the cpydock side arrays synth builds from them (hydrogens get -1)
    lig = synth.duplex(6, 3)
    cp = synth.add_cpydock(lig)
    h = np.asarray(lig["heavy"]).astype(bool)
    ref = np.full(len(h), -1.0)
    ref[h] = oracle.lr_sasa(np.asarray(lig["coords"])[h],
                            np.array([synth._RASP.get(t, 0.0) for t, k in zip(lig["types"], h) if k]))
    assert np.array_equal(cp["asa"], ref)


def test_synthetic_config0_shape_and_charges():
    c0 = synth.config0()
    rec, lig = c0["rec"], c0["lig"]
    assert len(rec["coords"]) == 12625
    assert 1100 <= len(lig["coords"]) <= 1400
    assert abs(rec["ele"].sum() - 10.0) < 1e-9
    assert np.ptp(rec["ele"]) <= 1.6 and np.all(np.abs(rec["ele"]) <= 0.81)
    assert (lig["ele"] == -1.0).sum() == 40 and np.all((lig["ele"] == 0) | (lig["ele"] == -1))
    assert np.array_equal(rec["coords"], rec["coords"].astype(np.float32).astype(np.float64))
    assert rec["chain_radius"] >= 30.0
    # nonbonded spacing: atoms more than two bonds apart stay >= 3.0 A apart
    c = rec["coords"]
    d = np.linalg.norm(c[3:200, None, :] - c[None, :1000, :], axis=2)
    i, j = np.nonzero(d < 2.99)
    assert np.all(np.abs((i + 3) - j) <= 2)
    c0b = synth.config0()
    assert np.array_equal(c0b["rec"]["coords"], rec["coords"])


def test_reference_arm_generators_equal_the_library_ones():
    # the benchmark's CPU reference arm makes its inputs with the oracle's
    # chain and StdRng instead of liblkg's: the same bits, including a chain
    # long enough to grow its confining radius (config 0: 30 -> 58 A)
    for n, seed, r0 in ((2000, 5, 30.0), (12625, 42, 30.0), (800, 11003, 12.0)):
        a, ra = synth.chain(n, seed, r0=r0)
        b, rb = synth.chain(n, seed, r0=r0, gen=oracle.Generators)
        assert ra == rb and np.array_equal(a.view(np.uint64), b.view(np.uint64))
    c = np.random.default_rng(0).normal(size=(100, 3)) * 20
    assert np.array_equal(synth.setup_poses(c, 3, 10, 7), synth.setup_poses(c, 3, 10, 7, gen=oracle.Generators))


def test_cpy_flag_matches_reference_view():
    hyd = np.array([1, 0, 1, 1, 0, 0, 1])
    f = compat.cpy_flag(hyd)
    # flag(i) = i even and hyd[i // 2] != 0
    exp = [1 if (i % 2 == 0 and hyd[i // 2] != 0) else 0 for i in range(len(hyd))]
    assert list(f) == exp


# ---------------------------------------------------------------- surrogate oracle
def test_mlp_oracle_gradient_matches_finite_differences():
    from oracle import mlp as omlp
    rng = np.random.default_rng(0)
    p = omlp.he_params(1)
    X = rng.normal(size=(16, omlp.IN))
    t = rng.normal(size=16)
    loss, g, _ = omlp.loss_and_grad(p, X, t, emulate=False)
    offs = np.concatenate([[0], np.cumsum(omlp.SIZES)])
    h = 1e-6
    for k in range(8):
        for i in rng.integers(offs[k], offs[k + 1], size=3):
            pp, pm = p.copy(), p.copy()
            pp[i] += h
            pm[i] -= h
            fd = (omlp.loss_and_grad(pp, X, t, emulate=False)[0] - omlp.loss_and_grad(pm, X, t, emulate=False)[0]) / (2 * h)
            assert abs(fd - g[i]) <= 1e-6 * (1.0 + abs(g[i])), (k, i, fd, g[i])


def test_mlp_oracle_bf16_rounding():
    from oracle import mlp as omlp
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 0.0, 65504.0])
    r = omlp.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0          # tie -> even
    assert r[2] == 1.0078125                     # above the tie -> up
    assert abs(r[3] + 3.140625) < 1e-12
    bits = omlp.f64_to_bf16_bits(x)
    assert np.array_equal(omlp.bf16_bits_to_f64(bits), r)


# ------------------------------------------------- gso files and rankings
GSO_TEXT = (
    "#Coordinates  RecID  LigID  Luciferin  Neighbor's number  Vision Range  Scoring\n"
    "(1.0000000, -2.5000000, 3.1250000, 0.5000000, 0.5000000, -0.5000000, 0.5000000)    0    0   "
    "7.12345678  2 0.280 -12.50000000\n"
    "(4.0000000, 5.0000000, 6.0000000, 1.0000000, 0.0000000, 0.0000000, 0.0000000)    0    0   "
    "9.00000000  0 0.200 31.25000000\n"
    "not a pose line\n"
    "(7.0000000, 8.0000000, 9.0000000, 1.0000000, 0.0000000, 0.0000000, 0.0000000, 0.1000000)    0    0   "
    "1.50000000  5 5.000 3.00000000\n")


def test_parse_gso_follows_the_reference_reader(tmp_path):
    # parse_gso_file (src/bin/lightdock.rs:123-148): ids count every non-comment line
    rank = importlib.import_module("lklight-gpu_b200.rank")
    p = tmp_path / "gso_3.out"
    p.write_text(GSO_TEXT)
    e = rank.parse_gso(str(p))
    assert [x["glowworm"] for x in e] == [0, 1, 3]
    assert e[0]["translation"] == [1.0, -2.5, 3.125] and e[0]["rotation"] == [0.5, 0.5, -0.5, 0.5]
    assert e[0]["luciferin"] == 7.12345678 and e[0]["scoring"] == -12.5
    assert e[2]["extents"] == [0.1]


def test_rank_lists_in_the_reference_format(tmp_path):
    # write_rank_file (src/bin/lightdock.rs:888-903)
    rank = importlib.import_module("lklight-gpu_b200.rank")
    for sid in range(2):
        (tmp_path / ("swarm_%d" % sid)).mkdir()
        (tmp_path / ("swarm_%d" % sid) / "gso_3.out").write_text(GSO_TEXT)
    ranked = rank.rank(2, 3, str(tmp_path))
    lines = (tmp_path / "ranking.list").read_text().split("\n")
    assert lines[0] == "# Rank Swarm Glowworm Luciferin Scoring PDB Coords"
    assert lines[1] == "    1    0     1     9.000000    31.250000 swarm_0/lightdock_1.pdb (4.000,5.000,6.000)"
    assert lines[2] == "    2    1     1     9.000000    31.250000 swarm_1/lightdock_1.pdb (4.000,5.000,6.000)"
    assert lines[6] == "    6    1     0     7.123457   -12.500000 swarm_1/lightdock_0.pdb (1.000,-2.500,3.125)"
    assert [r["luciferin"] for r in ranked] == [9.0, 9.0, 7.12345678, 7.12345678, 1.5, 1.5]


def test_bench_tile_shape_without_the_autotuner():
    # a shape on the command line is used as given; --no-autotune keeps the
    # library's defaults (zeros: the context picks them)
    import argparse
    import bench
    a = argparse.Namespace(tile=64, group=8, cell=6.0, xsub=8, no_autotune=False)
    assert bench.pick_shape(a, [], 0) == dict(tile=64, group=8, cell=6.0, xsub=8, source="command line")
    a = argparse.Namespace(tile=0, group=0, cell=0.0, xsub=0, no_autotune=True)
    assert bench.pick_shape(a, [], 0) == dict(tile=0, group=0, cell=0.0, xsub=0, source="library default")


def test_bench_top5_overlap_rule():
    # tools/analyze_perf3.py:50-55: a pose of run A counts when some top-5
    # pose of run B lies within 2 A on every axis; ranks by descending score
    import bench
    tr_a = np.array([[0.0, 0, 0], [10, 0, 0], [20, 0, 0], [30, 0, 0], [40, 0, 0], [50, 0, 0]])
    sc_a = np.array([6.0, 5, 4, 3, 2, 1])
    tr_b = tr_a + np.array([1.9, -1.9, 0.0])
    assert bench.top5_overlap(tr_a, sc_a, tr_b, sc_a) == 1.0
    tr_b2 = tr_a.copy()
    tr_b2[0] += [2.1, 0, 0]
    assert bench.top5_overlap(tr_a, sc_a, tr_b2, sc_a) == 0.8
    # run B's top 5 exclude its lowest-scored pose
    sc_b = np.array([1.0, 5, 4, 3, 2, 6])
    assert bench.top5_overlap(tr_a, sc_a, tr_a, sc_b) == 0.8


def test_receptor_distance_bound_never_exceeds_the_nearest_atom():
    # the warp kernels skip a ligand group when this bound at its centre
    # exceeds its candidate radius: it must never exceed the true distance
    # to the nearest receptor atom, and it should be tight enough to skip
    # (within the grid's slack of 2 sqrt(3) cell half-diagonals + 0.01 A)
    import numpy as np
    from scipy.spatial import cKDTree
    for nr, seed in ((1500, 3), (6000, 8)):
        rec = synth.globule(nr, seed)
        c = rec["coords"]
        rng = np.random.default_rng(seed)
        lo, hi = c.min(0) - 35.0, c.max(0) + 35.0
        pts = rng.uniform(lo, hi, size=(20000, 3))
        pts = np.vstack([pts, c[:500] + rng.normal(0, 1.0, size=(500, 3))])   # near the atoms too
        lb = lkg.receptor_distance_bound(c, pts).astype(np.float64)
        d, _ = cKDTree(c).query(pts)
        assert np.all(lb <= d + 1e-9), float((lb - d).max())
        inside = lb < 24.0
        slack = 2.0 * np.sqrt(3.0) * 2.0 + 0.02
        assert np.all(lb[inside] >= np.minimum(d[inside], 24.0) - slack)
        assert (lb > 15.0).mean() > 0.2   # far points are recognised as far


def test_receptor_distance_bound_gives_up_on_a_spread_receptor():
    # a receptor spread over kilometres would need a huge bound grid: the
    # library builds none (the kernels then enumerate every group) and the
    # bound is 0, still a lower bound
    import numpy as np
    c = np.array([[0.0, 0.0, 0.0], [1.0, 2.0, 3.0], [4.0e5, 0.0, 0.0]])
    lb = lkg.receptor_distance_bound(c, np.array([[50.0, 50.0, 50.0], [0.0, 0.0, 0.0]]))
    assert np.array_equal(lb, np.zeros(2, np.float32))

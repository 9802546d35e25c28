"""Surrogate MLP on the GPU: the BF16 tensor-core forward / backward kernels
against the FP64 CPU MLP oracle (oracle/mlp.py), and online training on
exact energies.

Tolerances: against the oracle run with the device's BF16 rounding points
(``emulate=True``) the outputs agree within 1e-2 (a stored activation can
round to the neighbouring BF16 value when the FP32 accumulation order
differs) and every gradient block within 3 % relative L2 error; against the
plain FP64 network (``emulate=False``) the gradient keeps cosine >= 0.99.
"""
import numpy as np
import pytest

from oracle import mlp as omlp
from tests.lkg_helpers import config0, lkg, synth

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def sur():
    ctx = lkg.Context()
    c0 = config0()
    cid = ctx.add_complex("dna", c0["rec"], c0["lig"])
    s = lkg.Surrogate(ctx, cid, seed=5)
    yield ctx, cid, s
    s.close()
    ctx.close()


def _blocks(v):
    out, o = [], 0
    for s in omlp.SIZES:
        out.append(v[o:o + s]); o += s
    return out


def test_nparams_matches_oracle(sur):
    assert lkg.Surrogate.nparams() == omlp.NPARAM


def test_params_roundtrip(sur):
    _, _, s = sur
    p = omlp.he_params(11).astype(np.float32)
    s.set_params(p)
    assert np.array_equal(s.params(), p)


@pytest.mark.parametrize("n", [7, 256, 1000])
def test_gradient_matches_fp64_oracle(sur, n):
    _, _, s = sur
    rng = np.random.default_rng(n)
    p = omlp.he_params(n)
    s.set_params(p.astype(np.float32))
    p32 = p.astype(np.float32).astype(np.float64)
    X = rng.normal(0.0, 1.0, size=(n, omlp.IN))
    Xb = omlp.f64_to_bf16_bits(X)
    t = rng.normal(0.0, 1.0, n).astype(np.float32)
    y, g, loss = s.grad(Xb, t)
    Xr = omlp.bf16_bits_to_f64(Xb)
    l_ref, g_ref, y_ref = omlp.loss_and_grad(p32, Xr, t.astype(np.float64), emulate=True)
    assert np.abs(y - y_ref).max() < 1e-2 * (1.0 + np.abs(y_ref).max())
    assert abs(loss - l_ref) < 1e-2 * (1.0 + l_ref)
    for k, (a, b) in enumerate(zip(_blocks(g.astype(np.float64)), _blocks(g_ref))):
        err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        assert err < 3e-2, (k, err)
    # and the plain FP64 network: the BF16 gradient points the same way
    _, g64, _ = omlp.loss_and_grad(p32, Xr, t.astype(np.float64), emulate=False)
    cos = float(g @ g64 / (np.linalg.norm(g) * np.linalg.norm(g64)))
    assert cos > 0.99, cos


def test_features_are_finite_and_bounded(sur):
    ctx, cid, s = sur
    c0 = config0()
    pos = synth.to_kernel_poses(synth.setup_poses(c0["rec"]["coords"], 4, 64, 9))
    d = torch.tensor(pos, device="cuda")
    f = omlp.bf16_bits_to_f64(s.features_device(len(pos), d.data_ptr()))
    assert np.isfinite(f).all()
    assert np.abs(f).max() < 1e3
    # the constant feature and the zero padding
    assert np.all(f[:, 7 + 3 * 16] == 1.0)
    assert np.all(f[:, 8 + 3 * 16:] == 0.0)


def test_online_training_learns_exact_energies(sur):
    ctx, cid, s = sur
    c0 = config0()
    pos = synth.to_kernel_poses(synth.setup_poses(c0["rec"]["coords"], 40, 150, 21))
    scores = ctx.score(cid, pos)
    n_train = 4096
    s.set_params(omlp.he_params(3).astype(np.float32))
    s.set_target_scale(scores[:n_train])
    dp = torch.tensor(pos, device="cuda")
    ds = torch.tensor(scores, device="cuda")
    first = s.train_device(n_train, dp.data_ptr(), ds.data_ptr(), epochs=1, batch=512, lr=1e-3)
    last = s.train_device(n_train, dp.data_ptr(), ds.data_ptr(), epochs=60, batch=512, lr=1e-3)
    assert last < 0.5 * first, (first, last)
    # held-out poses: predictions rank like the exact energies
    n_test = len(pos) - n_train
    pred = torch.zeros(n_test, dtype=torch.float64, device="cuda")
    s.predict_device(n_test, dp[n_train:].data_ptr(), pred.data_ptr())
    torch.cuda.synchronize()
    pr = pred.cpu().numpy()
    ex = scores[n_train:]
    rank = lambda v: np.argsort(np.argsort(v))
    rho = np.corrcoef(rank(pr), rank(ex))[0, 1]
    assert np.isfinite(pr).all()
    assert rho > 0.5, rho


@pytest.mark.parametrize("n", [100, 1000, 4096])
def test_tcgen05_forward_matches_mma_sync_and_the_oracle(sur, n):
    # the forward layers, the backward-data products and the weight
    # gradients (MN-major operands) on tcgen05 (TMA-fed, TMEM accumulators)
    # against the mma.sync kernels and the FP64 oracle
    _, _, s = sur
    rng = np.random.default_rng(100 + n)
    p = omlp.he_params(7 + n)
    s.set_params(p.astype(np.float32))
    X = rng.normal(0.0, 1.0, size=(n, omlp.IN))
    Xb = omlp.f64_to_bf16_bits(X)
    t = rng.normal(0.0, 1.0, n).astype(np.float32)
    s.set_backend(False)
    try:
        y0, g0, l0 = s.grad(Xb, t)
    finally:
        s.set_backend(True)
    y1, g1, l1 = s.grad(Xb, t)
    assert s.status() == 0
    scale = 1.0 + np.abs(y0).max()
    assert np.abs(y1 - y0).max() < 1e-2 * scale
    p32 = p.astype(np.float32).astype(np.float64)
    _, g_ref, y_ref = omlp.loss_and_grad(p32, omlp.bf16_bits_to_f64(Xb), t.astype(np.float64), emulate=True)
    assert np.abs(y1 - y_ref).max() < 1e-2 * (1.0 + np.abs(y_ref).max())
    cos = float(g1 @ g_ref / (np.linalg.norm(g1) * np.linalg.norm(g_ref)))
    assert cos > 0.999, cos
    for k, (a, b) in enumerate(zip(_blocks(g1.astype(np.float64)), _blocks(g0.astype(np.float64)))):
        err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        assert err < 3e-2, (k, err)


def test_pipelined_forward_equals_the_per_tile_kernel(sur):
    # more row tiles than SMs: every forward layer runs on the persistent,
    # pipelined tcgen05 kernel (weights resident, A slabs through a ring,
    # two TMEM accumulators); its MMAs are the per-tile kernel's, so the
    # predictions equal those of calls small enough for the per-tile kernel
    ctx, cid, s = sur
    n = 40000 + 77   # a ragged last tile
    c0 = config0()
    pos = synth.to_kernel_poses(synth.setup_poses(c0["rec"]["coords"], 13, n // 13 + 1, 9))[:n]
    d = torch.tensor(pos, device="cuda")
    big = torch.zeros(n, dtype=torch.float64, device="cuda")
    s.predict_device(n, d.data_ptr(), big.data_ptr())
    small = torch.zeros(n, dtype=torch.float64, device="cuda")
    step = 4096   # 32 row tiles a call: the per-tile kernel
    for b0 in range(0, n, step):
        m = min(step, n - b0)
        s.predict_device(m, d.data_ptr() + 56 * b0, small.data_ptr() + 8 * b0)
    torch.cuda.synchronize()
    assert s.status() == 0
    a, b = big.cpu().numpy(), small.cpu().numpy()
    assert np.all(np.isfinite(a))
    print("pipelined vs per-tile predictions: max |diff| %.3g, bitwise equal %s" % (
        np.abs(a - b).max(), bool(np.array_equal(a, b))))
    assert np.abs(a - b).max() <= 1e-6 * (1.0 + np.abs(b).max())
    s.set_backend(False)
    try:
        ref = torch.zeros(n, dtype=torch.float64, device="cuda")
        s.predict_device(n, d.data_ptr(), ref.data_ptr())
        torch.cuda.synchronize()
        r = ref.cpu().numpy()
    finally:
        s.set_backend(True)
    assert np.abs(a - r).max() < 1e-2 * (1.0 + np.abs(r).max())


def test_tcgen05_predict_throughput_is_reported(sur):
    import time
    ctx, cid, s = sur
    n = 32768
    c0 = config0()
    pos = synth.to_kernel_poses(synth.setup_poses(c0["rec"]["coords"], 16, n // 16, 4))
    d = torch.tensor(pos, device="cuda")
    out = {}
    for tc in (False, True):
        s.set_backend(tc)
        pr = torch.zeros(n, dtype=torch.float64, device="cuda")
        s.predict_device(n, d.data_ptr(), pr.data_ptr())
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(20):
            s.predict_device(n, d.data_ptr(), pr.data_ptr())
        torch.cuda.synchronize()
        out[tc] = ((time.perf_counter() - t0) / 20, pr.cpu().numpy())
    s.set_backend(True)
    assert s.status() == 0
    flop = 2.0 * n * (64 * 256 + 2 * 256 * 256 + 256)
    print("surrogate predict, %d poses: mma.sync %.3f ms (%.1f TFLOP/s), tcgen05 %.3f ms (%.1f TFLOP/s)" % (
        n, out[False][0] * 1e3, flop / out[False][0] / 1e12, out[True][0] * 1e3, flop / out[True][0] / 1e12))
    a, b = out[False][1], out[True][1]
    assert np.abs(a - b).max() < 1e-2 * (1.0 + np.abs(a).max())

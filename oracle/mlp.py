"""FP64 CPU oracle of the pose-energy surrogate MLP (64 -> 256 -> 256 -> 256 -> 1).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the library's
BF16 tensor-core forward / backward kernels.  The surrogate has no
counterpart in the reference; this file is its specification:

* parameters, flat FP32 in the library's order W0 b0 W1 b1 W2 b2 w3 b3 with
  the W matrices stored [out][in];
* forward: H_k = ReLU(H_{k-1} W_{k-1}^T + b_{k-1}) for the three hidden
  layers, y = H_3 . w3 + b3;
* loss: mean squared error against the standardised targets;
* backward: the usual ReLU network gradients of that loss.

``emulate=True`` rounds where the device kernels round (the GEMM weights and
every stored activation / activation gradient to BF16, round to nearest
even; accumulation exact here, FP32 on the device); ``emulate=False`` is the
plain FP64 network.
"""
import numpy as np

IN, H = 64, 256
SIZES = [H * IN, H, H * H, H, H * H, H, H, 1]
NPARAM = int(sum(SIZES))


def bf16_round(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.ascontiguousarray(np.asarray(x, np.float64).astype(np.float32))
    b = f.view(np.uint32).astype(np.uint64)
    b = (b + (((b >> 16) & 1) + 0x7FFF)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def bf16_bits_to_f64(bits):
    return (np.asarray(bits, np.uint32) << 16).view(np.float32).astype(np.float64)


def f64_to_bf16_bits(x):
    f = bf16_round(x).astype(np.float32)
    return (f.view(np.uint32) >> 16).astype(np.uint16)


def unpack(p):
    p = np.asarray(p, np.float64)
    out, o = [], 0
    for s in SIZES:
        out.append(p[o:o + s]); o += s
    W0, b0, W1, b1, W2, b2, w3, b3 = out
    return W0.reshape(H, IN), b0, W1.reshape(H, H), b1, W2.reshape(H, H), b2, w3, b3[0]


def forward(p, X, emulate=True):
    """Outputs y (n,) and the hidden activations [H1, H2, H3]."""
    r = bf16_round if emulate else (lambda a: np.asarray(a, np.float64))
    W0, b0, W1, b1, W2, b2, w3, b3 = unpack(p)
    A = np.asarray(X, np.float64)
    hs = []
    for W, b in ((W0, b0), (W1, b1), (W2, b2)):
        A = r(np.maximum(A @ r(W).T + b, 0.0))
        hs.append(A)
    y = A @ w3 + b3
    return y, hs


def loss_and_grad(p, X, t, emulate=True):
    """Loss, flat gradient (library order) and outputs."""
    r = bf16_round if emulate else (lambda a: np.asarray(a, np.float64))
    X = np.asarray(X, np.float64)
    t = np.asarray(t, np.float64)
    n = len(t)
    W0, b0, W1, b1, W2, b2, w3, b3 = unpack(p)
    y, (H1, H2, H3) = forward(p, X, emulate)
    d = y - t
    loss = float(np.mean(d * d))
    dy = 2.0 * d / n
    g_w3 = H3.T @ dy
    g_b3 = np.array([dy.sum()])
    dC = r(np.where(H3 > 0, dy[:, None] * w3[None, :], 0.0))
    grads = {}
    for L, (W, Ain) in zip((2, 1, 0), ((W2, H2), (W1, H1), (W0, X))):
        grads[2 * L] = (dC.T @ Ain).ravel()
        grads[2 * L + 1] = dC.sum(axis=0)
        if L > 0:
            dC = r(np.where(Ain > 0, dC @ r(W), 0.0))
    g = np.concatenate([grads[0], grads[1], grads[2], grads[3], grads[4], grads[5], g_w3, g_b3])
    return loss, g, y


def he_params(seed):
    """A random parameter vector of the library's shape (He-uniform)."""
    rng = np.random.default_rng(seed)
    parts = []
    for k, s in enumerate(SIZES):
        fan = IN if k == 0 else H
        lim = np.sqrt(6.0 / fan) * (0.5 if k == 6 else 1.0)
        parts.append(rng.uniform(-lim, lim, s) if k % 2 == 0 else rng.uniform(-0.1, 0.1, s))
    return np.concatenate(parts)

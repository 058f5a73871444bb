"""FP32 numpy model of the radiance-cache MLP (cupbr_b200/csrc/cache_mlp.cu),
used as the checker for the tensor-core kernels.

`encode` / `forward` / `loss_and_grad` follow the kernels: the frequency
bands by FP32 double-angle steps, FP16 rounding of the encoded inputs,
weights, hidden activations, output and hidden-layer gradients, FP64
accumulation, so the kernels must agree to accumulation-order noise;
rounded=False gives the plain mathematical network (exact sin / cos) for
looser checks.
"""
from __future__ import annotations

import numpy as np

LAYERS = [(64, 96), (64, 64), (64, 64), (64, 64), (64, 64), (3, 64)]
GRAD_SCALE = 0.125
GRAD_CLAMP = 2048.0
HALF_MAX = 60000.0
BOUNCE_NORM = 16.0


def h16(x):
    return np.asarray(x, np.float32).astype(np.float16).astype(np.float32)


def split_params(p):
    out, k = [], 0
    for o, i in LAYERS:
        out.append(np.asarray(p[k:k + o * i], np.float32).reshape(o, i))
        k += o * i
    assert k == len(p)
    return out


def init_params(seed, scale=1.0):
    rng = np.random.default_rng(seed)
    ws = []
    for li, (o, i) in enumerate(LAYERS):
        a = np.sqrt((1.0 if li == len(LAYERS) - 1 else 6.0) / i) * scale
        ws.append(rng.uniform(-a, a, size=(o, i)).astype(np.float32))
    return np.concatenate([w.ravel() for w in ws])


def encode(recs, lo, inv_ext, rounded=True):
    """recs (n, 20) float32 -> (n, 96) features (see rc_encode)."""
    recs = np.asarray(recs, np.float32).reshape(-1, 20)
    n = len(recs)
    x = np.zeros((n, 96), np.float64)
    p = np.clip((recs[:, 0:3] - lo) * inv_ext, 0.0, 1.0).astype(np.float32)
    for a in range(3):
        if rounded:
            # band 0 correctly rounded, then the kernels' FP32 double-angle steps
            sn = np.sin(np.pi * p[:, a].astype(np.float64)).astype(np.float32)
            cs = np.cos(np.pi * p[:, a].astype(np.float64)).astype(np.float32)
            two = np.float32(2.0)
            for j in range(12):
                x[:, 24 * a + 2 * j] = sn
                x[:, 24 * a + 2 * j + 1] = cs
                s2 = (two * sn) * cs
                cs = (cs - sn) * (cs + sn)
                sn = s2
        else:
            for j in range(12):
                arg = np.pi * (2.0 ** j) * p[:, a].astype(np.float64)
                x[:, 24 * a + 2 * j] = np.sin(arg)
                x[:, 24 * a + 2 * j + 1] = np.cos(arg)
    x[:, 72:75] = recs[:, 4:7]
    x[:, 75:78] = recs[:, 8:11]
    x[:, 78] = recs[:, 7]
    x[:, 79:82] = recs[:, 12:15]
    x[:, 82] = 1.0
    x[:, 83] = np.clip(recs[:, 11], 0.0, BOUNCE_NORM) / BOUNCE_NORM
    x = x.astype(np.float32)
    return h16(x) if rounded else x


def forward(params, X, rounded=True):
    """Returns (y (n, 3), inputs of every layer)."""
    ws = [h16(w) if rounded else w for w in split_params(params)]
    xs = [X]
    h = X.astype(np.float64)
    for li, w in enumerate(ws):
        z = h @ w.astype(np.float64).T
        if li + 1 < len(ws):
            a = np.maximum(z, 0.0).astype(np.float32)
            a = h16(a) if rounded else a
            xs.append(a)
            h = a.astype(np.float64)
        else:
            return z.astype(np.float32), xs


def loss_and_grad(params, X, target, weight, rounded=True, kind="relative"):
    """Loss sum w (y - t)^2 / den / (3 sum w) and its gradient w.r.t. the
    parameters: den = y^2 + 0.01 held constant (relative) or 1 (l2)."""
    ws = [h16(w) if rounded else w for w in split_params(params)]
    y, xs = forward(params, X, rounded)
    d = y.astype(np.float64) - target
    den = y.astype(np.float64) ** 2 + 0.01 if kind == "relative" else np.ones_like(d)
    wsum = max(float(weight.sum()), 1.0)
    loss = float((weight[:, None] * d * d / den).sum() / (3.0 * wsum))
    g = weight[:, None] * 2.0 * d / den
    if rounded:
        g = h16(GRAD_SCALE * np.clip(g, -GRAD_CLAMP, GRAD_CLAMP)).astype(np.float64)
        scale = GRAD_SCALE
    else:
        scale = 1.0
    grads = [None] * len(ws)
    dy = g
    for li in range(len(ws) - 1, -1, -1):
        grads[li] = dy.T @ xs[li].astype(np.float64)
        if li > 0:
            dx = dy @ ws[li].astype(np.float64)
            dx = dx * (xs[li] > 0)
            dy = h16(np.clip(dx, -HALF_MAX, HALF_MAX)).astype(np.float64) if rounded else dx
    flat = np.concatenate([gr.ravel() for gr in grads]) / (scale * 3.0 * wsum)
    return loss, flat.astype(np.float32)


def random_records(n, lo, hi, seed, targets=True):
    """n training / query records inside the box [lo, hi]."""
    rng = np.random.default_rng(seed)
    r = np.zeros((n, 20), np.float32)
    r[:, 0:3] = rng.uniform(lo, hi, size=(n, 3))
    d = rng.normal(size=(n, 3))
    r[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    nn = rng.normal(size=(n, 3))
    r[:, 8:11] = nn / np.linalg.norm(nn, axis=1, keepdims=True)
    r[:, 7] = rng.uniform(0.0, 1.0, n)
    r[:, 11] = rng.integers(1, 9, n)
    r[:, 12:15] = rng.uniform(0.0, 1.0, size=(n, 3))
    if targets:
        r[:, 16:19] = rng.uniform(0.0, 2.0, size=(n, 3))
        r[:, 19] = (rng.uniform(size=n) > 0.1).astype(np.float32)
    return r


def adam_step(params, grad, lr=1e-2, b1=0.9, b2=0.99, eps=1e-15, m=None, v=None, t=1):
    m = np.zeros_like(params) if m is None else m
    v = np.zeros_like(params) if v is None else v
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    return (params - lr * mh / (np.sqrt(vh) + eps)).astype(np.float32), m, v


def constant_params(value):
    """Weights for which the network answers `value` (RGB, each exactly
    representable in FP16) for every input: the constant input feature 82
    feeds hidden unit 0 of every layer with 1, the output reads it."""
    ws = [np.zeros((o, i), np.float32) for o, i in LAYERS]
    ws[0][0, 82] = 1.0
    for li in range(1, 5):
        ws[li][0, 0] = 1.0
    ws[5][:, 0] = np.asarray(value, np.float32)
    return np.concatenate([w.ravel() for w in ws])

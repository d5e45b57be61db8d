"""ORACLE — test infrastructure only.

CPU restatement (numpy) of the radiance-cache MLP's forward and backward
passes with the BF16 roundings the tensor-core kernels apply: BF16 inputs,
weights and hidden activations, exact products accumulated in FP64 here
(FP32 on the GPU), FP32 outputs, the relative L2 loss
sum_c (y_c - t_c)^2 / (y_c^2 + 0.01) / (3 n) with its denominator held
constant, and BF16 backward activations (output gradient, masked data
gradients).  Used by tests/ as the gradient checker of the GPU kernels.
"""
import numpy as np


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    x = np.ascontiguousarray(x, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32)
    return np.where(np.isnan(x), x, out)


def bf16_bits(x):
    """BF16 bit patterns (uint16) of float32 values."""
    return (bf16(x).view(np.uint32) >> 16).astype(np.uint16)


def split(w):
    """Master weight vector -> [W0..W3 (64x64), W4 (64x3)] as [in][out]."""
    w = np.asarray(w)
    layers = [w[l * 4096:(l + 1) * 4096].reshape(64, 64) for l in range(4)]
    layers.append(w[4 * 4096:].reshape(64, 3))
    return layers


def _identity(x):
    return np.asarray(x, np.float64)


def forward(w, x, rnd=bf16):
    """x: (n, 64) BF16-valued features.  Returns (layer inputs [X0, H1..H4], y).
    rnd=_identity gives the exact (unrounded, FP64) network."""
    f = np.float32 if rnd is bf16 else np.float64
    W = [rnd(l).astype(np.float64) for l in split(w)]
    acts = [np.asarray(x, f)]
    for l in range(4):
        z = (acts[-1].astype(np.float64) @ W[l]).astype(f)
        acts.append(rnd(np.maximum(z, 0.0)).astype(f))
    y = (acts[-1].astype(np.float64) @ W[4]).astype(f)
    return acts, y


def loss_and_grad(w, x, t, rnd=bf16, stop_denominator=True):
    """Mean relative L2 loss and its gradient wrt the master weights (flat).
    The kernels hold the denominator constant; stop_denominator=False gives
    the full derivative (for finite-difference checks of the exact network)."""
    f = np.float32 if rnd is bf16 else np.float64
    n = x.shape[0]
    scale = f(1.0 / (3.0 * n))
    acts, y = forward(w, x, rnd)
    t = np.asarray(t, f)[:, :3]
    e = y - t
    den = y * y + f(0.01)
    loss = float(np.sum((e * e / den).astype(np.float64)) * scale)
    d = f(2.0) * e / den
    if not stop_denominator:
        d = d - f(2.0) * y * e * e / (den * den)
    go = rnd(d * scale).astype(f)
    W = [rnd(l).astype(np.float64) for l in split(w)]
    grads = [None] * 5
    grads[4] = acts[4].astype(np.float64).T @ go.astype(np.float64)
    g = rnd(((go.astype(np.float64) @ W[4].T) * (acts[4] > 0)).astype(f)).astype(f)
    for l in range(3, -1, -1):
        grads[l] = acts[l].astype(np.float64).T @ g.astype(np.float64)
        if l > 0:
            g = rnd(((g.astype(np.float64) @ W[l].T) * (acts[l] > 0)).astype(f)).astype(f)
    flat = np.concatenate([grads[l].reshape(-1) for l in range(5)])
    return loss, flat.astype(f), y


def adam(w, m, v, g, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (float32), returns (w, m, v)."""
    m = np.float32(b1) * m + np.float32(1 - b1) * g
    v = np.float32(b2) * v + np.float32(1 - b2) * g * g
    mh = m / np.float32(1 - b1 ** step)
    vh = v / np.float32(1 - b2 ** step)
    return (w - np.float32(lr) * mh / (np.sqrt(vh) + np.float32(eps))).astype(np.float32), m, v

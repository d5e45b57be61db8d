"""The radiance-cache oracle (oracle/mlp.py): its backward pass against finite
differences of the exact network, BF16 rounding against torch, Adam."""
import numpy as np
import torch

from oracle import mlp


def _problem(n=40, seed=0):
    rng = np.random.default_rng(seed)
    w = (rng.uniform(-1, 1, 16576) * np.sqrt(6 / 64)).astype(np.float64)
    x = rng.uniform(-1, 1, (n, 64))
    t = rng.uniform(0.1, 2.0, (n, 4))
    return w, x, t


def test_bf16_rounding_matches_torch():
    x = np.random.default_rng(1).standard_normal(10000).astype(np.float32) * 10
    assert np.array_equal(mlp.bf16(x), torch.tensor(x).bfloat16().float().numpy())


def test_exact_backward_matches_finite_differences():
    w, x, t = _problem()
    _, g, _ = mlp.loss_and_grad(w, x, t, rnd=mlp._identity, stop_denominator=False)
    rng = np.random.default_rng(3)
    idx = np.concatenate([rng.choice(16384, 24, replace=False), 16384 + rng.choice(192, 8, replace=False)])
    h = 1e-5
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        lp, _, _ = mlp.loss_and_grad(wp, x, t, rnd=mlp._identity)
        lm, _, _ = mlp.loss_and_grad(wm, x, t, rnd=mlp._identity)
        num = (lp - lm) / (2 * h)
        assert abs(num - g[i]) <= 1e-6 + 1e-4 * abs(num), (i, num, g[i])


def test_bf16_gradient_close_to_exact():
    w, x, t = _problem(n=256, seed=5)
    _, g_exact, _ = mlp.loss_and_grad(w, x, t, rnd=mlp._identity)
    _, g_bf, _ = mlp.loss_and_grad(w.astype(np.float32), mlp.bf16(x.astype(np.float32)), t.astype(np.float32))
    rel = np.linalg.norm(g_bf - g_exact) / np.linalg.norm(g_exact)
    assert rel < 0.05, rel


def test_adam_first_step_moves_by_lr():
    g = np.random.default_rng(2).standard_normal(100).astype(np.float32)
    w = np.zeros(100, np.float32)
    w2, m, v = mlp.adam(w, np.zeros_like(w), np.zeros_like(w), g, 1, lr=1e-3)
    np.testing.assert_allclose(np.abs(w2), 1e-3, rtol=1e-3)

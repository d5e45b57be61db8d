"""Radiance-cache MLP on the tcgen05 tensor cores against the CPU oracle
(oracle/mlp.py): forward outputs, the loss gradient of a training step, the
Adam update, and that training reduces the loss."""
import numpy as np
import pytest
import torch

from oracle import mlp

pytestmark = pytest.mark.gpu


def _batch(n, seed):
    rng = np.random.default_rng(seed)
    x = mlp.bf16(rng.uniform(-1, 1, (n, 64)).astype(np.float32))
    t = np.zeros((n, 4), np.float32)
    t[:, :3] = rng.uniform(0.05, 2.0, (n, 3))
    return x, t


def _dev(x, t):
    xd = torch.from_numpy(mlp.bf16_bits(x).view(np.int16).copy()).cuda()
    td = torch.from_numpy(t).cuda()
    return xd, td


@pytest.mark.parametrize('n', [1000, 4096, 300001])
def test_cache_forward_matches_oracle(vb, gpu_ctx, n):
    # 300,001 rows: several tiles per pipeline (the next tile streamed while
    # the current one runs) and a ragged last tile read past the end.
    cache = vb.RadianceCache(gpu_ctx, seed=3)
    w = cache.weights()
    x, t = _batch(n, 1)
    xd, _ = _dev(x, t)
    out = torch.zeros((n, 4), dtype=torch.float32, device='cuda')
    cache.infer(xd.data_ptr(), n, out.data_ptr())
    torch.cuda.synchronize()
    _, y = mlp.forward(w, x)
    got = out.cpu().numpy()[:, :3]
    # FP32 accumulation order differs from the oracle's, which can move a BF16
    # rounding of a hidden activation by one unit.
    assert np.abs(got - y).max() <= 2e-2 * np.abs(y).max(), np.abs(got - y).max()
    assert np.mean(np.abs(got - y) <= 1e-3 * (1 + np.abs(y))) >= 0.99
    again = torch.zeros_like(out)
    cache.infer(xd.data_ptr(), n, again.data_ptr())
    torch.cuda.synchronize()
    assert torch.equal(out, again)
    cache.close()


@pytest.mark.parametrize('n', [1000, 65536])
def test_cache_gradient_matches_oracle(vb, gpu_ctx, n):
    cache = vb.RadianceCache(gpu_ctx, seed=5)
    w = cache.weights()
    x, t = _batch(n, 2)
    xd, td = _dev(x, t)
    cache.train(xd.data_ptr(), td.data_ptr(), n, update=False)
    g, loss = cache.gradient()
    loss_ref, g_ref, _ = mlp.loss_and_grad(w, x, t)
    assert abs(loss - loss_ref) <= 1e-3 * loss_ref, (loss, loss_ref)
    rel = np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref)
    assert rel < 1e-2, rel
    for l, (a, b) in enumerate(zip(mlp.split(g), mlp.split(g_ref))):
        r = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-30)
        assert r < 2e-2, (l, r)
    np.testing.assert_array_equal(cache.weights(), w)  # update=False leaves the weights
    cache.close()


def test_cache_adam_update_matches_oracle(vb, gpu_ctx):
    cache = vb.RadianceCache(gpu_ctx, seed=7)
    w = cache.weights()
    x, t = _batch(2048, 3)
    xd, td = _dev(x, t)
    cache.train(xd.data_ptr(), td.data_ptr(), 2048, update=True)
    g, _ = cache.gradient()
    w_ref, _, _ = mlp.adam(w, np.zeros_like(w), np.zeros_like(w), g, 1)
    np.testing.assert_allclose(cache.weights(), w_ref, rtol=1e-5, atol=1e-7)
    cache.close()


def test_cache_training_reduces_loss(vb, gpu_ctx):
    # Targets from a fixed smooth function of the features: the network must fit it.
    cache = vb.RadianceCache(gpu_ctx, seed=11)
    cache.set_optimizer(lr=1e-2)
    n = 16384
    rng = np.random.default_rng(4)
    x = mlp.bf16(rng.uniform(-1, 1, (n, 64)).astype(np.float32))
    t = np.zeros((n, 4), np.float32)
    t[:, 0] = 1.0 + 0.5 * np.sin(3 * x[:, 0])
    t[:, 1] = 1.0 + 0.5 * x[:, 1] * x[:, 2]
    t[:, 2] = 0.5 + np.abs(x[:, 3])
    xd, td = _dev(x, t)
    losses = []
    for step in range(300):
        cache.train(xd.data_ptr(), td.data_ptr(), n, update=True)
        if step % 50 == 0 or step == 299:
            losses.append(cache.gradient()[1])
    assert losses[-1] < 0.1 * losses[0], losses
    cache.close()

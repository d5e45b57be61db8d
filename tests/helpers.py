"""Shared helpers for the test-suite: seeded ray batches and image statistics."""
import numpy as np


def seeded_rays(n, lo, hi, seed, tmax=3.0e38, targets=None):
    """n rays (8 floats: origin, 0, direction, tmax) with origins uniform in the
    box [lo, hi] and directions uniform on the sphere; with `targets` (k, 3),
    half of the rays are aimed exactly at those points (edges, vertices) to
    provoke ties between neighbouring triangles."""
    rng = np.random.default_rng(seed)
    lo = np.asarray(lo, np.float32)
    hi = np.asarray(hi, np.float32)
    o = (lo + (hi - lo) * rng.random((n, 3))).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    if targets is not None and len(targets):
        k = n // 2
        tgt = targets[rng.integers(0, len(targets), k)]
        d[:k] = (tgt - o[:k]).astype(np.float32)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 4:7] = d
    rays[:, 7] = tmax
    return rays


def edge_targets(pos, idx):
    """Midpoints of triangle edges and the vertices themselves."""
    p = pos.reshape(-1, 3)
    t = idx.reshape(-1, 3)
    mids = [(p[t[:, a]] + p[t[:, b]]) * 0.5 for a, b in ((0, 1), (1, 2), (2, 0))]
    return np.concatenate(mids + [p]).astype(np.float32)

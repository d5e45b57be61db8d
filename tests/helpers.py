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


def pixel_z(sum_a, sq_a, n_a, sum_b, sq_b, n_b):
    """Per-pixel, per-channel two-sample z statistic of two Monte Carlo
    estimates given their FP64 sums and sums of squares over n_a and n_b
    samples: (mean_a - mean_b) / sqrt(var_a / n_a + var_b / n_b), with the
    unbiased sample variances.  A tiny floor keeps pixels whose samples are
    all equal (a directly seen emitter, the empty background) finite: equal
    means give z = 0 there, different means a large |z|."""
    sum_a, sq_a, sum_b, sq_b = (np.asarray(x, np.float64) for x in (sum_a, sq_a, sum_b, sq_b))
    ma, mb = sum_a / n_a, sum_b / n_b
    va = np.maximum(sq_a / n_a - ma * ma, 0.0) * n_a / (n_a - 1.0)
    vb = np.maximum(sq_b / n_b - mb * mb, 0.0) * n_b / (n_b - 1.0)
    floor = (1e-6 * (np.abs(ma) + np.abs(mb))) ** 2 + 1e-20
    return (ma - mb) / np.sqrt(va / n_a + vb / n_b + floor)


def path_sums(values):
    """Sums and sums of squares over axis 0 of per-path radiance
    (frames, ..., 3), with NaN/Inf samples zeroed as the film does."""
    v = np.asarray(values, np.float64)
    bad = ~np.isfinite(v).all(-1, keepdims=True)
    v = np.where(bad, 0.0, v)
    return v.sum(0), (v * v).sum(0)


def mean_z(sum_a, sq_a, n_a, sum_b, sq_b, n_b):
    """z statistic of the difference of two images' means (over all pixels
    and channels), from per-pixel FP64 sums and sums of squares: robust to a
    few bright paths (a reflected sun) that dominate a plain relative mean."""
    sum_a, sq_a, sum_b, sq_b = (np.asarray(x, np.float64) for x in (sum_a, sq_a, sum_b, sq_b))
    ma, mb = sum_a / n_a, sum_b / n_b
    va = np.maximum(sq_a / n_a - ma * ma, 0.0) * n_a / (n_a - 1.0)
    vb = np.maximum(sq_b / n_b - mb * mb, 0.0) * n_b / (n_b - 1.0)
    k = ma.size
    se = np.sqrt((va / n_a + vb / n_b).sum()) / k
    return (ma.mean() - mb.mean()) / max(se, 1e-30)


def write_room_textures(folder, seed=7):
    """The image files of scenes.textured_room, written with OpenCV from a
    seeded generator: an RGB checker PNG with noise, a grey gradient PNG and
    a smooth RGB JPEG (4:2:0)."""
    import os
    import cv2
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:48, 0:64]
    check = ((xx // 8 + yy // 8) % 2).astype(bool)
    rgb = np.where(check[..., None], np.array([200, 60, 40]), np.array([30, 120, 220]))
    rgb = np.clip(rgb + rng.integers(-20, 21, rgb.shape), 0, 255).astype(np.uint8)
    cv2.imwrite(os.path.join(folder, 'checker.png'), rgb[..., ::-1])
    g = (np.add.outer(np.arange(32) * 5, np.arange(32) * 3) % 256).astype(np.uint8)
    cv2.imwrite(os.path.join(folder, 'gradient.png'), g)
    y, x = np.mgrid[0:24, 0:40] / 8.0
    photo = np.stack([128 + 100 * np.sin(x + 0.3 * y), 128 + 90 * np.cos(0.7 * x - y), 128 + 80 * np.sin(x * y / 3)], -1)
    cv2.imwrite(os.path.join(folder, 'photo.jpg'), np.clip(photo, 0, 255).astype(np.uint8)[..., ::-1],
                [cv2.IMWRITE_JPEG_QUALITY, 90])

"""Closest-hit and any-hit parity of the BVH8 traversal kernels against the
oracle: primitive ids, barycentrics and t bit-exact on seeded ray batches
(ties in t resolve to the lower primitive id on both sides)."""
import numpy as np
import pytest

import oracle
from helpers import edge_targets, seeded_rays
from vision_b200 import scenes

pytestmark = pytest.mark.gpu


def _soup(n_tris, seed):
    rng = np.random.default_rng(seed)
    c = rng.random((n_tris, 3)) * 2.0 - 1.0
    P = (c[:, None, :] + 0.08 * rng.normal(size=(n_tris, 3, 3))).astype(np.float32)
    # A watertight fan around a shared vertex exercises edge ties.
    fan = []
    k = 16
    for i in range(k):
        a0, a1 = 2 * np.pi * i / k, 2 * np.pi * (i + 1) / k
        fan.append([[0, 0, 0], [0.5 * np.cos(a0), 0.5 * np.sin(a0), 0], [0.5 * np.cos(a1), 0.5 * np.sin(a1), 0]])
    P = np.concatenate([P, np.array(fan, np.float32)])
    return P.reshape(-1).tolist(), list(range(P.shape[0] * 3))


def _check(s, o, rays):
    h_gpu, t_gpu = s.trace_closest(rays)
    h_cpu, t_cpu = o.trace_closest(rays)
    miss = h_cpu[:, 1] == 0xffffffff
    assert np.array_equal(h_gpu[:, 1], h_cpu[:, 1]), np.nonzero(h_gpu[:, 1] != h_cpu[:, 1])[0][:10]
    assert np.array_equal(h_gpu[:, 0], h_cpu[:, 0])
    assert np.array_equal(h_gpu[~miss, 2:], h_cpu[~miss, 2:])
    assert np.array_equal(t_gpu.view(np.uint32), t_cpu.view(np.uint32))
    occ_gpu = s.trace_any(rays)
    occ_cpu = o.trace_any(rays)
    assert np.array_equal(occ_gpu, occ_cpu)
    assert np.array_equal(occ_gpu.astype(bool), ~miss)
    return miss.mean()


def test_box_room_closest_hit_bit_exact(vb, gpu_ctx):
    s = vb.Scene(gpu_ctx, scenes.box_room()).build_accel()
    o = oracle.OracleScene(s)
    tg = edge_targets(s.export('pos', np.float32), s.export('idx', np.uint32))
    rays = seeded_rays(1 << 20, [-0.6, -0.1, -0.6], [0.6, 1.1, 1.9], seed=11, targets=tg)
    miss_rate = _check(s, o, rays)
    assert 0.0 < miss_rate < 0.9


@pytest.mark.parametrize('collapse, leaf', [('sah', 1), ('sah', 3), ('greedy', 1), ('greedy', 3)])
def test_triangle_soup_closest_hit_bit_exact(vb, gpu_ctx, collapse, leaf):
    # Both ways of choosing each wide node's children, and leaves of one and
    # of three triangles: the BVH changes, the hits do not.
    P, I = _soup(20000, 5)
    sc = scenes.box_room(width=4, height=4)
    sc['render_setting']['bvh_collapse'] = collapse
    sc['render_setting']['bvh_leaf_size'] = leaf
    sc['shapes'].append({'type': 'mesh', 'name': 'soup', 'param': {'positions': P, 'indices': I,
                                                                  'material': 'Floor'}})
    s = vb.Scene(gpu_ctx, sc).build_accel()
    assert s.info()['bvh_depth'] >= 3
    o = oracle.OracleScene(s)
    tg = edge_targets(s.export('pos', np.float32), s.export('idx', np.uint32))
    rays = seeded_rays(1 << 18, [-1.2, -1.2, -1.2], [1.2, 1.2, 1.2], seed=12, targets=tg)
    _check(s, o, rays)


def test_finite_tmax_and_empty_batch(vb, gpu_ctx):
    s = vb.Scene(gpu_ctx, scenes.box_room()).build_accel()
    o = oracle.OracleScene(s)
    rays = seeded_rays(4096, [-0.4, 0.1, -0.4], [0.4, 0.9, 0.4], seed=13, tmax=0.3)
    _check(s, o, rays)
    h, t = s.trace_closest(np.zeros((0, 8), np.float32))
    assert h.shape == (0, 4)

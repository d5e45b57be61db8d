"""Instancing (reference Geometry::build_accel: one BLAS per mesh and an IAS
over the instances, src/base/mgr/geometry.cpp:20-52; MeshRegistry shares
equal meshes): shapes with equal vertices and triangles share one
object-space mesh, and scenes whose instances repeat their meshes are traced
through a two-level BVH.  CPU side: mesh sharing, the choice of levels, and
that each instance's world-space vertices are its mesh through its
transform."""
import numpy as np

from vision_b200 import scenes


def test_equal_shapes_share_one_mesh(vb, host_ctx):
    s = vb.Scene(host_ctx, scenes.box_room(16, 16)).build_accel()
    info = s.info()
    # Five 1 x 1 wall quads share a mesh; the light quad and the two boxes
    # are their own: four meshes, eight instances.  The room is small, so it
    # keeps one world-space BVH by default.
    assert info['mesh_count'] == 4 and info['instance_count'] == 8
    assert info['two_level'] == 0
    assert np.array_equal(s.export('inst_mesh', np.uint32), [0, 0, 0, 0, 0, 1, 2, 3])


def test_instancing_modes(vb, host_ctx):
    sc = scenes.box_room(16, 16)
    sc['render_setting']['instancing'] = True
    assert vb.Scene(host_ctx, sc).build_accel().info()['two_level'] == 1
    big = scenes.instanced_scene(width=16, height=16, copies=16, subdivisions=5, patch=260)
    s = vb.Scene(host_ctx, big).build_accel()
    info = s.info()
    # 16 copies of one icosphere (20,480) and one grid (135,200 triangles):
    # 2.5 M triangles from two meshes, traced through two levels by default.
    assert info['mesh_count'] == 2 and info['instance_count'] == 32 and info['two_level'] == 1
    assert info['prim_count'] == 16 * (20480 + 135200)
    big['render_setting']['instancing'] = False
    assert vb.Scene(host_ctx, big).build_accel().info()['two_level'] == 0


def test_instance_world_vertices_follow_their_transform(vb, host_ctx):
    big = scenes.instanced_scene(width=16, height=16, copies=4, subdivisions=3, patch=10)
    s = vb.Scene(host_ctx, big).build_accel()
    mp = s.export('mesh_pos', np.float32).reshape(-1, 3)
    meshes = s.export('meshes', np.uint32).reshape(-1, 6)
    inst_mesh = s.export('inst_mesh', np.uint32)
    w2o = s.export('inst_w2o', np.float32).reshape(-1, 4, 4)  # [c][r]
    pos = s.export('pos', np.float32).reshape(-1, 3)
    inst = s.export('instances', np.uint32).reshape(-1, 4)
    idx = s.export('idx', np.uint32).reshape(-1, 3)
    for i in range(len(inst_mesh)):
        m = meshes[inst_mesh[i]]
        first_prim, count = inst[i, 2], inst[i, 3]
        assert count == m[3]
        wv = pos[idx[first_prim:first_prim + count].ravel()]
        M = w2o[i].T.astype(np.float64)  # row-major world-to-object
        ov = (np.c_[wv, np.ones(len(wv))] @ M.T)[:, :3]
        mi = s.export('mesh_idx', np.uint32).reshape(-1, 3)[m[2]:m[2] + m[3]].ravel()
        np.testing.assert_allclose(ov, mp[m[0] + mi], atol=2e-5)

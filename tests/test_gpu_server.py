"""Render-job server: a job's film equals vs_render of the same scene, camera,
resolution and frames; the same job gives the same film alone and inside a
mix of concurrent jobs of other scenes, resolutions and spp; real-time jobs
continue their scene's resident ReSTIR history; admission keeps the job-slot
limit; latency statistics are ordered."""
import numpy as np
import pytest

from vision_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def served(vb, gpu_ctx):
    box = vb.Scene(gpu_ctx, scenes.box_room(64, 48, sampler='pcg')).build_accel()
    big = vb.Scene(gpu_ctx, scenes.large_scene(48, 40, subdivisions=3, grid=60, tiles=3, sky_width=256,
                                               sky_height=128, max_depth=6)).build_accel()
    return box, big


def test_server_job_equals_render(vb, gpu_ctx, served):
    box, big = served
    srv = vb.Server(gpu_ctx, hbm_budget=4 << 30, max_jobs=8, paths_per_batch=1 << 16)
    ids = [srv.add_scene(box), srv.add_scene(big)]
    for sid, scene in zip(ids, (box, big)):
        info = scene.info()
        j = srv.submit(sid, info['width'], info['height'], 6, frame_begin=0)
        got = srv.result(j, timeout=120)
        scene.render(0, 6)
        ref = scene.film()
        close = np.abs(got - ref) <= 1e-5 + 1e-5 * np.abs(ref)
        assert close.all(-1).mean() >= 0.999, close.all(-1).mean()
    srv.close()


def test_server_mix_material_scene(vb, gpu_ctx, served):
    # Mix and add materials in a served scene: their hits take the mix
    # shading class of the batch graphs, as in the wavefront schedule.
    box, _ = served
    mixed = vb.Scene(gpu_ctx, scenes.mix_room(40, 32, sampler='pcg', max_depth=6)).build_accel()
    srv = vb.Server(gpu_ctx, hbm_budget=4 << 30, max_jobs=8, paths_per_batch=1 << 15)
    ids = [srv.add_scene(mixed), srv.add_scene(box)]
    jobs = [srv.submit(ids[0], 40, 32, 5, frame_begin=0), srv.submit(ids[1], 64, 48, 3, frame_begin=2)]
    got = srv.result(jobs[0], timeout=120)
    srv.result(jobs[1], timeout=120)
    mixed.render(0, 5)
    ref = mixed.film()
    assert np.isfinite(got).all() and ref[..., :3].max() > 0
    close = np.abs(got - ref) <= 1e-5 + 1e-5 * np.abs(ref)
    assert close.all(-1).mean() >= 0.999, close.all(-1).mean()
    srv.close()


def test_server_same_alone_and_in_mix(vb, gpu_ctx, served):
    box, big = served
    srv = vb.Server(gpu_ctx, hbm_budget=4 << 30, max_jobs=16, paths_per_batch=1 << 15)
    b, g = srv.add_scene(box), srv.add_scene(big)
    cam = scenes.camera_c2w((0.05, 0.45, 1.8), (0.0, 0.5, 0.0))
    alone = srv.result(srv.submit(b, 40, 30, 9, frame_begin=3, c2w=cam, fov_y=40.0), timeout=120)
    rng = np.random.default_rng(0)
    mix = []
    for k in range(10):
        sid = (b, g)[k % 2]
        w, h = [(32, 32), (48, 40), (64, 48), (24, 16)][rng.integers(0, 4)]
        mix.append(srv.submit(sid, w, h, int(rng.choice([1, 4, 16])), frame_begin=int(rng.integers(0, 50))))
        if k == 4:
            target = srv.submit(b, 40, 30, 9, frame_begin=3, c2w=cam, fov_y=40.0)
    in_mix = srv.result(target, timeout=120)
    for j in mix:
        srv.result(j, timeout=120)
    assert np.array_equal(alone, in_mix)
    st = srv.stats()
    assert st['completed'] == st['submitted'] == 12
    assert st['batches'] > 1 and st['graph_launches'] == st['batches']
    assert st['p50_ms'] <= st['p95_ms'] <= st['p99_ms'] <= st['max_ms']
    srv.close()


def test_server_realtime_jobs_keep_reservoirs_resident(vb, gpu_ctx, served):
    # Real-time (ReSTIR) jobs on a resident rt scene: each job renders its
    # frames into the scene's film with the scene's reservoirs resident, so
    # consecutive jobs continue one temporal history (job k's camera is the
    # previous camera of job k + 1's first frame).  Each job's film equals
    # vs_restir_frame run directly on a twin scene with the same cameras,
    # frame indices and film restarts, while path-tracing jobs of another
    # scene share the batches.
    box, _ = served
    w, h = 48, 32
    sc = scenes.many_lights(w, h, emitters=200, seed=5, M_light=8, history_limit=20, spatial_neighbours=5,
                            spatial_radius=8.0, max_depth=4)
    rt = vb.Scene(gpu_ctx, sc).build_accel()
    twin = vb.Scene(gpu_ctx, sc).build_accel()
    cams = scenes.camera_spline(3, seed=3)
    srv = vb.Server(gpu_ctx, hbm_budget=4 << 30, max_jobs=8, paths_per_batch=1 << 15)
    r, b = srv.add_scene(rt), srv.add_scene(box)
    assert srv.stats()['resident_bytes'] > 64 * w * h * 9  # reservoirs and surfaces count against the budget
    jobs, pt_jobs = [], []
    for k in range(3):
        jobs.append(srv.submit(r, w, h, 3, frame_begin=3 * k, c2w=cams[k], fov_y=40.0))
        pt_jobs.append(srv.submit(b, 32, 32, 4, frame_begin=k))
    got = [srv.result(j, timeout=120) for j in jobs]
    for j in pt_jobs:
        srv.result(j, timeout=120)
    with pytest.raises(vb.VisionError):
        srv.submit(r, w + 8, h, 1)  # real-time jobs render at their scene's resolution
    st = srv.stats()
    assert st['completed'] == 6
    srv.close()
    for k in range(3):
        twin.set_camera(cams[k], 40.0)
        for i in range(3):
            twin.restir_frame(3 * k + i, i)
        assert np.array_equal(got[k], twin.film()), k


def test_server_admission_limit(vb, gpu_ctx, served):
    box, _ = served
    srv = vb.Server(gpu_ctx, hbm_budget=4 << 30, max_jobs=2, paths_per_batch=1 << 14)
    b = srv.add_scene(box)
    jobs = [srv.submit(b, 32, 32, 8, frame_begin=i) for i in range(6)]
    for j in jobs:
        srv.result(j, timeout=120)
    st = srv.stats()
    assert st['peak_jobs'] <= 2 and st['completed'] == 6
    assert st['peak_bytes'] <= 2 * 32 * 32 * 16
    srv.close()


def test_server_rejects(vb, gpu_ctx, served):
    box, _ = served
    srv = vb.Server(gpu_ctx, hbm_budget=1 << 30, max_jobs=2, paths_per_batch=1 << 12)
    b = srv.add_scene(box)
    with pytest.raises(vb.VisionError):
        srv.submit(b, 128, 128, 1)      # one frame larger than a batch
    with pytest.raises(vb.VisionError):
        srv.submit(7, 16, 16, 1)        # unknown scene
    rt = vb.Scene(gpu_ctx, scenes.box_room(16, 16, dimension=3)).build_accel()
    with pytest.raises(vb.UnsupportedError):
        srv.add_scene(rt)
    srv.close()


def test_server_budget_counts_resident_scenes(vb, gpu_ctx, served):
    # The HBM budget covers the resident scenes as well as the batch scratch
    # and the job films: a scene that does not fit beside the others is
    # refused, and the stats report the resident and scratch bytes.
    box, big = served
    srv = vb.Server(gpu_ctx, hbm_budget=4 << 30, max_jobs=4, paths_per_batch=1 << 15)
    srv.add_scene(box)
    r_box = srv.stats()['resident_bytes']
    srv.add_scene(big)
    st = srv.stats()
    r_big = st['resident_bytes'] - r_box
    scratch = st['scratch_bytes']
    srv.close()
    assert r_box > 0 and r_big > 12 << 20 and scratch > 0  # the sky's RGB table alone is 12.6 MB
    srv = vb.Server(gpu_ctx, hbm_budget=scratch + r_box + r_big // 2, max_jobs=4, paths_per_batch=1 << 15)
    srv.add_scene(box)
    with pytest.raises(vb.VisionError) as e:
        srv.add_scene(big)
    assert 'budget' in str(e.value)
    assert srv.stats()['resident_bytes'] == r_box
    # A job whose film does not fit beside the resident scene is refused too.
    with pytest.raises(vb.VisionError):
        srv.submit(0, 4096, 4096, 1)
    srv.close()

"""Benchmark of the spectral path-tracing hot path on B200.

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload large_scene|box_room]

Workloads: `large_scene` (default) — the 2.3 M-triangle seeded scene
(displaced icosphere on a 1000 x 1000 ground of 100 material tiles, GGX gold /
dispersive glass / principled materials, procedural HDR sky), 1024 x 1024,
64 spp, max depth 16; `box_room` — the 36-triangle box room, 256 x 256, 16 spp,
max depth 8.  One step renders the whole workload once (every pixel, every
frame of its spp, through vs_render on the GPU).  value = paths of all ranks / max-over-ranks
device time of the K timed steps, in Mpaths/s.  Multi-GPU runs are
independent replicas (weak scaling); the path has no exchange step.
--impl reference times the reference integrator's CPU restatement (the
reference itself does not build offline) on the host cores.

The default run (large_scene, one GPU) also runs the metric's other workloads
after the headline and reports them under `sub`: the box room, the ReSTIR
frame, the radiance cache (time to relMSE 1e-2) and a serving run (its job
count in its config); --no-sub skips them.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # Box room: 256 x 256, 16 spp, max depth 8, 4 hero wavelengths, 6500 K
    # blackbody light, PCG sampler seed 0, FP32 film.
    'box_room': dict(kind='box_room', width=256, height=256, spp=16, max_depth=8, dimension=4, sampler='pcg', seed=0),
    # Large seeded scene: 1024 x 1024, 64 spp, max depth 16, 4 hero
    # wavelengths, PCG sampler, scene seed 1, FP32 film.
    'large_scene': dict(kind='large_scene', width=1024, height=1024, spp=64, max_depth=16, dimension=4, sampler='pcg',
                        seed=1),
}
# Real-time ReSTIR on the many-light box room: 1920 x 1080, 1 spp per frame,
# 10,000 blackbody emitters, power light sampler, 32 light candidates,
# temporal M-cap 20, one spatial pass of 5 neighbours within 30 px, camera on
# a seeded 64-frame spline; one step = one frame (direct + indirect + combine).
WORKLOADS['many_lights'] = dict(kind='many_lights', width=1920, height=1080, spp=1, frames=64, emitters=10000,
                                M_light=32, history_limit=20, spatial_neighbours=5, spatial_radius=30.0,
                                max_depth=8, dimension=3, sampler='pcg', seed=7)
# Serving: Poisson arrivals (lambda = 50 jobs/s, seeded) of render jobs with
# resolution uniform over {256^2, 512^2, 1024^2, 1920x1080}, spp uniform over
# {1, 4, 16, 64}, each on one of 4 resident scenes (box room, large scene,
# many-light box room geometry with the plain tracer, 10 M-triangle instanced
# scene), HBM admission budget 150 GB; one step = one job.  The full
# configuration is 10,000 jobs; --steps sets how many are submitted.
WORKLOADS['serving'] = dict(kind='serving', rate=50.0, jobs=10000, hbm_budget_gb=150, max_jobs=64,
                            paths_per_batch=1 << 24, seed=21,
                            resolutions=[[256, 256], [512, 512], [1024, 1024], [1920, 1080]],
                            spp=[1, 4, 16, 64], scenes=['box_room', 'large_scene', 'many_lights_pt', 'instanced'])
# Learned radiance cache on the box room at 1920 x 1080 (3 hero wavelengths,
# the cache's 3 spectral outputs): paths end in the cache after two bounces,
# 65,536 training samples per frame
# (two-bounce-longer suffixes), Adam lr 1e-3.  One step = one cached frame
# (with its training step).  Quality: relMSE against a plain FP64-accumulated
# render of `reference_spp` frames, and the time each method needs to reach
# relMSE 1e-2.
WORKLOADS['radiance_cache'] = dict(kind='radiance_cache', width=1920, height=1080, max_depth=8, dimension=3,
                                   sampler='pcg', seed=0, train_samples=65536, lr=1e-3, warmup_frames=256,
                                   reference_spp=1024, target_relmse=1e-2)
DEFAULT_WORKLOAD = 'large_scene'
DEFAULT_STEPS = {'box_room': 100, 'large_scene': 5, 'many_lights': 64, 'serving': 200, 'radiance_cache': 64}

# DRAM bytes per path of k_render measured by ncu (dram__bytes_read.sum +
# dram__bytes_write.sum of one launch divided by its paths; profiles/).
NCU_TRAFFIC_PER_PATH = {('large_scene', 'persistent'): 383.6e6 / 2097152,
                        ('box_room', 'persistent'): 7.42e6 / 1048576,
                        # all wavefront kernels of one render (2,097,152 and 1,048,576 paths)
                        ('large_scene', 'wavefront'): 3059.95e6 / 2097152,
                        ('box_room', 'wavefront'): 1990.0e6 / 1048576}

# Issue-slot utilisation and active threads per instruction of the dominant
# traversal kernel, from the committed one-kernel ncu capture of the same
# workload's 2-spp case (the binding measure of the L1/L2-resident traversal).
NCU_ISSUE = {('large_scene', 'wavefront'): {
    'issue_active': 0.652, 'threads_per_inst': 12.95,
    'issue_source': 'ncu sm__inst_issued / smsp__thread_inst_executed_per_inst_executed of k_wf_extend '
                    '(profiles/k_wf_extend_large_scene.md)'}}

# Algorithmic bytes per pixel-frame of the ReSTIR frame, from the record sizes
# (64 B surfaces and reservoirs, 32 B extensions and BSDF samples, 16 B
# radiance, 8 B motion vectors, 16 B light-candidate fetch of 8 B alias +
# 36 B triangle + 64 B light record) for M light candidates and S spatial
# neighbours:
#   direct shader0: surface write 64 + motion 8 + BSDF sample 32 + previous
#     reservoir and surface 128 + passthrough write 64 + M x 108
#   direct shader1: own surface + passthrough 128 + S x 128 + radiance 16 + reservoir 64
#   indirect initial: surface 64 + BSDF sample 32 + sample 64 + radiance 16
#   indirect temporal: surface 64 + sample 64 + BSDF sample 32 + motion 8 + previous 128 + write 64
#   indirect spatial: surface 64 + passthrough 64 + S x 128 + radiance 16 + reservoir 64
#   combine: 2 x 16 radiance + film read/write 32
def restir_bytes_per_pixel(M, S):
    return ((64 + 8 + 32 + 128 + 64 + M * 108) + (128 + S * 128 + 16 + 64) + (64 + 32 + 64 + 16) +
            (64 + 64 + 32 + 8 + 128 + 64) + (64 + 64 + S * 128 + 16 + 64) + (32 + 32))


def scenes_module():
    """The scene builders (vision_b200/scenes.py, plain Python).  Loaded from
    its file when the vision_b200 package is not imported, so that the
    reference arm never loads the CUDA library."""
    if 'vision_b200' in sys.modules:
        from vision_b200 import scenes
        return scenes
    import importlib.util
    spec = importlib.util.spec_from_file_location('vision_scenes', os.path.join(ROOT, 'vision_b200', 'scenes.py'))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def workload_scene(name):
    scenes = scenes_module()
    w = WORKLOADS[name]
    if w['kind'] == 'box_room':
        return scenes.box_room(width=w['width'], height=w['height'], max_depth=w['max_depth'],
                               dimension=w['dimension'], sampler=w['sampler'], seed=w['seed'])
    if w['kind'] == 'large_scene':
        return scenes.large_scene(width=w['width'], height=w['height'], max_depth=w['max_depth'],
                                  dimension=w['dimension'], sampler=w['sampler'], seed=w['seed'])
    if w['kind'] == 'many_lights':
        return scenes.many_lights(width=w['width'], height=w['height'], emitters=w['emitters'], seed=w['seed'],
                                  M_light=w['M_light'], history_limit=w['history_limit'],
                                  spatial_neighbours=w['spatial_neighbours'], spatial_radius=w['spatial_radius'],
                                  max_depth=w['max_depth'], sampler=w['sampler'])
    raise ValueError(name)


def sample_pixels(width, height, count, seed=5):
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(width * height, size=min(count, width * height), replace=False)).astype(np.uint32)


def measured_peaks():
    p = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get('hbm_gbs', 6650.0), 'measured'
    return 6650.0, 'fallback'


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    FIELDS = ['clocks.sm', 'clocks.max.sm', 'power.draw', 'clocks_event_reasons.hw_slowdown',
              'clocks_event_reasons.hw_thermal_slowdown', 'clocks_event_reasons.sw_thermal_slowdown',
              'clocks_event_reasons.sw_power_cap']

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.gpu), '--query-gpu=' + ','.join(self.FIELDS),
                                          '--format=csv,noheader,nounits', '-lms', '100'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['nvidia-smi unavailable']}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for line in self.lines:
            parts = [x.strip() for x in line.split(',')]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower() == 'active':
                    reasons.add(n)
        return {'sm_mhz': float(np.median(sm)) if sm else None, 'sm_max_mhz': max(mx) if mx else None,
                'reasons': sorted(reasons), 'samples': len(sm)}


def cpu_baseline(doc, spp, budget_s=12.0):
    """The oracle (a scalar C++ port of the reference integrator, with its own
    scene ingestion of the workload's scene document) on all host cores, on a
    fixed seeded subset of the workload's pixels (at most 262,144), frame after
    frame (frame indices continue past the workload's spp) until the time
    budget is used."""
    import oracle
    o = oracle.OracleScene.from_json(doc)
    threads = os.cpu_count()
    pixels = sample_pixels(o.width, o.height, min(o.width * o.height, 262144))
    o.paths(pixels[:256], 0, 1, threads=threads)  # warm-up
    frames = 0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < budget_s:
        o.paths(pixels, frames, 1, threads=threads)
        frames += 1
    dt = time.perf_counter() - t0
    paths = frames * pixels.size
    return {'value': paths / dt / 1e6, 'unit': 'Mpaths/s', 'cores': threads, 'kind': 'port',
            'sample': '%d seeded pixels x %d frames of the %dx%d workload (%d paths) in %.1f s' % (
                pixels.size, frames, o.width, o.height, paths, dt)}


def restir_cpu_frames(scene, w, frames, budget_s=None):
    """The oracle's ReSTIR frames (CPU restatement) on all host cores along the
    workload's camera spline; returns (frames done, seconds)."""
    import oracle
    from vision_b200 import scenes
    o = oracle.OracleScene(scene)
    ort = oracle.OracleRestir(o, w['width'], w['height'])
    cams = scenes.camera_spline(w['frames'], seed=3)
    threads = os.cpu_count()
    done = 0
    t0 = time.perf_counter()
    for f in range(frames):
        scene.set_camera(cams[f % len(cams)], 40.0)
        ort.frame(scene.export('camera'), scene.restir_params(f), 0, threads)
        done += 1
        if budget_s is not None and time.perf_counter() - t0 > budget_s:
            break
    return done, time.perf_counter() - t0, threads


def run_reference(args, rank):
    """Reference arm: the CPU restatement of the reference integrator on the
    host cores (the reference's CUDA/OptiX build cannot be built offline)."""
    if rank != 0:
        return
    import oracle
    w = WORKLOADS[args.workload]
    if w['kind'] not in ('box_room', 'large_scene', 'many_lights'):
        print(json.dumps({'impl': 'reference', 'unavailable': 'the reference has no %s path (a new workload of this '
                                                               'build; its CPU restatement is the plain tracer)'
                          % w['kind']}))
        return
    if w['kind'] == 'many_lights':
        # The ReSTIR frame parameters (camera transforms, resampling settings)
        # still come from the library's host-side scene layer on this arm.
        import vision_b200 as vb
        ctx = vb.Context(-1)
        scene = vb.Scene(ctx, workload_scene(args.workload)).build_accel()
        restir_cpu_frames(scene, w, args.warmup)
        frames, dt, threads = restir_cpu_frames(scene, w, args.steps)
        npix = w['width'] * w['height']
        value = frames * npix / dt / 1e6
        line = {'metric': 'Mpaths/s', 'value': value, 'unit': 'Mpaths/s', 'n_gpus': args.gpus, 'steps': frames,
                'warmup': args.warmup, 'ms_per_step': dt * 1e3 / frames, 'higher_is_better': True,
                'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
                'config': {'workload': args.workload, **{k: v for k, v in w.items() if k != 'kind'},
                           'step': 'one full ReSTIR frame (every pixel) per step'},
                'impl': 'reference',
                'cpu_baseline': {'value': value, 'unit': 'Mpaths/s', 'cores': threads, 'kind': 'port',
                                 'sample': '%d full frames of %dx%d' % (frames, w['width'], w['height'])},
                'e2e': {'value': value, 'unit': 'Mpaths/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
        print(json.dumps(line))
        return
    # The oracle's own scene ingestion: the reference arm never loads the
    # library (vision_b200 is not imported on this path).
    o = oracle.OracleScene.from_json(workload_scene(args.workload))
    threads = os.cpu_count()
    pixels = sample_pixels(o.width, o.height, min(o.width * o.height, 262144))
    npix = pixels.size
    for i in range(args.warmup):
        o.paths(pixels, i % w['spp'], 1, threads=threads)
    t0 = time.perf_counter()
    for i in range(args.steps):
        o.paths(pixels, i % w['spp'], 1, threads=threads)
    dt = time.perf_counter() - t0
    value = args.steps * npix / dt / 1e6
    line = {'metric': 'Mpaths/s', 'value': value, 'unit': 'Mpaths/s', 'n_gpus': args.gpus, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': dt * 1e3 / args.steps, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
            'config': {'workload': args.workload, **{k: v for k, v in w.items() if k != 'kind'},
                       'step': '1 spp of %d seeded pixels of the workload per step' % npix},
            'impl': 'reference',
            'cpu_baseline': {'value': value, 'unit': 'Mpaths/s', 'cores': threads, 'kind': 'port',
                             'sample': '%d seeded pixels x 1 frame (%d paths) per step' % (npix, npix)},
            'e2e': {'value': value, 'unit': 'Mpaths/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=None)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--workload', default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-sub', action='store_true',
                    help='skip the other workloads that the default run reports under `sub`')
    ap.add_argument('--schedule', default='wavefront', choices=['wavefront', 'wavefront_binned', 'persistent', 'grid'],
                    help='path scheduling of the megakernel (both give the same film)')
    ap.add_argument('--reference-spp', type=int, default=None,
                    help='radiance_cache: spp of the FP64 plain reference (default 1024; the full specification '
                         'is 65536)')
    ap.add_argument('--decompose', action='store_true',
                    help='radiance_cache: also measure relMSE at 16 spp of the plain tracer cut after 1, 2, 3 '
                         'and all bounces (what bounds the cache speed-up)')
    ap.add_argument('--rates', default=None,
                    help='serving: comma-separated arrival rates (jobs/s) measured one after another on the same '
                         'resident scenes; the first is the headline, all are listed under `sweep`')
    ap.add_argument('--spp', type=int, default=None,
                    help='override the workload spp (profiling runs on a smaller launch; reported in config)')
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 20 if args.impl == 'reference' else DEFAULT_STEPS[args.workload]
    rank = int(os.environ.get('RANK', '0'))
    world = int(os.environ.get('WORLD_SIZE', '1'))
    local_rank = int(os.environ.get('LOCAL_RANK', '0'))
    if args.impl == 'reference':
        run_reference(args, rank)
        return

    import torch
    import vision_b200 as vb
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120))
    w = dict(WORKLOADS[args.workload])
    if args.spp:
        w['spp'] = args.spp
    if args.reference_spp and w['kind'] == 'radiance_cache':
        w['reference_spp'] = args.reference_spp
    line = RUNNERS[w['kind']](args, w, rank, world, local_rank, dist)
    if rank == 0 and world == 1 and args.workload == DEFAULT_WORKLOAD and not args.no_sub:
        line['sub'] = run_sub(args, local_rank)
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


# The other workloads of the metric, run after the headline in the default
# invocation (one GPU) and reported under the line's `sub` key: the box room
# (the plain tracer's stated target configuration), the ReSTIR frame, the
# radiance cache's time to relMSE 1e-2 and a serving run of SUB_STEPS['serving']
# jobs of the seeded Poisson sequence.
SUB_STEPS = {'box_room': 100, 'many_lights': 32, 'radiance_cache': 16, 'serving': 200}


def run_sub(args, local_rank):
    out = {}
    for name, steps in SUB_STEPS.items():
        sub_args = argparse.Namespace(**vars(args))
        sub_args.workload, sub_args.steps, sub_args.warmup = name, steps, max(args.warmup, 3)
        sub_args.no_cpu_baseline, sub_args.spp = True, None
        w = dict(WORKLOADS[name])
        t0 = time.perf_counter()
        line = RUNNERS[w['kind']](sub_args, w, 0, 1, local_rank, None)
        line['wall_s'] = round(time.perf_counter() - t0, 1)
        out[name] = line
    return out


def run_plain(args, w, rank, world, local_rank, dist):
    """The plain tracer workloads (large scene, box room): one step renders
    every pixel at the workload's spp through vs_render."""
    import torch
    import vision_b200 as vb
    ctx = vb.Context(local_rank)
    scene = vb.Scene(ctx, workload_scene(args.workload))
    t0 = time.perf_counter()
    scene.build_accel()
    build_s = time.perf_counter() - t0
    scene.set_schedule(args.schedule)
    info = scene.info()
    spp = w['spp']
    npix = w['width'] * w['height']
    paths_per_step = npix * spp
    # A dedicated stream: the library and the CUDA events must share it (the
    # legacy default stream does not order against the library's own stream).
    torch_stream = torch.cuda.Stream()
    torch.cuda.set_stream(torch_stream)
    stream = torch_stream.cuda_stream

    # Algorithmic bytes per path (B_path = 32 + sum over segments of
    # 80 N_node + 36 N_tri + 180), from an instrumented render outside the timing.
    segs, nodes, tris = scene.render_stats(0, spp)
    bytes_per_path = 32.0 + (80.0 * nodes + 36.0 * tris + 180.0 * segs) / paths_per_step

    for i in range(args.warmup):
        scene.render(0, spp, stream=stream)
    torch.cuda.synchronize()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device='cuda')
    clocks = ClockSampler(torch.cuda.current_device())
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    scene.timing_enable(True)
    launches0 = vb.launch_count()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for i in range(args.steps):
        flush.zero_()  # L2 flush between timed steps (inputs are smaller than L2)
        starts[i].record()
        scene.render(0, spp, stream=stream)
        ends[i].record()
    torch.cuda.synchronize()
    launches = vb.launch_count() - launches0
    clk = clocks.stop()
    if dist:
        dist.barrier()
    step_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    render_ms, film_ms, render_launches = scene.timing_read()
    scene.timing_enable(False)
    t = torch.tensor([step_ms, render_ms], dtype=torch.float64, device='cuda')
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    step_ms, render_ms = float(t[0]), float(t[1])
    value = world * paths_per_step * args.steps / (step_ms / 1e3) / 1e6

    # End to end through the public API with host buffers: camera in, film out.
    cam = scene.export('camera', np.float32)[:16].copy()
    film_host = torch.empty((info['height'], info['width'], 4), dtype=torch.float32).pin_memory()
    film_np = film_host.numpy()
    e2e_steps = max(3, args.steps // 2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        vb.lib.vs_camera_set(scene.handle, vb._ptr(cam), 40.0)
        scene.render(0, spp)
        ctx.check(vb.lib.vs_film_download(scene.handle, vb._ptr(film_np), film_np.nbytes, vb.FILM_LINEAR), 'film')
    e2e_s = time.perf_counter() - t0
    e2e_t = torch.tensor([e2e_s], dtype=torch.float64, device='cuda')
    if dist:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_value = world * paths_per_step * e2e_steps / float(e2e_t[0]) / 1e6

    peak, peak_src = measured_peaks()
    kernel_s = render_ms / 1e3 / max(render_launches, 1)
    achieved = bytes_per_path * paths_per_step / kernel_s / 1e9
    line = {
        'metric': 'Mpaths/s', 'value': value, 'unit': 'Mpaths/s', 'n_gpus': world, 'steps': args.steps,
        'warmup': args.warmup, 'ms_per_step': step_ms / args.steps, 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
        'config': {'workload': args.workload, **{k: v for k, v in w.items() if k != 'kind'},
                   'prims': info['prim_count'], 'bvh_nodes': info['bvh_node_count'],
                   'paths_per_step': paths_per_step, 'l2': 'flushed between steps (256 MiB write)',
                   'parallelism': 'replicas%d' % world, 'scene_build_s': round(build_s, 3),
                   'schedule': args.schedule},
        'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s', 'frac': achieved / peak,
                     'peak_source': peak_src,
                     'traffic': (NCU_TRAFFIC_PER_PATH[(args.workload, args.schedule)] * paths_per_step * args.steps /
                                 max(render_launches, 1)
                                 if (args.workload, args.schedule) in NCU_TRAFFIC_PER_PATH else None),
                     'traffic_source': 'ncu dram bytes per path of the committed profile (all kernels of the '
                                       'schedule for one render) x paths per launch',
                     'kernel': {'persistent': 'k_render_regen', 'grid': 'k_render',
                                'wavefront': 'wavefront (k_wf_extend, k_wf_shade, k_wf_shadow)',
                                'wavefront_binned': 'wavefront (k_wf_extend, k_wf_shade, k_wf_shadow; binned rays)'}[
                                    args.schedule],
                     'bytes_per_path': bytes_per_path,
                     'per_path': {'segments': segs / paths_per_step, 'nodes': nodes / paths_per_step,
                                  'tris': tris / paths_per_step},
                     'kernel_ms_per_launch': kernel_s * 1e3, 'film_ms_per_launch': film_ms / max(render_launches, 1)},
        'clocks': clk,
        'e2e': {'value': e2e_value, 'unit': 'Mpaths/s', 'h2d_bytes_per_step': 64,
                'd2h_bytes_per_step': int(film_np.nbytes)},
        'gpu_launches': int(launches),
    }
    issue = NCU_ISSUE.get((args.workload, args.schedule))
    if issue:
        line['roofline'].update(issue)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line['cpu_baseline'] = cpu_baseline(workload_scene(args.workload), spp)
    return line


def run_restir(args, w, rank, world, local_rank, dist):
    """The many-light ReSTIR workload: one step = one real-time frame along
    the camera spline (frame index = step), film restarted each frame."""
    import torch
    import vision_b200 as vb
    from vision_b200 import scenes
    ctx = vb.Context(local_rank)
    scene = vb.Scene(ctx, workload_scene(args.workload))
    t0 = time.perf_counter()
    scene.build_accel()
    build_s = time.perf_counter() - t0
    info = scene.info()
    npix = w['width'] * w['height']
    cams = scenes.camera_spline(w['frames'], seed=3)
    torch_stream = torch.cuda.Stream()
    torch.cuda.set_stream(torch_stream)
    stream = torch_stream.cuda_stream
    frame = 0

    def step(stream_ptr):
        nonlocal frame
        scene.set_camera(cams[frame % len(cams)], 40.0)
        scene.restir_frame(frame, 0, stream=stream_ptr)
        frame += 1

    for _ in range(args.warmup):
        step(stream)
    torch.cuda.synchronize()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device='cuda')
    clocks = ClockSampler(torch.cuda.current_device())
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    scene.timing_enable(True)
    launches0 = vb.launch_count()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for i in range(args.steps):
        flush.zero_()
        starts[i].record()
        step(stream)
        ends[i].record()
    torch.cuda.synchronize()
    launches = vb.launch_count() - launches0
    clk = clocks.stop()
    if dist:
        dist.barrier()
    step_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    frame_ms, _, frame_launches = scene.timing_read()
    scene.timing_enable(False)
    t = torch.tensor([step_ms, frame_ms], dtype=torch.float64, device='cuda')
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    step_ms, frame_ms = float(t[0]), float(t[1])
    value = world * npix * args.steps / (step_ms / 1e3) / 1e6

    # End to end through the public API with host buffers: camera in, film out.
    film_host = torch.empty((info['height'], info['width'], 4), dtype=torch.float32).pin_memory()
    film_np = film_host.numpy()
    e2e_steps = max(3, args.steps // 2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        c2w = np.ascontiguousarray(cams[frame % len(cams)].T)
        ctx.check(vb.lib.vs_camera_set(scene.handle, vb._ptr(c2w), 40.0), 'camera')
        ctx.check(vb.lib.vs_restir_frame(scene.handle, frame, 0, None), 'restir_frame')
        frame += 1
        ctx.check(vb.lib.vs_film_download(scene.handle, vb._ptr(film_np), film_np.nbytes, vb.FILM_LINEAR), 'film')
    e2e_s = time.perf_counter() - t0
    e2e_t = torch.tensor([e2e_s], dtype=torch.float64, device='cuda')
    if dist:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_value = world * npix * e2e_steps / float(e2e_t[0]) / 1e6

    peak, peak_src = measured_peaks()
    bpp = restir_bytes_per_pixel(w['M_light'], w['spatial_neighbours'])
    frame_s = frame_ms / 1e3 / max(frame_launches, 1)
    achieved = bpp * npix / frame_s / 1e9
    line = {
        'metric': 'Mpaths/s', 'value': value, 'unit': 'Mpaths/s', 'n_gpus': world, 'steps': args.steps,
        'warmup': args.warmup, 'ms_per_step': step_ms / args.steps, 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
        'config': {'workload': args.workload, **{k: v for k, v in w.items() if k != 'kind'},
                   'path': 'one pixel of one ReSTIR frame (camera path, direct and indirect resampling)',
                   'prims': info['prim_count'], 'lights': info['light_count'],
                   'l2': 'flushed between steps (256 MiB write)',
                   'parallelism': 'replicas%d' % world, 'scene_build_s': round(build_s, 3)},
        'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s', 'frac': achieved / peak,
                     'peak_source': peak_src, 'traffic': None, 'kernel': 'restir frame (6 kernels)',
                     'bytes_per_pixel_frame': bpp, 'frame_ms': frame_s * 1e3},
        'clocks': clk,
        'e2e': {'value': e2e_value, 'unit': 'Mpaths/s', 'h2d_bytes_per_step': 64 + 4,
                'd2h_bytes_per_step': int(film_np.nbytes)},
        'gpu_launches': int(launches),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        frames, dt, threads = restir_cpu_frames(scene, w, 2, budget_s=20.0)
        line['cpu_baseline'] = {'value': frames * npix / dt / 1e6, 'unit': 'Mpaths/s', 'cores': threads,
                                'kind': 'port', 'sample': '%d full %dx%d frames of the oracle ReSTIR' % (
                                    frames, w['width'], w['height'])}
    return line


def relmse(img, ref, eps=1e-2):
    """Mean over pixels and channels of (img - ref)^2 / (ref^2 + eps)."""
    return float(np.mean((img - ref) ** 2 / (ref ** 2 + eps)))


# spp of the equal-time quality curves (plain and cached).
QUALITY_SPP = (1, 2, 4, 8, 16, 32, 64)


def run_cache(args, w, rank, world, local_rank, dist):
    """Cache-terminated rendering: throughput of the cached frames (with their
    training steps) and time to relMSE 1e-2 against an FP64 plain reference,
    next to the plain tracer's."""
    import torch
    import vision_b200 as vb
    from vision_b200 import scenes
    ctx = vb.Context(local_rank)
    sc = scenes.box_room(w['width'], w['height'], max_depth=w['max_depth'], dimension=w['dimension'],
                         sampler=w['sampler'], seed=w['seed'])
    # The reference uses another PCG stream seed, so its samples are
    # independent of the timed renders' (frames 0, 1, ... of seed `seed`).
    ref_sc = scenes.box_room(w['width'], w['height'], max_depth=w['max_depth'], dimension=w['dimension'],
                             sampler=w['sampler'], seed=w['seed'] + 7919)
    ref_scene = vb.Scene(ctx, ref_sc).build_accel()
    plain = vb.Scene(ctx, sc).build_accel()
    cached = vb.Scene(ctx, sc).build_accel()
    npix = w['width'] * w['height']
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream
    t0 = time.perf_counter()
    ref_scene.render(0, w['reference_spp'], fp64=True, stream=sp)
    ref_scene.synchronize()
    ref_s = time.perf_counter() - t0
    ref = ref_scene.film(vb.FILM_SUM64)[..., :3] / w['reference_spp']

    def timed(fn):
        torch.cuda.synchronize()
        t = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        return time.perf_counter() - t

    # Plain tracer: time and relMSE per spp.
    plain_curve = []
    for spp in QUALITY_SPP:
        dt = timed(lambda: plain.render(0, spp, stream=sp))
        plain_curve.append((spp, dt, relmse(plain.film()[..., :3], ref)))
    # Cached: warm-up training, then timed frames (training continues).
    cache = vb.RadianceCache(ctx, seed=1)
    cache.set_optimizer(lr=w['lr'])
    train_s = timed(lambda: cached.render_cached(cache, 0, w['warmup_frames'], train_samples=w['train_samples'],
                                                 stream=sp))
    cached_curve = []
    for spp in QUALITY_SPP:
        dt = timed(lambda: cached.render_cached(cache, 0, spp, train_samples=w['train_samples'], stream=sp))
        cached_curve.append((spp, dt, relmse(cached.film()[..., :3], ref)))
    # Throughput of the timed cached frames (CUDA events, L2 flushed between steps).
    flush = torch.empty(256 << 20, dtype=torch.uint8, device='cuda')
    for _ in range(args.warmup):
        cached.render_cached(cache, 0, 1, train_samples=w['train_samples'], stream=sp)
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    time.sleep(0.3)
    cached.timing_enable(True)
    launches0 = vb.launch_count()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for i in range(args.steps):
        flush.zero_()
        starts[i].record()
        cached.render_cached(cache, i, 1, train_samples=w['train_samples'], stream=sp)
        ends[i].record()
    torch.cuda.synchronize()
    launches = vb.launch_count() - launches0
    clk = clocks.stop()
    step_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    frame_ms, _, _ = cached.timing_read()
    cached.timing_enable(False)
    value = npix * args.steps / (step_ms / 1e3) / 1e6
    # End to end through the C ABI with a host film read per step.
    film_host = torch.empty((w['height'], w['width'], 4), dtype=torch.float32).pin_memory()
    film_np = film_host.numpy()
    e2e_steps = max(3, args.steps // 2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        ctx.check(vb.lib.vs_render_cached(cached.handle, cache.handle, 0, 1, w['train_samples'], vb.FILM_FP32, None),
                  'render_cached')
        ctx.check(vb.lib.vs_film_download(cached.handle, vb._ptr(film_np), film_np.nbytes, vb.FILM_LINEAR), 'film')
    e2e_value = npix * e2e_steps / (time.perf_counter() - t0) / 1e6

    def time_to(curve, extra=0.0):
        for spp, dt, r in curve:
            if r <= w['target_relmse']:
                return extra + dt, spp
        return None, None
    # Warm: the cache trained beforehand (an interactive session whose cache
    # keeps training frame after frame); cold: the warm-up training counted.
    tp, sp_p = time_to(plain_curve)
    tc, sp_c = time_to(cached_curve)
    tc_cold, _ = time_to(cached_curve, train_s)

    def time_model(curve):
        # relMSE of an unbiased estimate falls as 1/spp and the time grows as
        # spp: from the last point, the spp and time at the target.
        spp, dt, r = curve[-1]
        need = spp * r / w['target_relmse']
        return need * dt / spp, need
    tp_m, spp_p_m = time_model(plain_curve)
    tc_m, spp_c_m = time_model(cached_curve)
    decomposition = None
    if getattr(args, 'decompose', False):
        # What bounds the cache's speed-up: the plain tracer cut after d
        # bounces (emission and next-event estimates of the first d vertices)
        # against its own converged FP64 reference at equal spp.  With the
        # cache ending paths after 2 bounces, relMSE(full) / relMSE(d = 2) at
        # 16 spp, times the frame-time ratio, is the speed-up a perfect,
        # free cache would give.
        decomposition = []
        for d in (1, 2, 3, w['max_depth']):
            dsc = scenes.box_room(w['width'], w['height'], max_depth=d, dimension=w['dimension'],
                                  sampler=w['sampler'], seed=w['seed'])
            dref_sc = dict(dsc, sampler={'type': w['sampler'], 'param': {'seed': w['seed'] + 7919}})
            dref = vb.Scene(ctx, dref_sc).build_accel()
            dref.render(0, 1024, fp64=True, stream=sp)
            dref.synchronize()
            r = dref.film(vb.FILM_SUM64)[..., :3] / 1024.0
            ds = vb.Scene(ctx, dsc).build_accel()
            dt = timed(lambda: ds.render(0, 16, stream=sp))
            decomposition.append({'max_depth': d, 'relmse_16spp': relmse(ds.film()[..., :3], r), 's_16spp': dt})
            del ds, dref
    # Algorithmic flops of the network per frame: inference on every pixel's
    # query and every suffix end, training forward + backward on the samples.
    nt = w['train_samples']
    flops = 33152.0 * (npix + nt) + 99456.0 * nt
    peak_tf = 1389.6
    try:
        peak_tf = json.load(open(os.path.join(ROOT, 'MEASURED_PEAKS.json'))).get('bf16_tflops_sustained', peak_tf)
    except OSError:
        pass
    achieved_tf = flops / (frame_ms / 1e3 / args.steps) / 1e12
    line = {
        'metric': 'Mpaths/s', 'value': value, 'unit': 'Mpaths/s', 'n_gpus': world, 'steps': args.steps,
        'warmup': args.warmup, 'ms_per_step': step_ms / args.steps, 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'f32 path / bf16 network', 'data': 'synthetic',
        'config': {'workload': args.workload, **{k: v for k, v in w.items() if k != 'kind'},
                   'path': 'one cache-terminated camera path per pixel per frame, training step included',
                   'l2': 'flushed between steps (256 MiB write)', 'parallelism': 'replicas%d' % world},
        'quality': {'reference_s': ref_s, 'target_relmse': w['target_relmse'],
                    'plain': [{'spp': a, 's': b, 'relmse': c} for a, b, c in plain_curve],
                    'cached': [{'spp': a, 's': b, 'relmse': c} for a, b, c in cached_curve],
                    'cache_training_s': train_s,
                    'time_to_target_s': {'plain': tp, 'cached_warm': tc, 'cached_cold': tc_cold},
                    'spp_to_target': {'plain': sp_p, 'cached': sp_c},
                    'speedup_warm': (tp / tc) if (tp and tc) else None,
                    'speedup_cold': (tp / tc_cold) if (tp and tc_cold) else None,
                    'at_target_1_over_spp': {'plain_s': tp_m, 'plain_spp': spp_p_m, 'cached_s': tc_m,
                                             'cached_spp': spp_c_m, 'speedup_warm': tp_m / tc_m},
                    'variance_by_depth': decomposition},
        'roofline': {'bound': 'tensor', 'achieved': achieved_tf, 'peak': peak_tf, 'unit': 'TFLOP/s',
                     'frac': achieved_tf / peak_tf, 'peak_source': 'measured', 'traffic': None,
                     'kernel': 'radiance-cache frame (network share of the frame time)',
                     'flops_per_frame': flops, 'frame_ms': frame_ms / args.steps},
        'clocks': clk,
        'e2e': {'value': e2e_value, 'unit': 'Mpaths/s', 'h2d_bytes_per_step': 0,
                'd2h_bytes_per_step': int(film_np.nbytes)},
        'gpu_launches': int(launches),
    }
    return line


def serving_scenes():
    from vision_b200 import scenes
    return {'box_room': scenes.box_room(256, 256, max_depth=8, dimension=4, sampler='pcg'),
            'large_scene': scenes.large_scene(),
            'many_lights_pt': scenes.many_lights(256, 256, integrator='pt', dimension=4, max_depth=8),
            'instanced': scenes.instanced_scene()}


def serving_jobs(w, count):
    rng = np.random.default_rng(w['seed'])
    t = np.cumsum(rng.exponential(1.0 / w['rate'], count))
    res = rng.integers(0, len(w['resolutions']), count)
    spp = rng.integers(0, len(w['spp']), count)
    scn = rng.integers(0, len(w['scenes']), count)
    fb = rng.integers(0, 1 << 16, count)
    return [(float(t[i]), int(scn[i]), w['resolutions'][res[i]][0], w['resolutions'][res[i]][1],
             w['spp'][spp[i]], int(fb[i])) for i in range(count)]


def run_serving(args, w, rank, world, local_rank, dist):
    """The serving workload: jobs arrive on a seeded Poisson clock, go through
    the C-ABI server (host descriptor in, host film out) and are timed from
    submission to the film on the host."""
    import torch
    import vision_b200 as vb
    ctx = vb.Context(local_rank)
    t0 = time.perf_counter()
    built = {}
    for name, sc in serving_scenes().items():
        built[name] = vb.Scene(ctx, sc).build_accel()
    build_s = time.perf_counter() - t0
    # Algorithmic bytes per path of each scene (1 frame at its own resolution).
    bpp = {}
    for name, s in built.items():
        info = s.info()
        segs, nodes, tris = s.render_stats(0, 1)
        bpp[name] = 32.0 + (80.0 * nodes + 36.0 * tris + 180.0 * segs) / (info['width'] * info['height'])
    def make_server():
        srv = vb.Server(ctx, hbm_budget=int(w['hbm_budget_gb']) << 30, max_jobs=w['max_jobs'],
                        paths_per_batch=w['paths_per_batch'])
        return srv, {name: srv.add_scene(s) for name, s in built.items()}

    # Warm-up jobs on a separate server instance (not timed).
    warm, wids = make_server()
    for i in range(args.warmup):
        warm.result(warm.submit(wids[w['scenes'][i % 4]], 256, 256, 1, frame_begin=i), timeout=600)
    warm.close()
    peak, peak_src = measured_peaks()
    rates = [float(r) for r in args.rates.split(',')] if getattr(args, 'rates', None) else [w['rate']]
    runs = []
    for rate in rates:
        wr = dict(w, rate=rate)
        runs.append(serve_once(args, wr, make_server, bpp, peak, vb, torch))
    line = runs[0]
    line['config'].update({'scene_build_s': round(build_s, 1), 'parallelism': 'replicas%d' % world})
    if len(runs) > 1:
        # Latency and throughput per arrival rate, same job sequence (the
        # seeded arrival times scale with 1 / rate).
        line['sweep'] = [{'rate': r['config']['rate'], 'value': r['value'], 'latency_ms': r['latency_ms'],
                          'gpu_busy_s': r['server']['gpu_busy_s'], 'wall_s': r['ms_per_step'] * r['steps'] / 1e3}
                         for r in runs]
    return line


def serve_once(args, w, make_server, bpp, peak, vb, torch):
    """One serving run of args.steps jobs at arrival rate w['rate'] on a fresh
    server over the already resident scenes."""
    srv, ids = make_server()
    jobs = serving_jobs(w, args.steps)
    results = []
    done_bytes = [0]
    import queue
    pending = queue.Queue()

    def collect():
        while True:
            jid = pending.get()
            if jid is None:
                return
            out = srv.result(jid, timeout=-1.0)
            done_bytes[0] += out.nbytes
    collector = threading.Thread(target=collect)
    collector.start()
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    launches0 = vb.launch_count()
    start = time.perf_counter()
    for k, (t_arr, sidx, wd, h, spp, fb) in enumerate(jobs):
        delay = start + t_arr - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        jid = srv.submit(ids[w['scenes'][sidx]], wd, h, spp, frame_begin=fb)
        pending.put(jid)
        results.append((sidx, wd * h * spp))
    pending.put(None)
    collector.join()
    wall = time.perf_counter() - start
    launches = vb.launch_count() - launches0
    clk = clocks.stop()
    st = srv.stats()
    paths = float(sum(p for _, p in results))
    value = paths / wall / 1e6
    mean_bpp = sum(bpp[w['scenes'][s]] * p for s, p in results) / paths
    gpu_s = st['gpu_busy_s']
    achieved = mean_bpp * paths / gpu_s / 1e9 if gpu_s > 0 else None
    line = {
        'metric': 'Mpaths/s', 'value': value, 'unit': 'Mpaths/s', 'n_gpus': 1, 'steps': len(jobs),
        'warmup': args.warmup, 'ms_per_step': wall * 1e3 / len(jobs), 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
        'config': {'workload': args.workload, **{k: v for k, v in w.items() if k != 'kind'},
                   'jobs_submitted': len(jobs), 'step': 'one job (submit -> film on the host)'},
        'latency_ms': {'p50': st['p50_ms'], 'p95': st['p95_ms'], 'p99': st['p99_ms'], 'mean': st['mean_ms'],
                       'max': st['max_ms']},
        'server': {k: st[k] for k in ('completed', 'batches', 'graph_launches', 'gpu_busy_s', 'peak_jobs',
                                      'peak_bytes', 'resident_bytes', 'scratch_bytes')},
        'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                     'frac': achieved / peak if achieved else None, 'peak_source': 'measured', 'traffic': None,
                     'kernel': 'serving batches (wavefront kernels k_sv_*)', 'bytes_per_path': mean_bpp,
                     'gpu_busy_s': gpu_s},
        'clocks': clk,
        'e2e': {'value': value, 'unit': 'Mpaths/s', 'h2d_bytes_per_step': 96,
                'd2h_bytes_per_step': int(done_bytes[0] / max(len(jobs), 1))},
        'gpu_launches': int(launches),
    }
    srv.close()
    return line


RUNNERS = {'box_room': run_plain, 'large_scene': run_plain, 'many_lights': run_restir,
           'radiance_cache': run_cache, 'serving': run_serving}


if __name__ == '__main__':
    main()

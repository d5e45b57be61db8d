/*
 * vision_b200 — C ABI of the B200 spectral path-tracing hot path.
 *
 * The reference renderer (FaithZL/Vision) reaches its path tracer through a
 * C++ vtable ABI (src/sdk/vision.h:66-99, VisionRenderer: init_pipeline,
 * init_scene, add_instance, build_accel, update_camera, compile, render,
 * download_radiance) and through per-plugin DLLs built from the scene JSON
 * (src/base/node.h:109-118).  This header is the drop-in boundary for that
 * path: plain C, opaque handles, integer status codes, caller-owned buffers,
 * no exceptions and no torch or CUDA types in the signatures (streams are
 * passed as void*).
 *
 * Every entry point is thread-safe per handle: calls on one scene serialise
 * on that scene's lock.
 */
#ifndef VISION_B200_H
#define VISION_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define VS_OK 0
#define VS_E_INVALID 1     /* bad argument (null pointer, size mismatch) */
#define VS_E_UNSUPPORTED 2 /* plugin type or option outside this library; message names it */
#define VS_E_PARSE 3       /* malformed scene JSON */
#define VS_E_CUDA 4        /* CUDA runtime error; message has the CUDA error string */
#define VS_E_STATE 5       /* call out of order (e.g. render before build_accel) */
#define VS_E_NO_DEVICE 6   /* the context was created without a GPU */
#define VS_E_RANGE 7       /* size beyond a documented limit */

/* Film precision for vs_render (the reference film is FP32, normal.cpp:87-101). */
#define VS_FILM_FP32 0
#define VS_FILM_FP64 1

/* Film buffers for vs_film_download. */
#define VS_FILM_LINEAR 0     /* FP32 running mean, float4 per pixel (rt_buffer) */
#define VS_FILM_EXPOSED 1    /* tone_mapper(1 - exp(-linear * exposure)), float4 per pixel */
#define VS_FILM_SUM64 2      /* FP64 sums: double4 (r, g, b, samples) per pixel */
/* The final picture (Pipeline::final_picture, pipeline.cpp:313-329): the
 * collector's output (exposure, tone mapper) mapped once more by the tone
 * mapper, with the sRGB gamma (DISPLAY, float4; RGBA8, 8-bit RGBA rounded to
 * the nearest step) or without it (HDR: the exr/hdr outputs). */
#define VS_FILM_DISPLAY 3
#define VS_FILM_HDR 4
#define VS_FILM_RGBA8 5
/* FP64 sums of squares: double4 (r^2, g^2, b^2, 0) per pixel, kept beside
 * VS_FILM_SUM64 by vs_render with VS_FILM_FP64 from frame 0; with the sums
 * they give each pixel's sample variance (the per-pixel z-test of two films). */
#define VS_FILM_SUMSQ64 6

typedef struct vs_context vs_context;
typedef struct vs_scene vs_scene;

/* Closest-hit record: reference TriangleHit{inst_id, prim_id, bary}. */
typedef struct vs_hit {
    uint32_t inst_id; /* 0xffffffff on a miss */
    uint32_t prim_id; /* global primitive index in shape order */
    float u, v;       /* barycentric weights of vertex 1 and vertex 2 */
} vs_hit;

typedef struct vs_scene_info {
    uint32_t vertex_count;
    uint32_t prim_count;
    uint32_t instance_count;
    uint32_t material_count;
    uint32_t light_count;
    uint32_t prim_alias_count;
    uint32_t spd_floats;
    uint32_t bvh_node_count;
    uint32_t bvh_depth;
    uint32_t width;
    uint32_t height;
    uint32_t spectrum_dim;
    uint32_t max_depth;
    uint32_t accel_built;
    uint32_t two_level;  /* 1: one BVH8 per mesh under a top level over instances */
    uint32_t mesh_count; /* distinct object-space meshes */
} vs_scene_info;

/* Library version: major * 10000 + minor * 100 + patch. */
int vs_version(void);

/* Creates a context on CUDA device `device`; device = -1 makes a host-only
 * context that can parse, build and export scenes but not render. */
int vs_context_create(int device, vs_context **out);
void vs_context_destroy(vs_context *ctx);
/* Message of the last failed call on this context (never NULL). */
const char *vs_last_error(const vs_context *ctx);

/* Scene from a vision_scene.json document (reference SceneDesc::from_json,
 * src/core/scene_desc.cpp:55-61, plus JsonImporter, importers/json/importer.cpp:16-23).
 * `table_cache` may name a file that caches the RGB->spectrum table (or be NULL). */
int vs_scene_load_json(vs_context *ctx, const char *json, size_t len, const char *base_dir,
                       const char *table_cache, vs_scene **out);
void vs_scene_destroy(vs_scene *scene);

/* One vertex of an SDK instance (reference sdk::Vertex, src/sdk/vision.h:24-30):
 * position, normal, uv and a second (lightmap) uv, 40 bytes. */
typedef struct vs_vertex {
    float pos[3];
    float n[3];
    float uv[2];
    float uv2[2];
} vs_vertex;

/* Appends a mesh instance (reference VisionRenderer::add_instance with an
 * sdk::Instance, src/sdk/vision.h:52-59,75 and vision.cpp:160-188): vert_num
 * vertices, tri_num triangles as index triples, `mat4` the object-to-world
 * 4x4, column-major (mat4[4c + r]; NULL = identity), and `material` the name
 * of a material of the scene, a material node as JSON text
 * ({"type", "name", "param"}, the reference's MaterialDesc) or NULL/"" for a
 * default diffuse material.  The instance id goes to *instance_id (may be
 * NULL).  The mesh is placed in world space; call vs_scene_build_accel before
 * rendering again.  Not while a render server uses the scene. */
int vs_scene_add_instance(vs_scene *scene, const vs_vertex *vertices, uint32_t vert_num, const uint32_t *triangles,
                          uint32_t tri_num, const float *mat4, const char *material, uint32_t *instance_id);

/* Removes every shape instance and the area lights on them; materials,
 * point, spot and environment lights stay (reference
 * VisionRenderer::clear_geometries, vision.cpp:120-123).  Add geometry and
 * call vs_scene_build_accel before rendering again. */
int vs_scene_clear_geometries(vs_scene *scene);

/* Restarts the film: the next vs_render must begin at frame 0 (reference
 * VisionRenderer::invalidation, vision.cpp:104-106). */
int vs_scene_invalidate(vs_scene *scene);

/* Builds the compressed BVH8 and uploads the scene to the device
 * (reference Geometry::build_accel, src/base/mgr/geometry.cpp:36-52;
 * SDK VisionRenderer::build_accel, src/sdk/vision.h:66-80).  Shapes with the
 * same vertices and triangles share one mesh; when a mesh has several
 * instances the acceleration structure has two levels, as the reference's
 * BLAS-per-mesh plus IAS: one BVH8 per mesh over its object-space triangles
 * and a top-level BVH8 over the instances' world boxes.  Scenes whose JSON
 * sets render_setting.instancing to false keep one BVH8 over world space. */
int vs_scene_build_accel(vs_scene *scene);

/* Film resolution (reference RadianceCollector::update_resolution,
 * src/base/sensor/radiance_collector.h:58-62). Resets the film. */
int vs_set_resolution(vs_scene *scene, uint32_t width, uint32_t height);

/* Camera-to-world 4x4 (column-major, 16 floats) and vertical field of view in
 * degrees (reference VisionRenderer::update_camera, src/sdk/vision.cpp:139-160). */
int vs_camera_set(vs_scene *scene, const float *c2w16, float fov_y_deg);

int vs_scene_info_get(const vs_scene *scene, vs_scene_info *out);

/* Copies one flattened scene array (VS_EXPORT_*) into dst; `bytes` must equal
 * the array size, which vs_scene_export_size reports. */
#define VS_EXPORT_POS 0         /* float[3] per vertex, world space */
#define VS_EXPORT_NRM 1         /* float[3] per vertex, world space, unnormalised */
#define VS_EXPORT_UV 2          /* float[2] per vertex */
#define VS_EXPORT_IDX 3         /* uint32[3] per primitive */
#define VS_EXPORT_PRIM_INST 4   /* uint32 per primitive */
#define VS_EXPORT_INSTANCES 5   /* 16 bytes per instance: mat, light, first_prim, prim_count */
#define VS_EXPORT_MATERIALS 6   /* 64 bytes per material */
#define VS_EXPORT_LIGHTS 7      /* 64 bytes per area light */
#define VS_EXPORT_PRIM_ALIAS 8  /* (float prob, uint32 alias) per entry */
#define VS_EXPORT_PRIM_PMF 9    /* float per entry */
#define VS_EXPORT_LIGHT_ALIAS 10
#define VS_EXPORT_LIGHT_PMF 11
#define VS_EXPORT_CAMERA 12     /* camera block, 112 bytes */
#define VS_EXPORT_INTEGRATOR 13 /* integrator block, 48 bytes */
#define VS_EXPORT_SPD 14        /* float */
#define VS_EXPORT_MATERIAL_RGB 15 /* float[3] per material */
#define VS_EXPORT_LIGHT_RGB 16  /* float[3] per light */
#define VS_EXPORT_BVH_NODES 17  /* 80 bytes per node */
#define VS_EXPORT_BVH_TRIS 18   /* float[12] per primitive in leaf order */
#define VS_EXPORT_LUTS 19       /* float albedo tables of the compensated lobes (empty if unused) */
#define VS_EXPORT_ENV 20        /* environment light block, 160 bytes (empty without one) */
#define VS_EXPORT_ENV_TEX 21    /* float[4] per texel of the environment map */
#define VS_EXPORT_ENV_MARGINAL 22       /* alias entries over rows */
#define VS_EXPORT_ENV_MARGINAL_FUNC 23  /* float row integrals */
#define VS_EXPORT_ENV_COND 24           /* alias entries per texel (row-major) */
#define VS_EXPORT_ENV_COND_FUNC 25      /* float weight per texel */
#define VS_EXPORT_RGB2SPEC 26   /* float[4] x 3 x 64^3 RGB -> spectrum coefficient table */
/* Instancing: the distinct object-space meshes and each instance's mesh and
 * world-to-object transform (the two-level BVH traces rays in object space). */
#define VS_EXPORT_MESH_POS 27   /* float[3] per object-space vertex */
#define VS_EXPORT_MESH_IDX 28   /* uint32[3] per mesh triangle, relative to its mesh's first vertex */
#define VS_EXPORT_MESHES 29     /* 24 bytes per mesh: first vertex, vertex count, first triangle, count, hash */
#define VS_EXPORT_INST_MESH 30  /* uint32 per instance */
#define VS_EXPORT_INST_W2O 31   /* float[16] per instance, column-major world-to-object */
#define VS_EXPORT_TEXELS 32     /* float[4] per texel of the image-node textures (linear RGB, 0) */
#define VS_EXPORT_TEXTURES 33   /* 16 bytes per texture: texel offset, width, height, 0 */
int vs_scene_export_size(const vs_scene *scene, int what, size_t *bytes);
int vs_scene_export(const vs_scene *scene, int what, void *dst, size_t bytes);

/* Renders frames [frame_begin, frame_begin + frame_count), one sample per
 * pixel per frame (reference PathTracingIntegrator::render, pt.cpp:90-99),
 * accumulating into the FP32 running-mean film (and the FP64 sums when
 * film_precision = VS_FILM_FP64).  frame_begin = 0 resets the film.
 * `stream` is a cudaStream_t or NULL for the context's stream. Asynchronous. */
int vs_render(vs_scene *scene, uint32_t frame_begin, uint32_t frame_count, int film_precision, void *stream);

/* How vs_render schedules camera paths on the GPU.  All give the same film.
 * VS_SCHEDULE_GRID: one path per thread over a grid that covers all paths of
 * a launch.  VS_SCHEDULE_PERSISTENT: one resident wave of warps that keep 32
 * paths in flight each and refill the lanes of finished paths after every
 * bounce (path regeneration).  VS_SCHEDULE_WAVEFRONT (the default): waves of
 * up to 4,194,304 paths whose bounces run as separate kernels (closest hit,
 * shading sorted by material, shadow rays) over path state in device memory
 * (208 bytes per path slot, allocated on first use). */
#define VS_SCHEDULE_GRID 0
#define VS_SCHEDULE_PERSISTENT 1
#define VS_SCHEDULE_WAVEFRONT 2
/* The wavefront schedule with ray binning: before each traversal pass after
 * the camera rays, the queued rays are grouped by direction octant and the
 * cell of their origin in an 8 x 8 x 8 grid over the scene (a counting sort,
 * three small kernels), so that each warp traces rays that start close
 * together and visit children in the same order; 12 more bytes per slot. */
#define VS_SCHEDULE_WAVEFRONT_BINNED 3
int vs_render_schedule_set(vs_scene *scene, int schedule);

/* Waits for all work queued on the scene's stream. */
int vs_synchronize(vs_scene *scene);

/* Copies a film buffer (VS_FILM_*) to host memory (reference
 * VisionRenderer::download_radiance, src/sdk/vision.cpp:132-137). */
int vs_film_download(vs_scene *scene, void *dst, size_t bytes, int which);

/* Seeded ray batches against the scene's BVH.  Rays are 8 floats each:
 * origin xyz, unused, direction xyz, t_max; hits cover t in (0, t_max).
 * `_device` variants take device pointers and run on `stream`; `_host`
 * variants take host pointers and include the copies. */
int vs_trace_closest_device(vs_scene *scene, const float *rays, uint32_t n, vs_hit *hits, float *t, void *stream);
int vs_trace_closest_host(vs_scene *scene, const float *rays, uint32_t n, vs_hit *hits, float *t);
int vs_trace_any_device(vs_scene *scene, const float *rays, uint32_t n, uint32_t *occluded, void *stream);
int vs_trace_any_host(vs_scene *scene, const float *rays, uint32_t n, uint32_t *occluded);

/* Device sampler streams (parity hook for the reference's
 * IndependentSampler::start / next_1d, src/render_core/samplers/independent.cpp:24-42,
 * and the PCG32 option).  keys4 holds `count` host (px, py, sample, dim)
 * quadruples; stream i is started from keys4[4i..4i+3] with
 * kind 0 (independent: TEA seed, 24-bit LCG) or 1 (PCG32, stream `seed`), and
 * its `draws` draws go to out[i * draws ...] (host memory).  Synchronous. */
int vs_sampler_stream(vs_context *ctx, int kind, uint32_t seed, const uint32_t *keys4, uint32_t count, uint32_t draws,
                      float *out);

/* Number of kernels this library has launched since it was loaded. */
uint64_t vs_launch_count(void);

/* CUDA-event timing of the kernels vs_render launches on this scene.
 * vs_timing_enable(scene, 1) clears the record and starts timing;
 * vs_timing_read waits for the recorded events and returns the summed
 * megakernel and film-pass durations and the number of megakernel launches. */
int vs_timing_enable(vs_scene *scene, int enable);
int vs_timing_read(vs_scene *scene, double *render_ms, double *film_ms, uint32_t *render_launches);

/* Instrumented render of frames [frame_begin, frame_begin + frame_count) that
 * leaves the film untouched and returns traversal counters: out3[0] ray
 * segments traced (closest + shadow), out3[1] BVH8 nodes visited, out3[2]
 * triangle tests.  Synchronous; used to size the algorithmic bytes per path. */
int vs_render_stats(vs_scene *scene, uint32_t frame_begin, uint32_t frame_count, uint64_t *out3);

/* Allocation-free render for callers that cannot call cudaMalloc at render
 * time (a frame loop inside a fixed memory budget, an embedding application
 * whose allocator owns device memory).  No counterpart in the reference: it
 * is vs_render with the film in `film` (caller-owned device memory, float4
 * per pixel, holding the running mean of frames [0, frame_begin) when
 * frame_begin > 0) and the per-path radiance in a fixed 16 MiB array inside
 * the library, so it calls no cudaMalloc, cudaFree or allocating library
 * routine.  The first call on a device looks up that array's device address;
 * make it before any stream capture.  The address is kept for the process's
 * life, so do not call this after cudaDeviceReset on that device.
 * Resolutions above 1048576 pixels return VS_E_RANGE; a film pointer that is
 * not 16-byte aligned returns VS_E_INVALID.  All calls share the one array:
 * calls that overlap on the GPU (other streams, other threads) race and must
 * be serialised by the caller.  The scene must have been built with
 * vs_scene_build_accel. */
int vs_render_noalloc(vs_scene *scene, uint32_t frame_begin, uint32_t frame_count, float *film, void *stream);

/* Real-time ReSTIR frame for a scene loaded with integrator type "rt"
 * (reference RealTimeIntegrator::render, src/render_core/integrators/rt.cpp:144-160):
 * direct pass (ReSTIRDI shader0/shader1, ReSTIR/direct.cpp:519-557,638-674),
 * indirect pass (ReSTIRGI initial/temporal/spatial, ReSTIR/indirect.cpp:354-362)
 * and the combine kernel (rt.cpp:118-126), which adds direct + indirect into
 * the FP32 film as sample `film_index` of its running mean (0 restarts it).
 * `frame_index` selects the sampler streams and the reservoir/surface buffer
 * parity.  The camera of the previous vs_restir_frame call provides the
 * motion vectors (Sensor::store_prev_data, sensor.cpp:99-103); the first
 * frame after a reset uses the current camera.  Asynchronous on `stream`. */
int vs_restir_frame(vs_scene *scene, uint32_t frame_index, uint32_t film_index, void *stream);

/* Clears the ReSTIR history (surfaces, reservoirs, previous camera)
 * (ReSTIRDI/ReSTIRGI::prepare, direct.cpp:676-686, indirect.cpp:377-391). */
int vs_restir_reset(vs_scene *scene);

/* Parameter block that vs_restir_frame(scene, frame_index, ...) would use now
 * (resampling settings, camera transforms, previous camera):
 * VS_RESTIR_PARAMS_BYTES bytes.  Works on host-only contexts. */
#define VS_RESTIR_PARAMS_BYTES 448
int vs_restir_params(const vs_scene *scene, uint32_t frame_index, void *dst, size_t bytes);

/* Copies a per-pixel ReSTIR buffer of the last frame to host memory. */
#define VS_RESTIR_DI_RADIANCE 0  /* float4: direct radiance (linear sRGB) */
#define VS_RESTIR_GI_RADIANCE 1  /* float4: indirect radiance */
#define VS_RESTIR_MOTION 2       /* float2: motion vector in pixels */
#define VS_RESTIR_SURFACES 3     /* 64 bytes: SurfaceData of the frame */
#define VS_RESTIR_DI_RESERVOIRS 4 /* 64 bytes: direct reservoirs after spatial reuse */
#define VS_RESTIR_GI_RESERVOIRS 5 /* 64 bytes: indirect reservoirs after spatial reuse */
#define VS_RESTIR_HIT_BSDF 6     /* 32 bytes: BSDF sample of the direct pass */
#define VS_RESTIR_GI_SAMPLES 7   /* 64 bytes: initial indirect samples */
/* Of the last frame rendered with the denoiser on: */
#define VS_RESTIR_DENOISED 8      /* float4: the SVGF output (illumination * albedo + emission) */
#define VS_RESTIR_GBUFFER 9       /* 32 bytes: PixelGeometry (normal + width, film position,
                                     depth gradient, linear depth; -1: miss) */
#define VS_RESTIR_SVGF_ALBEDO 10  /* float4: material albedo, linear sRGB */
#define VS_RESTIR_SVGF_EMISSION 11 /* float4: emission seen by the camera ray */
#define VS_RESTIR_SVGF_DATA 12    /* 32 bytes: SVGFData (illumination, variance, history, moments)
                                     after the last a-trous pass */
#define VS_RESTIR_SVGF_MOTION 13  /* float2: G-buffer motion vector in pixels */
#define VS_RESTIR_SVGF_HISTORY 14 /* float: history length */
int vs_restir_download(vs_scene *scene, int which, void *dst, size_t bytes);

/* SVGF denoiser of the real-time frame (src/render_core/denoisers/SVGF/,
 * SVGF::dispatch svgf.cpp:86-101; the switch the reference sets from its GUI,
 * svgf.cpp:22).  When on, every vs_restir_frame ends with the SVGF passes over
 * the frame's film: a G-buffer of the camera rays (FrameBuffer::compute_geom
 * and compute_gradient), demodulation by the material albedo, temporal
 * reprojection with history, the moment filter, N a-trous passes and
 * modulation, the result read with VS_RESTIR_DENOISED.  Its settings come
 * from the integrator's "denoiser" node ({"type": "svgf", "param": {N, alpha,
 * moments_alpha, history_limit, moments_filter_radius, sigma_rt,
 * sigma_normal}}, the reference's defaults otherwise); vs_restir_reset clears
 * its history too.  Unlike the reference, whose moment filter and a-trous
 * passes overwrite the buffer they read, each pass reads one buffer and
 * writes another, so the output does not depend on thread scheduling. */
int vs_denoiser_enable(vs_scene *scene, int on);
/* The 48-byte SVGF settings block (N, alpha, moments_alpha, history_limit,
 * moments_filter_radius, sigma_rt, sigma_normal, reproject, filter_moments).
 * Works on host-only contexts. */
#define VS_DENOISER_PARAMS_BYTES 48
int vs_denoiser_params(const vs_scene *scene, void *dst, size_t bytes);

/* Render-job server: continuous batching of vs_render-equivalent jobs of mixed
 * resolution and spp over resident scenes.  No reference counterpart (the
 * reference renders one scene interactively); it serves the path above.
 * A native scheduler thread admits jobs while job slots and `hbm_budget`
 * bytes allow: the budget covers the resident scenes' device memory (counted
 * by vs_server_add_scene, which fails with VS_E_RANGE when a scene does not
 * fit), the two batch buffers of `paths_per_batch` paths reserved at creation
 * and each admitted job's float4 film.  The scheduler then keeps the GPU
 * busy with batches of whole frames from all admitted jobs, each batch one
 * CUDA-graph launch (work-table upload, persistent path kernel, film pass).
 * A job's film equals vs_render of the same scene, camera, resolution and
 * frames [frame_begin, frame_begin + spp).  Path-tracing scenes must use 4
 * hero wavelengths.
 * Real-time scenes (integrator "rt") are served with their ReSTIR buffers
 * resident: vs_server_add_scene allocates the scene's reservoirs, surfaces,
 * film and frame scratch at its resolution and counts them with the scene.
 * A job on such a scene renders spp ReSTIR frames (frame indices frame_begin
 * ..., one frame per batch, jobs of one scene in submission order) at the
 * scene's resolution with the job's camera; its film is the running mean of
 * its frames and equals vs_camera_set + vs_restir_frame(frame_begin + i, i)
 * on the scene.  The reservoirs and the previous camera carry over from one
 * job to the next, so a client's successive jobs continue one temporal
 * history; the server drives the scene's camera and film while it holds it.
 * Scenes must stay alive while the server uses them.  vs_server_destroy waits
 * for submitted jobs. */
typedef struct vs_server vs_server;
typedef struct vs_job_desc {
    uint32_t scene;         /* id from vs_server_add_scene */
    uint32_t width, height;
    uint32_t spp;           /* frames rendered; one path per pixel per frame */
    uint32_t frame_begin;   /* first frame index (sampler streams) */
    float fov_y_deg;        /* <= 0: the scene's camera field of view */
    int use_c2w;            /* 0: the scene's camera transform */
    float c2w[16];          /* camera-to-world, column-major */
} vs_job_desc;
typedef struct vs_server_stats {
    uint64_t submitted, completed, batches, graph_launches, kernel_launches;
    double paths;           /* paths of completed jobs */
    double wall_s;          /* first submission to last completion */
    double gpu_busy_s;      /* summed batch durations on the GPU */
    double p50_ms, p95_ms, p99_ms, mean_ms, max_ms; /* submission -> film on the host */
    uint64_t peak_bytes;    /* largest admitted job memory */
    uint32_t peak_jobs;     /* most jobs in flight at once */
    uint64_t resident_bytes; /* device memory of the resident scenes */
    uint64_t scratch_bytes;  /* the two batch buffers reserved at creation */
} vs_server_stats;
int vs_server_create(vs_context *ctx, uint64_t hbm_budget, uint32_t max_jobs, uint64_t paths_per_batch,
                     vs_server **out);
void vs_server_destroy(vs_server *server);
int vs_server_add_scene(vs_server *server, vs_scene *scene, uint32_t *scene_id);
/* Non-blocking; thread-safe. */
int vs_server_submit(vs_server *server, const vs_job_desc *job, uint64_t *job_id);
int vs_server_poll(vs_server *server, uint64_t job_id, int *done);
/* Waits up to timeout_s (< 0: no limit), copies the film (float4 per pixel)
 * and releases the job. */
int vs_server_result(vs_server *server, uint64_t job_id, float *dst, size_t bytes, double timeout_s);
int vs_server_stats_get(vs_server *server, vs_server_stats *out);
/* Message of the server's last failed call. */
const char *vs_server_last_error(const vs_server *server);

/* Radiance-cache MLP (no reference counterpart): 64 BF16 inputs, 4 hidden
 * layers of 64 with ReLU, 3 outputs, no biases; BF16 weights and activations
 * with FP32 accumulation on the tcgen05 tensor cores; FP32 master weights
 * trained with Adam on the mean relative L2 loss
 * sum_c (y_c - t_c)^2 / (y_c^2 + 0.01) / (3 n).  Feature rows are 64 BF16
 * values (128 bytes, 16-byte aligned); outputs and targets are float4 per row
 * (r, g, b, unused).  Pointers passed to _infer and _train are device
 * pointers; both run asynchronously on `stream`. */
#define VS_CACHE_PARAMS 16576
typedef struct vs_cache vs_cache;
/* Weights initialised uniformly in +-sqrt(6 / fan_in) from `seed`. */
int vs_cache_create(vs_context *ctx, uint64_t seed, vs_cache **out);
void vs_cache_destroy(vs_cache *cache);
/* Master weights W[l][in][out], layers 0..4 (4 x 64 x 64, then 64 x 3). */
int vs_cache_get_weights(vs_cache *cache, float *w, size_t count);
int vs_cache_set_weights(vs_cache *cache, const float *w, size_t count);
int vs_cache_set_optimizer(vs_cache *cache, float lr, float beta1, float beta2, float eps);
int vs_cache_infer(vs_cache *cache, const uint16_t *features, uint32_t n, float *out4, void *stream);
/* One training step on n samples; update = 0 computes the gradient and loss
 * without changing the weights. */
int vs_cache_train(vs_cache *cache, const uint16_t *features, const float *targets4, uint32_t n, int update,
                   void *stream);
/* Gradient (same layout as the weights) and loss of the last vs_cache_train. */
int vs_cache_gradient(vs_cache *cache, float *grad, size_t count, double *loss);
/* vs_render with paths that stop after two bounces into the radiance cache:
 * each pixel's path adds its emission and next-event estimates for two
 * bounces, then the cache's prediction at the third vertex times the path
 * throughput.  The cache's three outputs are the spectral radiance at the
 * path's three hero wavelengths (the hero wavelength is one of its inputs),
 * so scenes must use 3 hero wavelengths.  With train_samples > 0, that many
 * paths per frame (a strided pixel subset moving every frame) continue two
 * bounces further and the cache takes one Adam step per frame on their
 * suffix radiance plus the cache at the suffix end. */
int vs_render_cached(vs_scene *scene, vs_cache *cache, uint32_t frame_begin, uint32_t frame_count,
                     uint32_t train_samples, int film_precision, void *stream);

/* Copies a buffer of the last vs_render_cached frame to host memory: the
 * per-pixel query vertices and the training samples of that frame. */
#define VS_CACHE_QUERY_FEATURES 0   /* npix x 64 BF16: features of the query vertices */
#define VS_CACHE_QUERY_RECORDS 1    /* npix x 64 bytes: throughput, wavelengths, pdfs, gathered rgb + valid */
#define VS_CACHE_QUERY_OUTPUT 2     /* npix float4: cache output at the query vertices */
#define VS_CACHE_TRAIN_FEATURES 3   /* n_train x 64 BF16: features of the training vertices */
#define VS_CACHE_TRAIN_RECORDS 4    /* n_train x 64 bytes: suffix radiance + bootstrap flag, suffix throughput,
                                       wavelengths, pdfs */
#define VS_CACHE_SUFFIX_FEATURES 5  /* n_train x 64 BF16: features of the suffix ends */
#define VS_CACHE_SUFFIX_OUTPUT 6    /* n_train float4: cache output at the suffix ends */
#define VS_CACHE_TARGETS 7          /* n_train float4: training targets */
int vs_cache_download(vs_scene *scene, int which, void *dst, size_t bytes);

/* Albedo tables of the energy-compensated lobes (164864 floats: PureReflection
 * 32^2, Dielectric and DielectricInv 32^3 x 2, Specular 32^3).  which = 0: the
 * values the renderer uses (the reference's precomputed_table.h); which = 1:
 * the same tables regenerated from the lobe definitions (apps/precompute's
 * job), cached in cache_path.  No device work. */
int vs_albedo_luts(int which, const char *cache_path, float *out, size_t count);

/* Regenerates the albedo tables on the context's GPU with strata^2 stratified
 * samples per cell (strata = 32 evaluates the same estimator as
 * vs_albedo_luts(1, ...); the reference's apps/precompute used 2^21 samples,
 * material.h:121-163).  out holds `count` = the table's float count.
 * strata in [1, 4096], else VS_E_RANGE; VS_E_NO_DEVICE on host-only contexts. */
int vs_albedo_luts_gpu(vs_context *ctx, uint32_t strata, float *out, size_t count);

/* RGB -> sigmoid coefficients with the uplift table (reference
 * RGBToSpectrumTable::decode_albedo / decode_unbound, hero.cpp:92-141).
 * mode 0 = albedo (out[3] = luminance), 1 = unbound (out[3] = scale). */
int vs_rgb_to_spectrum(vs_context *ctx, const char *table_cache, const float *rgb3, int mode, float *out4);

#ifdef __cplusplus
}
#endif

#endif /* VISION_B200_H */

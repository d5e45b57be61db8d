// Render-job server: continuous batching of path-tracing jobs of mixed
// resolution and spp over scenes resident on one device (server.cu).
#pragma once

#include <cstdint>
#include <functional>
#include <string>

#include <cuda_runtime.h>

#include "vs_devscene.h"

namespace vs {

// Resident scenes per server and work items per batch.
constexpr uint32_t kMaxServeScenes = 8;
constexpr uint32_t kMaxServeItems = 256;

struct ServeJob {
    uint32_t scene;       // id from Server::add_scene
    Camera cam;           // sensor of the job (resolution, transform)
    uint32_t frame_begin; // first frame (sampler stream); frames frame_begin .. frame_begin + spp - 1
    uint32_t spp;
};

struct ServeStats {
    uint64_t submitted, completed, rejected;
    uint64_t batches, graph_launches, kernel_launches;
    double paths;            // paths of completed jobs
    double wall_s;           // first submission to last completion
    double gpu_busy_s;       // summed batch durations (CUDA events)
    double p50_ms, p95_ms, p99_ms, mean_ms, max_ms;  // submit -> film on the host
    uint64_t peak_bytes;     // largest admitted job memory
    uint32_t peak_jobs;      // largest number of jobs in flight
    uint64_t resident_bytes; // device memory of the resident scenes
    uint64_t scratch_bytes;  // the two batch buffers reserved at creation
};

// A resident real-time (ReSTIR) scene driven by the server.  `frame` renders
// one ReSTIR frame of the scene with the job's sensor into the scene's own
// film (film_index 0 restarts the running mean) on `stream` and adds its
// kernel launches to *launches; `film` is that film (float4 per pixel).  The
// scene's reservoirs, surfaces and previous camera stay resident between
// calls, so consecutive jobs on the scene continue one temporal history.
struct RtServeHooks {
    std::function<int(const Camera &cam, uint32_t frame, uint32_t film_index, cudaStream_t stream,
                      unsigned *launches, std::string &err)>
        frame;
    const float4 *film = nullptr;
};

class Server;

// Status codes follow include/vision_b200.h (0 = OK); `err` gets the message.
int server_create(int device, uint64_t hbm_budget, uint32_t max_jobs, uint64_t paths_per_batch, Server **out,
                  std::string &err);
void server_destroy(Server *s);
// `bytes`: the scene's device memory, counted against the HBM budget for as
// long as the server holds the scene.
int server_add_scene(Server *s, const DeviceScene &scene, uint64_t bytes, uint32_t *id, std::string &err);
// A real-time scene: `bytes` counts its geometry and its resident per-pixel
// buffers (reservoirs, surfaces, film), all allocated before the call.  Jobs
// on it render at the scene's resolution, one frame per batch, in submission
// order.
int server_add_rt_scene(Server *s, const Camera &cam, uint64_t bytes, RtServeHooks hooks, uint32_t *id,
                        std::string &err);
// The sensor of a resident scene (its camera when it was added).
int server_scene_camera(Server *s, uint32_t id, const Camera **cam, std::string &err);
int server_submit(Server *s, const ServeJob &job, uint64_t *id, std::string &err);
// done = 1 when the job's film is on the host.
int server_poll(Server *s, uint64_t id, int *done, std::string &err);
// Waits (timeout_s < 0: forever) and copies the film (float4 per pixel,
// running mean over the job's frames) to dst; releases the job.
int server_result(Server *s, uint64_t id, float *dst, size_t bytes, double timeout_s, std::string &err);
void server_stats(Server *s, ServeStats *out);

}  // namespace vs

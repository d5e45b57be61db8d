// Render-job server: continuous batching of path-tracing jobs of mixed
// resolution and spp over scenes resident on one device.
//
// A native scheduler thread admits submitted jobs while job slots and the HBM
// budget allow (each job holds its float4 film on the device), and keeps the
// GPU busy with batches: every batch takes whole frames from all admitted jobs
// (a fair share each, then the leftover capacity in admission order), so jobs
// that arrive while others render start at the next batch and their work
// overlaps.  A batch is one CUDA-graph launch: the work table upload (pinned
// host -> device), then the batch's paths as wavefront waves (k_sv_generate
// maps each slot to its job, scene, pixel and frame; per bounce k_sv_extend,
// k_sv_shade<C> for every shading class C and k_sv_shadow run the shared
// wavefront bodies with each slot's own scene), then the film pass
// k_serve_film (each job's running mean in frame order).  Two graph instances
// with their own tables, path slots and radiance buffers alternate, so the
// host prepares batch i + 1 while batch i runs.  Results are copied to pinned host memory in stream order after the
// job's last batch; latency is submission to that copy.
//
// A job's film equals vs_render of the same scene, camera, resolution and
// frames: every path uses the same sampler streams and the film the same
// running mean in the same frame order, whatever the batch composition.
#include "vs_wavefront.cuh"
#include "vs_launch.h"
#include "vs_server.h"
#include "../../include/vision_b200.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

namespace vs {

namespace {

constexpr int SN = 4;  // hero wavelengths of served scenes

struct ServeItem {
    Camera cam;
    uint32_t scene;
    uint32_t frame_begin;   // sampler frame of the item's first frame
    uint32_t frame_count;
    uint32_t film_index;    // running-mean index of the first frame
    uint64_t path_begin;    // first path of the item in the batch
    uint64_t pix_begin;     // first film pixel of the item in the batch
    float4 *film;
    uint32_t npix;
    uint32_t pad;
};
static_assert(sizeof(ServeItem) == 176, "ServeItem layout");

struct ServeTable {
    unsigned long long next;  // path counter of the persistent kernel (0 at upload)
    unsigned long long total_paths;
    unsigned long long total_pix;
    uint32_t count;
    uint32_t pad;
    ServeItem items[kMaxServeItems];
};

__device__ __forceinline__ uint32_t find_item(const unsigned long long *begin, uint32_t count, uint64_t p) {
    uint32_t lo = 0, hi = count - 1u;
    while (lo < hi) {
        uint32_t mid = (lo + hi + 1u) >> 1;
        if (begin[mid] <= p) lo = mid;
        else hi = mid - 1u;
    }
    return lo;
}

// Path slots of one wavefront wave of a batch.
constexpr uint64_t kServeWaveSlots = 1ull << 22;

// The resident scenes, copied into shared memory by each CTA.
struct SharedScenes {
    const DeviceScene *s;
    __device__ __forceinline__ const DeviceScene &operator()(uint32_t id) const { return s[id]; }
};

__device__ __forceinline__ void load_scenes(const DeviceScene *scenes, DeviceScene *dst) {
    const uint32_t *src = reinterpret_cast<const uint32_t *>(scenes);
    uint32_t *d = reinterpret_cast<uint32_t *>(dst);
    const uint32_t words = static_cast<uint32_t>(sizeof(DeviceScene) * kMaxServeScenes / 4);
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) d[i] = src[i];
    __syncthreads();
}

// Camera paths of the wave that starts at batch path `base`: slot i holds
// batch path base + i, mapped to its item (job), pixel and frame.
__global__ void __launch_bounds__(128) k_sv_generate(const DeviceScene *scenes, const ServeTable *tab,
                                                     const __grid_constant__ WfBuffers b, uint64_t base,
                                                     float4 *radiance) {
    __shared__ DeviceScene s_scene[kMaxServeScenes];
    __shared__ unsigned long long s_begin[kMaxServeItems];
    const uint32_t count = tab->count;
    const uint64_t total = tab->total_paths;
    for (uint32_t i = threadIdx.x; i < count; i += blockDim.x) s_begin[i] = tab->items[i].path_begin;
    load_scenes(scenes, s_scene);
    const uint32_t n = base < total ? static_cast<uint32_t>(min(static_cast<uint64_t>(b.capacity), total - base)) : 0u;
    if (blockIdx.x == 0 && threadIdx.x < kWfCounters) b.count[threadIdx.x] = threadIdx.x == 0 ? n : 0u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint64_t p = base + i;
        const uint32_t k = find_item(s_begin, count, p);
        const ServeItem &it = tab->items[k];
        const uint64_t local = p - s_begin[k];
        const uint32_t npix = it.npix;
        const uint32_t f = static_cast<uint32_t>(local / npix);
        const uint32_t pix = static_cast<uint32_t>(local - static_cast<uint64_t>(f) * npix);
        const uint32_t w = it.cam.width;
        const DeviceScene &s = s_scene[it.scene];
        PathState<SN> ps;
        path_start<SN>(s, it.cam, pix % w, pix / w, it.frame_begin + f, ps);
        if (s.ip.max_depth == 0u) {
            radiance[p] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
            continue;
        }
        wf::store<SN>(b, i, ps, it.scene);
        b.queue[0][i] = i;
    }
}

__global__ void __launch_bounds__(128) k_sv_extend(const DeviceScene *scenes, const __grid_constant__ WfBuffers b,
                                                   uint32_t cur) {
    __shared__ DeviceScene s_scene[kMaxServeScenes];
    load_scenes(scenes, s_scene);
    wf::extend<kLevelsAny>(SharedScenes{s_scene}, b, cur);
}

// Shading of class C (0: misses, 1 + MaterialType: hits of that material).
template <uint32_t C>
__global__ void __launch_bounds__(128) k_sv_shade(const DeviceScene *scenes, const __grid_constant__ WfBuffers b,
                                                  uint32_t cur, uint64_t base, float4 *radiance) {
    __shared__ DeviceScene s_scene[kMaxServeScenes];
    load_scenes(scenes, s_scene);
    wf::shade<SN, C>(SharedScenes{s_scene}, b, cur, base, radiance);
}

__global__ void __launch_bounds__(128) k_sv_shadow(const DeviceScene *scenes, const __grid_constant__ WfBuffers b,
                                                   uint64_t base, float4 *radiance) {
    __shared__ DeviceScene s_scene[kMaxServeScenes];
    load_scenes(scenes, s_scene);
    wf::shadow<kLevelsAny>(SharedScenes{s_scene}, b, base, radiance);
}

// NormalRadianceCollector::add_sample (normal.cpp:87-101) per job pixel over
// the item's frames in order.
__global__ void k_serve_film(const ServeTable *tab, const float4 *radiance) {
    __shared__ unsigned long long s_begin[kMaxServeItems];
    const uint32_t count = tab->count;
    const uint64_t total = tab->total_pix;
    for (uint32_t i = threadIdx.x; i < count; i += blockDim.x) s_begin[i] = tab->items[i].pix_begin;
    __syncthreads();
    if (count == 0) return;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t q = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; q < total; q += stride) {
        const uint32_t k = find_item(s_begin, count, q);
        const ServeItem &it = tab->items[k];
        const uint32_t pix = static_cast<uint32_t>(q - s_begin[k]);
        float4 acc = it.film_index == 0 ? make_float4(0, 0, 0, 0) : it.film[pix];
        for (uint32_t f = 0; f < it.frame_count; ++f) {
            float4 v = radiance[it.path_begin + static_cast<uint64_t>(f) * it.npix + pix];
            bool bad = isnan(v.x) || isnan(v.y) || isnan(v.z) || isinf(v.x) || isinf(v.y) || isinf(v.z);
            if (bad) v = make_float4(0, 0, 0, 0);
            float a = 1.0f / static_cast<float>(it.film_index + f + 1u);
            acc.x = acc.x + a * (v.x - acc.x);
            acc.y = acc.y + a * (v.y - acc.y);
            acc.z = acc.z + a * (v.z - acc.z);
            acc.w = acc.w + a * (v.w - acc.w);
        }
        it.film[pix] = acc;
    }
}

using Clock = std::chrono::steady_clock;

struct Job {
    uint64_t id = 0;
    ServeJob desc{};
    uint32_t npix = 0;
    uint64_t bytes = 0;       // device memory counted against the budget
    uint64_t host_bytes = 0;  // the film on the host (float4 per pixel)
    bool rt = false;          // frames of a resident real-time scene
    float4 *film = nullptr;
    float *host = nullptr;   // pinned result
    uint32_t scheduled = 0;  // frames put into batches
    bool done = false;
    bool failed = false;
    Clock::time_point t_submit, t_done;
};

struct Inflight {
    int slot;
    std::vector<std::shared_ptr<Job>> finishing;
};

}  // namespace

class Server {
public:
    int device = 0;
    uint64_t budget = 0, scratch = 0;
    uint32_t max_jobs = 0;
    uint64_t batch_paths = 0;
    cudaStream_t stream = nullptr;
    DeviceScene *d_scenes = nullptr;
    uint32_t nscenes = 0;
    Camera scene_cam[kMaxServeScenes];
    bool scene_rt[kMaxServeScenes] = {};
    RtServeHooks rt_hooks[kMaxServeScenes];
    ServeTable *h_tab[2] = {nullptr, nullptr};
    ServeTable *d_tab[2] = {nullptr, nullptr};
    float4 *d_rad[2] = {nullptr, nullptr};
    WfBuffers wfb[2] = {};
    void *wf_mem[2] = {nullptr, nullptr};
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    uint32_t graph_depth = 0;   // bounce iterations captured in the graphs
    uint32_t need_depth = 0;    // largest max_depth of the resident scenes
    unsigned graph_kernels = 0; // kernel nodes per graph
    cudaEvent_t ev_start[2] = {nullptr, nullptr}, ev_end[2] = {nullptr, nullptr};

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Job>> pending;
    std::vector<std::shared_ptr<Job>> active;  // admitted, in admission order
    std::unordered_map<uint64_t, std::shared_ptr<Job>> jobs;
    std::deque<Inflight> inflight;
    uint64_t next_id = 1;
    uint64_t mem_used = 0;
    uint64_t resident = 0;  // device memory of the resident scenes
    uint64_t batch_no = 0;
    bool stop = false;
    std::string error;
    std::thread worker;

    // Statistics (under mu).
    ServeStats st{};
    std::vector<double> latencies_ms;
    bool any_submit = false;
    Clock::time_point t_first, t_last;

    ~Server() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv_work.notify_all();
        if (worker.joinable()) worker.join();
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        for (auto &kv : jobs) {
            if (kv.second->film) cudaFree(kv.second->film);
            if (kv.second->host) cudaFreeHost(kv.second->host);
        }
        for (int k = 0; k < 2; ++k) {
            if (graph[k]) cudaGraphExecDestroy(graph[k]);
            if (h_tab[k]) cudaFreeHost(h_tab[k]);
            if (d_tab[k]) cudaFree(d_tab[k]);
            if (d_rad[k]) cudaFree(d_rad[k]);
            if (wf_mem[k]) cudaFree(wf_mem[k]);
            if (ev_start[k]) cudaEventDestroy(ev_start[k]);
            if (ev_end[k]) cudaEventDestroy(ev_end[k]);
        }
        if (d_scenes) cudaFree(d_scenes);
        if (stream) cudaStreamDestroy(stream);
    }

    cudaError_t init() {
        cudaError_t e = cudaSetDevice(device);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaMalloc(&d_scenes, sizeof(DeviceScene) * kMaxServeScenes);
        if (e == cudaSuccess) e = cudaMemset(d_scenes, 0, sizeof(DeviceScene) * kMaxServeScenes);
        for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
            e = cudaHostAlloc(&h_tab[k], sizeof(ServeTable), cudaHostAllocDefault);
            if (e == cudaSuccess) std::memset(h_tab[k], 0, sizeof(ServeTable));
            if (e == cudaSuccess) e = cudaMalloc(&d_tab[k], sizeof(ServeTable));
            if (e == cudaSuccess) e = cudaMalloc(&d_rad[k], batch_paths * sizeof(float4));
            if (e == cudaSuccess) e = cudaEventCreate(&ev_start[k]);
            if (e == cudaSuccess) e = cudaEventCreate(&ev_end[k]);
        }
        for (int k = 0; k < 2 && e == cudaSuccess; ++k) e = alloc_slots(k);
        if (e == cudaSuccess) e = capture(1);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e == cudaSuccess) worker = std::thread([this] { run(); });
        return e;
    }

    static uint32_t wave_slots(uint64_t batch_paths) {
        return static_cast<uint32_t>(std::min<uint64_t>(batch_paths, kServeWaveSlots));
    }

    // Path slots of graph instance k (one wave), one allocation.
    cudaError_t alloc_slots(int k) {
        const uint32_t n = wave_slots(batch_paths);
        const size_t bytes = static_cast<size_t>(n) * kWfBytesPerSlot + 16 * 16 + 4 * kWfCounters + 256;
        cudaError_t e = cudaMalloc(&wf_mem[k], bytes);
        if (e != cudaSuccess) return e;
        char *p = static_cast<char *>(wf_mem[k]);
        auto take = [&](size_t sz) {
            char *r = p;
            p += (sz + 15) & ~size_t(15);
            return r;
        };
        WfBuffers &b = wfb[k];
        b.capacity = n;
        b.o = reinterpret_cast<float4 *>(take(16ull * n));
        b.d = reinterpret_cast<float4 *>(take(16ull * n));
        b.tp = reinterpret_cast<float4 *>(take(16ull * n));
        b.lam = reinterpret_cast<float4 *>(take(16ull * n));
        b.pdf = reinterpret_cast<float4 *>(take(16ull * n));
        b.L = reinterpret_cast<float4 *>(take(16ull * n));
        b.st = reinterpret_cast<uint4 *>(take(16ull * n));
        b.hit = reinterpret_cast<Hit *>(take(16ull * n));
        b.queue[0] = reinterpret_cast<uint32_t *>(take(4ull * n));
        b.queue[1] = reinterpret_cast<uint32_t *>(take(4ull * n));
        b.sh_o = reinterpret_cast<float4 *>(take(16ull * n));
        b.sh_d = reinterpret_cast<float4 *>(take(16ull * n));
        b.sh_c = reinterpret_cast<float4 *>(take(16ull * n));
        b.tq = reinterpret_cast<uint32_t *>(take(4ull * n * kWfClasses));
        b.count = reinterpret_cast<uint32_t *>(take(4 * kWfCounters));
        return cudaSuccess;
    }

    // (Re)captures both batch graphs with `depth` bounce iterations per wave.
    // No batch may be in flight.
    cudaError_t capture(uint32_t depth) {
        // One k_sv_shade<C> per shading class, in the graph and here.
        static_assert(kWfClasses == 8, "k_sv_shade launches cover classes 0..7");
        int sms = 0, per_ext = 0, per_shadow = 0, per_gen = 0, per_shade[kWfClasses] = {};
        cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_gen, k_sv_generate, 128, 0);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_ext, k_sv_extend, 128, 0);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_shade[0], k_sv_shade<0>, 128, 0);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_shade[1], k_sv_shade<1>, 128, 0);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_shade[2], k_sv_shade<2>, 128, 0);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_shade[3], k_sv_shade<3>, 128, 0);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_shade[4], k_sv_shade<4>, 128, 0);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_shade[5], k_sv_shade<5>, 128, 0);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_shade[6], k_sv_shade<6>, 128, 0);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_shade[7], k_sv_shade<7>, 128, 0);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_shadow, k_sv_shadow, 128, 0);
        if (e != cudaSuccess) return e;
        auto grid_of = [&](int per) { return static_cast<unsigned>(std::max(1, sms * std::max(per, 1))); };
        const unsigned g_gen = grid_of(per_gen), g_ext = grid_of(per_ext), g_shadow = grid_of(per_shadow);
        unsigned g_shade[kWfClasses];
        for (uint32_t c = 0; c < kWfClasses; ++c) g_shade[c] = grid_of(per_shade[c]);
        const unsigned film_grid = static_cast<unsigned>(std::max(1, sms * 4));
        const uint32_t slots = wave_slots(batch_paths);
        const uint64_t waves = (batch_paths + slots - 1) / slots;
        for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
            if (graph[k]) {
                cudaGraphExecDestroy(graph[k]);
                graph[k] = nullptr;
            }
            cudaGraph_t g = nullptr;
            e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) break;
            cudaMemcpyAsync(d_tab[k], h_tab[k], sizeof(ServeTable), cudaMemcpyHostToDevice, stream);
            for (uint64_t w = 0; w < waves; ++w) {
                const uint64_t base = w * slots;
                k_sv_generate<<<g_gen, 128, 0, stream>>>(d_scenes, d_tab[k], wfb[k], base, d_rad[k]);
                for (uint32_t bounce = 0; bounce < depth; ++bounce) {
                    const uint32_t cur = bounce & 1u;
                    k_sv_extend<<<g_ext, 128, 0, stream>>>(d_scenes, wfb[k], cur);
                    k_sv_shade<0><<<g_shade[0], 128, 0, stream>>>(d_scenes, wfb[k], cur, base, d_rad[k]);
                    k_sv_shade<1><<<g_shade[1], 128, 0, stream>>>(d_scenes, wfb[k], cur, base, d_rad[k]);
                    k_sv_shade<2><<<g_shade[2], 128, 0, stream>>>(d_scenes, wfb[k], cur, base, d_rad[k]);
                    k_sv_shade<3><<<g_shade[3], 128, 0, stream>>>(d_scenes, wfb[k], cur, base, d_rad[k]);
                    k_sv_shade<4><<<g_shade[4], 128, 0, stream>>>(d_scenes, wfb[k], cur, base, d_rad[k]);
                    k_sv_shade<5><<<g_shade[5], 128, 0, stream>>>(d_scenes, wfb[k], cur, base, d_rad[k]);
                    k_sv_shade<6><<<g_shade[6], 128, 0, stream>>>(d_scenes, wfb[k], cur, base, d_rad[k]);
                    k_sv_shade<7><<<g_shade[7], 128, 0, stream>>>(d_scenes, wfb[k], cur, base, d_rad[k]);
                    k_sv_shadow<<<g_shadow, 128, 0, stream>>>(d_scenes, wfb[k], base, d_rad[k]);
                }
            }
            k_serve_film<<<film_grid, 256, 0, stream>>>(d_tab[k], d_rad[k]);
            e = cudaStreamEndCapture(stream, &g);
            if (e == cudaSuccess) e = cudaGraphInstantiate(&graph[k], g, 0);
            if (g) cudaGraphDestroy(g);
        }
        if (e == cudaSuccess) {
            graph_depth = depth;
            graph_kernels = static_cast<unsigned>(waves * (1 + (2ull + kWfClasses) * depth) + 1);
        }
        return e;
    }

    // Marks every job of a failed batch or admission as failed (under mu).
    void fail_locked(const std::string &msg) {
        if (error.empty()) error = msg;
        for (auto &j : active) {
            j->failed = true;
            j->done = true;
        }
        active.clear();
        cv_done.notify_all();
    }

    void complete_oldest() {
        Inflight b = inflight.front();
        inflight.pop_front();
        cudaError_t e = cudaEventSynchronize(ev_end[b.slot]);
        Clock::time_point now = Clock::now();
        float ms = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev_start[b.slot], ev_end[b.slot]);
        std::lock_guard<std::mutex> lk(mu);
        if (e != cudaSuccess) {
            fail_locked(std::string("server batch: ") + cudaGetErrorString(e));
            return;
        }
        st.gpu_busy_s += ms * 1e-3;
        for (auto &j : b.finishing) {
            j->t_done = now;
            j->done = true;
            j->film = nullptr;  // freed in stream order after the result copy
            mem_used -= j->bytes;
            double lat = std::chrono::duration<double, std::milli>(now - j->t_submit).count();
            latencies_ms.push_back(lat);
            st.completed += 1;
            st.paths += static_cast<double>(j->npix) * j->desc.spp;
            t_last = now;
            active.erase(std::remove(active.begin(), active.end(), j), active.end());
        }
        cv_done.notify_all();
        cv_work.notify_all();
    }

    void run() {
        cudaSetDevice(device);
        for (;;) {
            std::vector<std::shared_ptr<Job>> work, rt_work;
            {
                std::unique_lock<std::mutex> lk(mu);
                // Admission: job slots and the HBM budget (resident scenes, the
                // two batch scratch buffers and the admitted jobs' films).
                while (!pending.empty() && active.size() < max_jobs &&
                       scratch + resident + mem_used + pending.front()->bytes <= budget) {
                    std::shared_ptr<Job> j = pending.front();
                    pending.pop_front();
                    cudaError_t e = j->rt ? cudaSuccess : cudaMallocAsync(&j->film, j->bytes, stream);
                    if (e != cudaSuccess) {
                        j->failed = j->done = true;
                        j->film = nullptr;
                        if (error.empty()) error = std::string("server admission: ") + cudaGetErrorString(e);
                        cv_done.notify_all();
                        continue;
                    }
                    mem_used += j->bytes;
                    active.push_back(j);
                    st.peak_bytes = std::max(st.peak_bytes, mem_used);
                    st.peak_jobs = std::max<uint32_t>(st.peak_jobs, static_cast<uint32_t>(active.size()));
                }
                // Path-tracing jobs with frames left, and the oldest admitted
                // real-time job of each real-time scene (its frames follow the
                // scene's earlier jobs).
                bool rt_taken[kMaxServeScenes] = {};
                for (auto &j : active) {
                    if (j->scheduled >= j->desc.spp) continue;
                    if (!j->rt) {
                        work.push_back(j);
                    } else if (!rt_taken[j->desc.scene]) {
                        rt_taken[j->desc.scene] = true;
                        rt_work.push_back(j);
                    }
                }
                if (work.empty() && rt_work.empty() && inflight.empty()) {
                    if (stop) return;
                    cv_work.wait(lk, [&] { return stop || !pending.empty(); });
                    continue;
                }
            }
            if (work.empty() && rt_work.empty()) {
                complete_oldest();
                continue;
            }
            if (inflight.size() >= 2) complete_oldest();
            uint32_t depth;
            {
                std::lock_guard<std::mutex> lk(mu);
                depth = need_depth;
            }
            if (depth > graph_depth) {
                while (!inflight.empty()) complete_oldest();
                cudaError_t e = capture(depth);
                if (e != cudaSuccess) {
                    std::lock_guard<std::mutex> lk(mu);
                    fail_locked(std::string("server graph capture: ") + cudaGetErrorString(e));
                    continue;
                }
            }
            launch_batch(work, rt_work);
        }
    }

    // One batch: one ReSTIR frame of each real-time job in `rt_work`, then a
    // fair share of the batch's paths for every path-tracing job with frames
    // left (whole frames, at least one), then the remaining capacity in
    // admission order; one item per job with contiguous frames.
    void launch_batch(const std::vector<std::shared_ptr<Job>> &work, const std::vector<std::shared_ptr<Job>> &rt_work) {
        const int slot = static_cast<int>(batch_no & 1u);
        ServeTable &t = *h_tab[slot];
        std::vector<uint32_t> frames(work.size(), 0);
        uint64_t left = batch_paths;
        uint64_t share = work.empty() ? batch_paths : std::max<uint64_t>(batch_paths / work.size(), 1);
        size_t nitems = 0;
        for (size_t i = 0; i < work.size() && nitems < kMaxServeItems; ++i) {
            const Job &j = *work[i];
            uint64_t rem = j.desc.spp - j.scheduled;
            uint64_t fr = std::min<uint64_t>(rem, std::max<uint64_t>(1, share / j.npix));
            fr = std::min<uint64_t>(fr, left / j.npix);
            if (fr == 0) continue;
            frames[i] = static_cast<uint32_t>(fr);
            left -= fr * j.npix;
            ++nitems;
        }
        for (size_t i = 0; i < work.size(); ++i) {
            const Job &j = *work[i];
            if (frames[i] == 0 && nitems >= kMaxServeItems) continue;
            uint64_t rem = j.desc.spp - j.scheduled - frames[i];
            uint64_t fr = std::min<uint64_t>(rem, left / j.npix);
            if (fr == 0) continue;
            if (frames[i] == 0) ++nitems;
            frames[i] += static_cast<uint32_t>(fr);
            left -= fr * j.npix;
        }
        Inflight b;
        b.slot = slot;
        t.next = 0;
        t.count = 0;
        uint64_t paths = 0, pix = 0;
        for (size_t i = 0; i < work.size(); ++i) {
            if (frames[i] == 0) continue;
            Job &j = *work[i];
            ServeItem &it = t.items[t.count++];
            it.cam = j.desc.cam;
            it.scene = j.desc.scene;
            it.frame_begin = j.desc.frame_begin + j.scheduled;
            it.frame_count = frames[i];
            it.film_index = j.scheduled;
            it.path_begin = paths;
            it.pix_begin = pix;
            it.film = j.film;
            it.npix = j.npix;
            it.pad = 0;
            paths += static_cast<uint64_t>(frames[i]) * j.npix;
            pix += j.npix;
            j.scheduled += frames[i];
            if (j.scheduled == j.desc.spp) b.finishing.push_back(work[i]);
        }
        t.total_paths = paths;
        t.total_pix = pix;
        cudaError_t e = cudaEventRecord(ev_start[slot], stream);
        // Real-time frames first, in stream order: a finished job's film is
        // copied out before the scene's next job restarts it.
        unsigned rt_launches = 0;
        std::string rt_err;
        int rt_rc = VS_OK;
        for (size_t i = 0; i < rt_work.size() && e == cudaSuccess && rt_rc == VS_OK; ++i) {
            Job &j = *rt_work[i];
            const RtServeHooks &h = rt_hooks[j.desc.scene];
            rt_rc = h.frame(j.desc.cam, j.desc.frame_begin + j.scheduled, j.scheduled, stream, &rt_launches, rt_err);
            if (rt_rc != VS_OK) break;
            j.scheduled += 1;
            if (j.scheduled == j.desc.spp) {
                e = cudaMemcpyAsync(j.host, h.film, j.host_bytes, cudaMemcpyDeviceToHost, stream);
                b.finishing.push_back(rt_work[i]);
            }
        }
        if (e == cudaSuccess && rt_rc == VS_OK && t.count > 0) e = cudaGraphLaunch(graph[slot], stream);
        for (size_t i = 0; i < b.finishing.size() && t.count > 0; ++i) {
            Job &j = *b.finishing[i];
            if (j.rt) continue;
            if (e == cudaSuccess) e = cudaMemcpyAsync(j.host, j.film, j.host_bytes, cudaMemcpyDeviceToHost, stream);
            if (e == cudaSuccess) e = cudaFreeAsync(j.film, stream);
        }
        if (e == cudaSuccess) e = cudaEventRecord(ev_end[slot], stream);
        std::lock_guard<std::mutex> lk(mu);
        if (rt_rc != VS_OK) {
            fail_locked("server real-time frame: " + rt_err);
            return;
        }
        if (e != cudaSuccess) {
            fail_locked(std::string("server launch: ") + cudaGetErrorString(e));
            return;
        }
        st.batches += 1;
        st.kernel_launches += rt_launches;
        if (t.count > 0) {
            st.graph_launches += 1;
            st.kernel_launches += graph_kernels;
            add_launches(graph_kernels);
        }
        ++batch_no;
        inflight.push_back(std::move(b));
    }
};

int server_create(int device, uint64_t hbm_budget, uint32_t max_jobs, uint64_t paths_per_batch, Server **out,
                  std::string &err) {
    *out = nullptr;
    if (max_jobs == 0 || paths_per_batch == 0) {
        err = "max_jobs and paths_per_batch must be positive";
        return VS_E_INVALID;
    }
    std::unique_ptr<Server> s(new Server());
    s->device = device;
    s->budget = hbm_budget;
    s->max_jobs = max_jobs;
    s->batch_paths = paths_per_batch;
    s->scratch = 2ull * paths_per_batch * sizeof(float4) + 2ull * sizeof(ServeTable) +
                 2ull * Server::wave_slots(paths_per_batch) * kWfBytesPerSlot;
    if (s->scratch >= hbm_budget) {
        err = "HBM budget below the batch scratch buffers";
        return VS_E_RANGE;
    }
    s->st.scratch_bytes = s->scratch;
    cudaError_t e = s->init();
    if (e != cudaSuccess) {
        err = std::string("server init: ") + cudaGetErrorString(e);
        return VS_E_CUDA;
    }
    *out = s.release();
    return VS_OK;
}

void server_destroy(Server *s) { delete s; }

int server_add_scene(Server *s, const DeviceScene &scene, uint64_t bytes, uint32_t *id, std::string &err) {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->nscenes >= kMaxServeScenes) {
        err = "too many resident scenes";
        return VS_E_RANGE;
    }
    if (s->scratch + s->resident + bytes > s->budget) {
        err = "resident scenes above the HBM budget";
        return VS_E_RANGE;
    }
    if (scene.ip.spectrum_dim != SN) {
        err = "served scenes must use 4 hero wavelengths";
        return VS_E_UNSUPPORTED;
    }
    // A synchronous copy, not on the server's stream: the scheduler thread may
    // be capturing that stream into a graph.
    cudaSetDevice(s->device);
    cudaError_t e = cudaMemcpy(s->d_scenes + s->nscenes, &scene, sizeof(DeviceScene), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        err = std::string("server scene upload: ") + cudaGetErrorString(e);
        return VS_E_CUDA;
    }
    s->scene_cam[s->nscenes] = scene.cam;
    s->need_depth = std::max(s->need_depth, scene.ip.max_depth);
    s->resident += bytes;
    s->st.resident_bytes = s->resident;
    *id = s->nscenes++;
    return VS_OK;
}

int server_add_rt_scene(Server *s, const Camera &cam, uint64_t bytes, RtServeHooks hooks, uint32_t *id,
                        std::string &err) {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->nscenes >= kMaxServeScenes) {
        err = "too many resident scenes";
        return VS_E_RANGE;
    }
    if (s->scratch + s->resident + bytes > s->budget) {
        err = "resident scenes above the HBM budget";
        return VS_E_RANGE;
    }
    if (!hooks.frame || !hooks.film) {
        err = "real-time scene without its frame hooks";
        return VS_E_INVALID;
    }
    // Its slot of the path-tracing scene table stays zero: path-tracing
    // batches never name it.
    s->scene_cam[s->nscenes] = cam;
    s->scene_rt[s->nscenes] = true;
    s->rt_hooks[s->nscenes] = std::move(hooks);
    s->resident += bytes;
    s->st.resident_bytes = s->resident;
    *id = s->nscenes++;
    return VS_OK;
}

int server_scene_camera(Server *s, uint32_t id, const Camera **cam, std::string &err) {
    std::lock_guard<std::mutex> lk(s->mu);
    if (id >= s->nscenes) {
        err = "unknown scene id";
        return VS_E_INVALID;
    }
    *cam = &s->scene_cam[id];
    return VS_OK;
}

int server_submit(Server *s, const ServeJob &job, uint64_t *id, std::string &err) {
    uint64_t npix = static_cast<uint64_t>(job.cam.width) * job.cam.height;
    if (npix == 0 || job.spp == 0) {
        err = "empty job";
        return VS_E_INVALID;
    }
    if (job.scene >= s->nscenes) {
        err = "unknown scene id";
        return VS_E_INVALID;
    }
    bool rt;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        rt = s->scene_rt[job.scene];
        if (rt && (job.cam.width != s->scene_cam[job.scene].width || job.cam.height != s->scene_cam[job.scene].height)) {
            err = "real-time jobs render at their scene's resolution";
            return VS_E_INVALID;
        }
    }
    if (!rt && npix > s->batch_paths) {
        err = "job resolution above the batch size";
        return VS_E_RANGE;
    }
    auto j = std::make_shared<Job>();
    j->desc = job;
    j->npix = static_cast<uint32_t>(npix);
    j->rt = rt;
    j->host_bytes = npix * sizeof(float4);
    // A real-time job renders into its scene's resident film: no device memory
    // of its own.
    j->bytes = rt ? 0 : j->host_bytes;
    if (s->scratch + s->resident + j->bytes > s->budget) {
        err = "job larger than the HBM budget";
        return VS_E_RANGE;
    }
    cudaSetDevice(s->device);
    cudaError_t e = cudaHostAlloc(&j->host, j->host_bytes, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        err = std::string("result buffer: ") + cudaGetErrorString(e);
        return VS_E_CUDA;
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (!s->error.empty()) {
            cudaFreeHost(j->host);
            err = s->error;
            return VS_E_CUDA;
        }
        j->id = s->next_id++;
        j->t_submit = Clock::now();
        if (!s->any_submit) {
            s->any_submit = true;
            s->t_first = j->t_submit;
        }
        s->st.submitted += 1;
        s->jobs[j->id] = j;
        s->pending.push_back(j);
        *id = j->id;
    }
    s->cv_work.notify_all();
    return VS_OK;
}

int server_poll(Server *s, uint64_t id, int *done, std::string &err) {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) {
        err = "unknown job id";
        return VS_E_INVALID;
    }
    *done = it->second->done ? 1 : 0;
    if (it->second->failed) {
        err = s->error;
        return VS_E_CUDA;
    }
    return VS_OK;
}

int server_result(Server *s, uint64_t id, float *dst, size_t bytes, double timeout_s, std::string &err) {
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) {
        err = "unknown job id";
        return VS_E_INVALID;
    }
    std::shared_ptr<Job> j = it->second;
    if (bytes != j->host_bytes) {
        err = "result size mismatch";
        return VS_E_INVALID;
    }
    auto ready = [&] { return j->done; };
    if (timeout_s < 0) {
        s->cv_done.wait(lk, ready);
    } else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
        err = "timed out";
        return VS_E_STATE;
    }
    if (j->failed) {
        err = s->error;
        s->jobs.erase(id);
        if (j->host) cudaFreeHost(j->host);
        return VS_E_CUDA;
    }
    std::memcpy(dst, j->host, bytes);
    cudaFreeHost(j->host);
    j->host = nullptr;
    s->jobs.erase(id);
    return VS_OK;
}

void server_stats(Server *s, ServeStats *out) {
    std::lock_guard<std::mutex> lk(s->mu);
    ServeStats r = s->st;
    std::vector<double> v = s->latencies_ms;
    std::sort(v.begin(), v.end());
    auto pct = [&](double q) {
        if (v.empty()) return 0.0;
        size_t i = static_cast<size_t>(q * (v.size() - 1) + 0.5);
        return v[std::min(i, v.size() - 1)];
    };
    r.p50_ms = pct(0.50);
    r.p95_ms = pct(0.95);
    r.p99_ms = pct(0.99);
    r.max_ms = v.empty() ? 0.0 : v.back();
    double sum = 0.0;
    for (double x : v) sum += x;
    r.mean_ms = v.empty() ? 0.0 : sum / v.size();
    r.wall_s = (s->any_submit && r.completed) ? std::chrono::duration<double>(s->t_last - s->t_first).count() : 0.0;
    *out = r;
}

cudaError_t upload_spectral_consts_serve(const float *x, const float *y, const float *z, const float *d65,
                                         float y_integral) {
    return upload_spectral_consts_tu(x, y, z, d65, y_integral);
}

}  // namespace vs

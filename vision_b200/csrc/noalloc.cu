// vs_render_noalloc: the render entry point for callers that cannot allocate
// device memory.
//
// vs_render keeps its per-path radiance (the scratch between the megakernel
// and the film pass) in a buffer it grows with cudaMalloc, and keeps the film
// in buffers it owns.  Some callers cannot allocate at render time: a frame
// loop that runs inside a fixed, pre-reserved memory budget, a host thread
// that must not take the driver's allocation locks while other work is in
// flight, or an embedding application whose allocator owns all device memory.
// For them this entry point takes the film as a caller-owned device buffer and
// keeps the radiance scratch in a fixed array compiled into the library, so it
// calls no cudaMalloc, cudaFree or allocating library routine.
//
// The scratch array is a file-scope __device__ variable: every GPU that loads
// the library holds its 16 MiB until the process exits.  In host code the
// array's name is only a host-side stand-in, not a device address, so the
// device address is looked up with cudaGetSymbolAddress once per device, the
// first time this entry point runs with that device current; that first call
// should therefore happen before any stream capture.  The looked-up address is
// kept for the life of the process: after cudaDeviceReset (or anything else
// that destroys and re-creates the device's primary context) the library's
// module is loaded again and the kept address is stale, so this entry point
// must not be used after such a reset.  Each chunk's megakernel writes every
// scratch entry that the following film pass reads, so the array needs no
// clearing between calls; calls that overlap on the GPU share it and race.
//
// The scene's lock is held from the argument checks to the last launch, as
// vs_render holds it: a concurrent vs_scene_build_accel (which frees and
// re-uploads the scene's device buffers) waits until the launches are queued.
#include "../../include/vision_b200.h"
#include "vs_launch.h"

#include <cstdint>
#include <mutex>

namespace vs {

// 2^20 float4 radiance entries = 16 MiB: one path per entry, reused chunk by
// chunk.  A single frame must fit, so resolutions above 2^20 pixels are
// rejected.
constexpr uint64_t kNoAllocScratchPaths = 1ull << 20;
static __device__ __align__(256) float4 g_noalloc_scratch[kNoAllocScratchPaths];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_symbol_mutex;
float4 *g_symbol_ptr[kMaxDevices] = {nullptr};

// Device address of g_noalloc_scratch on `device` (which must be current).
cudaError_t scratch_address(int device, float4 **out) {
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_symbol_mutex);
    if (!g_symbol_ptr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_symbol_ptr[device] = static_cast<float4 *>(p);
    }
    *out = g_symbol_ptr[device];
    return cudaSuccess;
}
}  // namespace

// Implemented in capi.cu.  noalloc_scene_mutex is the scene's lock;
// noalloc_prepare (called with that lock held) checks that the scene is on the
// device, makes its device current and returns its device view and the render
// stream.  Neither allocates.
std::mutex &noalloc_scene_mutex(vs_scene *scene);
int noalloc_prepare(vs_scene *scene, void *stream, DeviceScene *view, cudaStream_t *st, int *device);
int noalloc_fail(vs_scene *scene, int code, const char *msg);

}  // namespace vs

extern "C" int vs_render_noalloc(vs_scene *scene, uint32_t frame_begin, uint32_t frame_count, float *film,
                                 void *stream) {
    using namespace vs;
    if (!scene || !film) return VS_E_INVALID;
    if (reinterpret_cast<uintptr_t>(film) % 16 != 0)
        return noalloc_fail(scene, VS_E_INVALID,
                            "vs_render_noalloc: film must be 16-byte aligned (it is read and written as float4)");
    std::lock_guard<std::mutex> lock(noalloc_scene_mutex(scene));
    DeviceScene view;
    cudaStream_t st;
    int device = -1;
    int rc = noalloc_prepare(scene, stream, &view, &st, &device);
    if (rc != VS_OK) return rc;
    uint64_t npix = static_cast<uint64_t>(view.cam.width) * view.cam.height;
    if (npix > kNoAllocScratchPaths)
        return noalloc_fail(scene, VS_E_RANGE,
                            "vs_render_noalloc: resolution above 1048576 pixels (the fixed 16 MiB scratch holds one "
                            "frame of at most 2^20 paths)");
    float4 *scratch = nullptr;
    cudaError_t e = scratch_address(device, &scratch);
    if (e != cudaSuccess) return noalloc_fail(scene, VS_E_CUDA, cudaGetErrorString(e));
    const uint64_t frames_per_chunk = kNoAllocScratchPaths / npix;
    float4 *film4 = reinterpret_cast<float4 *>(film);
    // 64-bit counter: frames_per_chunk reaches 2^20, so a 32-bit f + chunk
    // could wrap for frame counts near 2^32 and never end the loop.
    for (uint64_t f = 0; f < frame_count; f += frames_per_chunk) {
        uint32_t fc = static_cast<uint32_t>(frame_count - f < frames_per_chunk ? frame_count - f : frames_per_chunk);
        uint32_t fb = frame_begin + static_cast<uint32_t>(f);
        e = launch_render(view, fb, fc, scratch, st);
        if (e == cudaSuccess) e = launch_film(scratch, static_cast<uint32_t>(npix), fb, fc, film4, nullptr, st);
        if (e != cudaSuccess) return noalloc_fail(scene, VS_E_CUDA, cudaGetErrorString(e));
    }
    return VS_OK;
}

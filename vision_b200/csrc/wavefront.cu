// Wavefront path tracing: the megakernel's bounce loop as a sequence of
// kernels over a wave of path slots.
//
//   k_wf_generate  camera paths of the wave (PathTracingIntegrator kernel
//                  body, pt.cpp:53-72): wavelengths, camera ray, queue 0
//   per bounce:
//   k_wf_extend    closest hit of every queued ray (traversal only)
//   k_wf_shade     path_shade: emission, light sample (shadow query), BSDF
//                  sample, Russian roulette, next ray; survivors to the other
//                  queue, shadow queries to the shadow queue
//   k_wf_shadow    any hit of every shadow query, contribution when unoccluded
//
// Each slot's sampler draws in the same order as the megakernel (light,
// BSDF, roulette per bounce) and the radiance is summed in the same order
// (emission of a bounce, then its next-event estimate), so every path gives
// the megakernel's radiance.  Queue counters live on the device; kernels loop
// over `count` with a grid stride, so no host synchronisation is needed.
#include "vs_wavefront.cuh"
#include "vs_launch.h"

#include <algorithm>
#include <atomic>

namespace vs {

namespace {

// The one scene of a vs_render call (the kernel's grid-constant parameter).
struct OneScene {
    const DeviceScene *s;
    __device__ __forceinline__ const DeviceScene &operator()(uint32_t) const { return *s; }
};

}  // namespace

// Slot i of the wave holds path base + i.
template <int N>
__global__ void __launch_bounds__(128) k_wf_generate(const __grid_constant__ DeviceScene s,
                                                     const __grid_constant__ WfBuffers b, uint32_t frame_begin,
                                                     uint64_t base, uint32_t n, float4 *radiance) {
    wf::generate<N>(s, s.cam, b, frame_begin, base, n, radiance);
}

__global__ void __launch_bounds__(128) k_wf_extend(const __grid_constant__ DeviceScene s,
                                                   const __grid_constant__ WfBuffers b, uint32_t cur) {
    wf::extend(OneScene{&s}, b, cur);
}

// Shading of class C (0: misses, 1 + MaterialType: hits of that material).
template <int N, uint32_t C>
__global__ void __launch_bounds__(128) k_wf_shade(const __grid_constant__ DeviceScene s,
                                                  const __grid_constant__ WfBuffers b, uint32_t cur, uint64_t base,
                                                  float4 *radiance) {
    wf::shade<N, C>(OneScene{&s}, b, cur, base, radiance);
}

__global__ void __launch_bounds__(128) k_wf_shadow(const __grid_constant__ DeviceScene s,
                                                   const __grid_constant__ WfBuffers b, uint64_t base,
                                                   float4 *radiance) {
    wf::shadow(OneScene{&s}, b, base, radiance);
}

namespace {

// Resident blocks of 128 threads per SM for each kernel, per device.
template <typename K>
cudaError_t resident_grid(K kernel, int dev, std::atomic<int> &cache, unsigned *grid) {
    int g = cache.load();
    if (g == 0) {
        int sms = 0, per_sm = 0;
        cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 128, 0);
        if (e != cudaSuccess) return e;
        g = sms * std::max(per_sm, 1);
        cache.store(g);
    }
    *grid = static_cast<unsigned>(g);
    return cudaSuccess;
}

struct ShadeGrids {
    unsigned g[kWfClasses];
};

template <int N, uint32_t C>
cudaError_t shade_grid(int dev, ShadeGrids &sg) {
    static std::atomic<int> cache[64];
    return resident_grid(k_wf_shade<N, C>, dev, cache[dev], &sg.g[C]);
}

template <int N, uint32_t C>
void launch_shade(const ShadeGrids &sg, uint32_t mask, const DeviceScene &s, const WfBuffers &b, uint32_t cur,
                  uint64_t base, float4 *radiance, cudaStream_t st, unsigned &n_launch) {
    if (!((mask >> C) & 1u)) return;
    k_wf_shade<N, C><<<sg.g[C], 128, 0, st>>>(s, b, cur, base, radiance);
    ++n_launch;
}

template <int N>
cudaError_t wave_loop(const DeviceScene &s, uint32_t frame_begin, uint64_t paths, float4 *radiance,
                      const WfBuffers &b, uint32_t class_mask, cudaStream_t st, unsigned *launches) {
    static std::atomic<int> g_gen[64], g_ext[64], g_shadow[64];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    unsigned grid_gen, grid_ext, grid_shadow;
    ShadeGrids sg{};
    if ((e = resident_grid(k_wf_generate<N>, dev, g_gen[dev], &grid_gen)) != cudaSuccess) return e;
    if ((e = resident_grid(k_wf_extend, dev, g_ext[dev], &grid_ext)) != cudaSuccess) return e;
    if ((e = resident_grid(k_wf_shadow, dev, g_shadow[dev], &grid_shadow)) != cudaSuccess) return e;
    if ((e = shade_grid<N, 0>(dev, sg)) != cudaSuccess) return e;
    if ((e = shade_grid<N, 1>(dev, sg)) != cudaSuccess) return e;
    if ((e = shade_grid<N, 2>(dev, sg)) != cudaSuccess) return e;
    if ((e = shade_grid<N, 3>(dev, sg)) != cudaSuccess) return e;
    if ((e = shade_grid<N, 4>(dev, sg)) != cudaSuccess) return e;
    if ((e = shade_grid<N, 5>(dev, sg)) != cudaSuccess) return e;
    if ((e = shade_grid<N, 6>(dev, sg)) != cudaSuccess) return e;
    const uint32_t mask = class_mask | 1u;
    unsigned n_launch = 0;
    for (uint64_t base = 0; base < paths; base += b.capacity) {
        const uint32_t n = static_cast<uint32_t>(std::min<uint64_t>(b.capacity, paths - base));
        const unsigned g = std::min<unsigned>(grid_gen, (n + 127u) / 128u);
        k_wf_generate<N><<<g, 128, 0, st>>>(s, b, frame_begin, base, n, radiance);
        ++n_launch;
        for (uint32_t bounce = 0; bounce < s.ip.max_depth; ++bounce) {
            const uint32_t cur = bounce & 1u;
            k_wf_extend<<<grid_ext, 128, 0, st>>>(s, b, cur);
            launch_shade<N, 0>(sg, mask, s, b, cur, base, radiance, st, n_launch);
            launch_shade<N, 1>(sg, mask, s, b, cur, base, radiance, st, n_launch);
            launch_shade<N, 2>(sg, mask, s, b, cur, base, radiance, st, n_launch);
            launch_shade<N, 3>(sg, mask, s, b, cur, base, radiance, st, n_launch);
            launch_shade<N, 4>(sg, mask, s, b, cur, base, radiance, st, n_launch);
            launch_shade<N, 5>(sg, mask, s, b, cur, base, radiance, st, n_launch);
            launch_shade<N, 6>(sg, mask, s, b, cur, base, radiance, st, n_launch);
            k_wf_shadow<<<grid_shadow, 128, 0, st>>>(s, b, base, radiance);
            n_launch += 2;
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (launches) *launches = n_launch;
    return cudaSuccess;
}

}  // namespace

cudaError_t launch_render_wavefront(const DeviceScene &s, uint32_t frame_begin, uint32_t frame_count,
                                    float4 *radiance, const WfBuffers &b, uint32_t class_mask, cudaStream_t st,
                                    unsigned *launches) {
    if (launches) *launches = 0;
    const uint64_t paths = static_cast<uint64_t>(s.cam.width) * s.cam.height * frame_count;
    if (paths == 0) return cudaSuccess;
    if (b.capacity == 0 || b.capacity > 0x7fffffffu) return cudaErrorInvalidValue;
    switch (s.ip.spectrum_dim) {
        case 1: return wave_loop<1>(s, frame_begin, paths, radiance, b, class_mask, st, launches);
        case 2: return wave_loop<2>(s, frame_begin, paths, radiance, b, class_mask, st, launches);
        case 3: return wave_loop<3>(s, frame_begin, paths, radiance, b, class_mask, st, launches);
        case 4: return wave_loop<4>(s, frame_begin, paths, radiance, b, class_mask, st, launches);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t upload_spectral_consts_wf(const float *x, const float *y, const float *z, const float *d65,
                                      float y_integral) {
    return upload_spectral_consts_tu(x, y, z, d65, y_integral);
}

}  // namespace vs

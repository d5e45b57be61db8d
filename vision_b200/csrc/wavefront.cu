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

// L: kLevelsFlat or kLevelsTwo, picked on the host from the scene.
template <int L>
__global__ void __launch_bounds__(128) k_wf_extend(const __grid_constant__ DeviceScene s,
                                                   const __grid_constant__ WfBuffers b, uint32_t cur) {
    wf::extend<L>(OneScene{&s}, b, cur);
}

// Shading of class C (0: misses, 1 + MaterialType: hits of that material).
template <int N, uint32_t C>
__global__ void __launch_bounds__(128) k_wf_shade(const __grid_constant__ DeviceScene s,
                                                  const __grid_constant__ WfBuffers b, uint32_t cur, uint64_t base,
                                                  float4 *radiance) {
    wf::shade<N, C>(OneScene{&s}, b, cur, base, radiance);
}

template <int L>
__global__ void __launch_bounds__(128) k_wf_shadow(const __grid_constant__ DeviceScene s,
                                                   const __grid_constant__ WfBuffers b, uint64_t base,
                                                   float4 *radiance) {
    wf::shadow<L>(OneScene{&s}, b, base, radiance);
}

// ---------------------------------------------------------------------------
// Ray binning: a counting sort of a queue by ray key (direction octant, then
// the Morton cell of the origin), so that the warps of the traversal pass
// take rays that start close together and visit the children in the same
// order.  The order of entries inside a bin is arbitrary; every path's result
// is independent of the order in which rays are traced.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t spread3(uint32_t v) {
    v &= 7u;
    return (v & 1u) | ((v & 2u) << 2) | ((v & 4u) << 4);
}

// Key of a ray: the scene box is the BVH root's quantisation grid (origin p,
// 255 steps of 2^e per axis).
__device__ __forceinline__ uint32_t ray_key(const uint4 &root, const float4 &o, const float4 &d) {
    const float px = __uint_as_float(root.x), py = __uint_as_float(root.y), pz = __uint_as_float(root.z);
    const float sx = __uint_as_float((root.w & 0xffu) << 23) * (8.0f / 255.0f);
    const float sy = __uint_as_float(((root.w >> 8) & 0xffu) << 23) * (8.0f / 255.0f);
    const float sz = __uint_as_float(((root.w >> 16) & 0xffu) << 23) * (8.0f / 255.0f);
    const uint32_t cx = static_cast<uint32_t>(fminf(fmaxf((o.x - px) / sx, 0.0f), 7.0f));
    const uint32_t cy = static_cast<uint32_t>(fminf(fmaxf((o.y - py) / sy, 0.0f), 7.0f));
    const uint32_t cz = static_cast<uint32_t>(fminf(fmaxf((o.z - pz) / sz, 0.0f), 7.0f));
    const uint32_t oct = (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
    return (oct << 9) | spread3(cx) | (spread3(cy) << 1) | (spread3(cz) << 2);
}

// Pass 1: the key of every entry of a queue of n = *len entries (src: the
// queue's slots, or null for entries 0..n-1 of the shadow queue) and the
// sizes of the bins.
__global__ void __launch_bounds__(256) k_bin_count(const __grid_constant__ DeviceScene s, const uint32_t *len,
                                                   const uint32_t *src, const float4 *o, const float4 *d,
                                                   uint32_t *keys, uint32_t *bins) {
    const uint32_t n = *len;
    const uint4 root = __ldg(s.nodes);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t e = src ? src[i] : i;
        const uint32_t key = ray_key(root, o[e], d[e]);
        keys[i] = key;
        const unsigned active = __activemask();
        const unsigned group = __match_any_sync(active, key);
        if (wf::lane_id() == __ffs(group) - 1) atomicAdd(bins + key, static_cast<uint32_t>(__popc(group)));
    }
}

// Pass 2 (one block of 1024 threads): bin write positions (exclusive prefix
// sums) to bins[kWfBins ...], sizes cleared for the next use.
__global__ void __launch_bounds__(1024) k_bin_scan(uint32_t *bins) {
    constexpr uint32_t per = kWfBins / 1024u;
    __shared__ uint32_t part[1024];
    uint32_t local[per];
    uint32_t sum = 0;
#pragma unroll
    for (uint32_t k = 0; k < per; ++k) {
        local[k] = bins[threadIdx.x * per + k];
        sum += local[k];
    }
    part[threadIdx.x] = sum;
    __syncthreads();
    for (uint32_t off = 1; off < 1024u; off <<= 1) {
        const uint32_t v = threadIdx.x >= off ? part[threadIdx.x - off] : 0u;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t pos = part[threadIdx.x] - sum;
#pragma unroll
    for (uint32_t k = 0; k < per; ++k) {
        bins[kWfBins + threadIdx.x * per + k] = pos;
        pos += local[k];
        bins[threadIdx.x * per + k] = 0u;
    }
}

// Pass 3: every entry to its bin (dst: the binned queue's slots, or the
// shadow queue's entry indices).
__global__ void __launch_bounds__(256) k_bin_scatter(const uint32_t *len, const uint32_t *src, const uint32_t *keys,
                                                     uint32_t *bins, uint32_t *dst) {
    const uint32_t n = *len;
    uint32_t *pos = bins + kWfBins;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t key = keys[i];
        const unsigned active = __activemask();
        const unsigned group = __match_any_sync(active, key);
        const int lane = wf::lane_id();
        const int leader = __ffs(group) - 1;
        uint32_t base = 0;
        if (lane == leader) base = atomicAdd(pos + key, static_cast<uint32_t>(__popc(group)));
        base = __shfl_sync(active, base, leader);
        // The bin sizes of pass 1 sum to n, so every position is below n.
        const uint32_t p = base + static_cast<uint32_t>(__popc(group & ((1u << lane) - 1u)));
        if (p < n) dst[p] = src ? src[i] : i;
    }
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
    static std::atomic<int> g_gen[64], g_ext[64], g_shadow[64], g_ext2[64], g_shadow2[64];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    unsigned grid_gen, grid_ext, grid_shadow;
    ShadeGrids sg{};
    if ((e = resident_grid(k_wf_generate<N>, dev, g_gen[dev], &grid_gen)) != cudaSuccess) return e;
    const bool two = s.two_level != 0u;
    if ((e = two ? resident_grid(k_wf_extend<kLevelsTwo>, dev, g_ext2[dev], &grid_ext)
                 : resident_grid(k_wf_extend<kLevelsFlat>, dev, g_ext[dev], &grid_ext)) != cudaSuccess)
        return e;
    if ((e = two ? resident_grid(k_wf_shadow<kLevelsTwo>, dev, g_shadow2[dev], &grid_shadow)
                 : resident_grid(k_wf_shadow<kLevelsFlat>, dev, g_shadow[dev], &grid_shadow)) != cudaSuccess)
        return e;
    if ((e = shade_grid<N, 0>(dev, sg)) != cudaSuccess) return e;
    if ((e = shade_grid<N, 1>(dev, sg)) != cudaSuccess) return e;
    if ((e = shade_grid<N, 2>(dev, sg)) != cudaSuccess) return e;
    if ((e = shade_grid<N, 3>(dev, sg)) != cudaSuccess) return e;
    if ((e = shade_grid<N, 4>(dev, sg)) != cudaSuccess) return e;
    if ((e = shade_grid<N, 5>(dev, sg)) != cudaSuccess) return e;
    if ((e = shade_grid<N, 6>(dev, sg)) != cudaSuccess) return e;
    if ((class_mask >> 7) & 1u)
        if ((e = shade_grid<N, 7>(dev, sg)) != cudaSuccess) return e;
    const uint32_t mask = class_mask | 1u;
    unsigned n_launch = 0;
    const bool binning = b.bin_key && b.bins && b.binned && b.sh_perm;
    int sms = 0;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    const unsigned grid_bin = static_cast<unsigned>(sms) * 8u;
    // The traversal passes read the binned queue (path slots) or the shadow
    // permutation instead of the queues in push order.
    WfBuffers bs = b;
    bs.sh_perm = binning ? b.sh_perm : nullptr;
    for (uint64_t base = 0; base < paths; base += b.capacity) {
        const uint32_t n = static_cast<uint32_t>(std::min<uint64_t>(b.capacity, paths - base));
        const unsigned g = std::min<unsigned>(grid_gen, (n + 127u) / 128u);
        k_wf_generate<N><<<g, 128, 0, st>>>(s, b, frame_begin, base, n, radiance);
        ++n_launch;
        for (uint32_t bounce = 0; bounce < s.ip.max_depth; ++bounce) {
            const uint32_t cur = bounce & 1u;
            // Camera rays (bounce 0) arrive in pixel order, already coherent.
            const bool bin_paths = binning && bounce > 0;
            WfBuffers be = b;
            be.sh_perm = nullptr;
            if (bin_paths) {
                k_bin_count<<<grid_bin, 256, 0, st>>>(s, b.count + cur, b.queue[cur], b.o, b.d, b.bin_key, b.bins);
                k_bin_scan<<<1, 1024, 0, st>>>(b.bins);
                k_bin_scatter<<<grid_bin, 256, 0, st>>>(b.count + cur, b.queue[cur], b.bin_key, b.bins, b.binned);
                be.queue[cur] = b.binned;
                n_launch += 3;
            }
            if (two) k_wf_extend<kLevelsTwo><<<grid_ext, 128, 0, st>>>(s, be, cur);
            else k_wf_extend<kLevelsFlat><<<grid_ext, 128, 0, st>>>(s, be, cur);
            launch_shade<N, 0>(sg, mask, s, b, cur, base, radiance, st, n_launch);
            launch_shade<N, 1>(sg, mask, s, b, cur, base, radiance, st, n_launch);
            launch_shade<N, 2>(sg, mask, s, b, cur, base, radiance, st, n_launch);
            launch_shade<N, 3>(sg, mask, s, b, cur, base, radiance, st, n_launch);
            launch_shade<N, 4>(sg, mask, s, b, cur, base, radiance, st, n_launch);
            launch_shade<N, 5>(sg, mask, s, b, cur, base, radiance, st, n_launch);
            launch_shade<N, 6>(sg, mask, s, b, cur, base, radiance, st, n_launch);
            launch_shade<N, 7>(sg, mask, s, b, cur, base, radiance, st, n_launch);
            if (binning) {
                k_bin_count<<<grid_bin, 256, 0, st>>>(s, b.count + 2, nullptr, b.sh_o, b.sh_d, b.bin_key, b.bins);
                k_bin_scan<<<1, 1024, 0, st>>>(b.bins);
                k_bin_scatter<<<grid_bin, 256, 0, st>>>(b.count + 2, nullptr, b.bin_key, b.bins, b.sh_perm);
                n_launch += 3;
            }
            if (two) k_wf_shadow<kLevelsTwo><<<grid_shadow, 128, 0, st>>>(s, bs, base, radiance);
            else k_wf_shadow<kLevelsFlat><<<grid_shadow, 128, 0, st>>>(s, bs, base, radiance);
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

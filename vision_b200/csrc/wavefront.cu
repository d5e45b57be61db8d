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
#include "vs_wavefront.h"
#include "vs_integrator.cuh"
#include "vs_launch.h"

#include <algorithm>
#include <atomic>

namespace vs {

namespace {

__device__ __forceinline__ float comp(const float4 &v, int i) {
    return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w;
}

template <int N>
__device__ __forceinline__ float4 pack4(const float *a) {
    return make_float4(a[0], N > 1 ? a[1] : 0.0f, N > 2 ? a[2] : 0.0f, N > 3 ? a[3] : 0.0f);
}

template <int N>
__device__ __forceinline__ void wf_store(const WfBuffers &b, uint32_t slot, const PathState<N> &ps) {
    b.o[slot] = make_float4(ps.ro.x, ps.ro.y, ps.ro.z, ps.scatter_pdf);
    b.d[slot] = make_float4(ps.rd.x, ps.rd.y, ps.rd.z, ps.eta_scale);
    b.tp[slot] = pack4<N>(ps.throughput.v);
    b.lam[slot] = pack4<N>(ps.wl.lambda);
    b.pdf[slot] = pack4<N>(ps.wl.pdf);
    b.L[slot] = make_float4(ps.L.x, ps.L.y, ps.L.z, 0.0f);
    b.st[slot] = make_uint4(static_cast<uint32_t>(ps.smp.state), static_cast<uint32_t>(ps.smp.state >> 32),
                            ps.bounce, 0u);
}

template <int N>
__device__ __forceinline__ void wf_load(const DeviceScene &s, const WfBuffers &b, uint32_t slot, PathState<N> &ps) {
    const float4 o = b.o[slot], d = b.d[slot], tp = b.tp[slot], lam = b.lam[slot], pdf = b.pdf[slot],
                 L = b.L[slot];
    const uint4 st = b.st[slot];
    ps.ro = make3(o.x, o.y, o.z);
    ps.scatter_pdf = o.w;
    ps.rd = make3(d.x, d.y, d.z);
    ps.eta_scale = d.w;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        ps.throughput.v[i] = comp(tp, i);
        ps.wl.lambda[i] = comp(lam, i);
        ps.wl.pdf[i] = comp(pdf, i);
    }
    ps.L = make3(L.x, L.y, L.z);
    ps.smp.state = static_cast<uint64_t>(st.x) | (static_cast<uint64_t>(st.y) << 32);
    ps.smp.kind = s.ip.sampler;
    ps.smp.seed = s.ip.seed;
    ps.bounce = st.z;
}

// Appends one entry per calling lane to a device queue: one atomicAdd per
// converged group of lanes, positions in lane order.
__device__ __forceinline__ uint32_t queue_push(uint32_t *counter) {
    const unsigned mask = __activemask();
    const int lane = static_cast<int>(threadIdx.x & 31u);
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, static_cast<uint32_t>(__popc(mask)));
    base = __shfl_sync(mask, base, leader);
    return base + static_cast<uint32_t>(__popc(mask & ((1u << lane) - 1u)));
}

}  // namespace

// Slot i of the wave holds path base + i.
template <int N>
__global__ void __launch_bounds__(128) k_wf_generate(const __grid_constant__ DeviceScene s, const __grid_constant__ WfBuffers b, uint32_t frame_begin, uint64_t base,
                                                     uint32_t n, float4 *radiance) {
    const uint32_t npix = s.cam.width * s.cam.height;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        b.count[0] = n;
        b.count[1] = 0u;
        b.count[2] = 0u;
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint64_t p = base + i;
        const uint32_t frame = frame_begin + static_cast<uint32_t>(p / npix);
        const uint32_t pix = static_cast<uint32_t>(p % npix);
        PathState<N> ps;
        path_start<N>(s, s.cam, pix % s.cam.width, pix / s.cam.width, frame, ps);
        if (s.ip.max_depth == 0u) {
            radiance[p] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
            continue;
        }
        wf_store<N>(b, i, ps);
        b.queue[0][i] = i;
    }
}

// Closest hits of queue `cur`.  Also clears the other queue and the shadow
// queue for the shading pass that follows (their previous users have
// finished: kernels of one stream run in order).
__global__ void __launch_bounds__(128) k_wf_extend(const __grid_constant__ DeviceScene s, const __grid_constant__ WfBuffers b, uint32_t cur) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        b.count[cur ^ 1u] = 0u;
        b.count[2] = 0u;
    }
    const uint32_t n = b.count[cur];
    const uint32_t *q = b.queue[cur];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t slot = q[i];
        const float4 o = b.o[slot], d = b.d[slot];
        RayPre rp = precompute_ray(make3(o.x, o.y, o.z), make3(d.x, d.y, d.z));
        Hit h;
        float t;
        if (!trace_closest(s, rp, 3.402823466e+38f, h, t)) h = Hit{kInvalid, kInvalid, 0.0f, 0.0f};
        b.hit[slot] = h;
    }
}

// One bounce of every queued path after its closest hit.
template <int N>
__global__ void __launch_bounds__(128) k_wf_shade(const __grid_constant__ DeviceScene s, const __grid_constant__ WfBuffers b, uint32_t cur, uint64_t base,
                                                  float4 *radiance) {
    const uint32_t n = b.count[cur];
    const uint32_t *q = b.queue[cur];
    const uint32_t max_depth = s.ip.max_depth;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t slot = q[i];
        PathState<N> ps;
        wf_load<N>(s, b, slot, ps);
        const Hit h = b.hit[slot];
        ShadowQuery sq;
        bool more = path_shade<N, false>(s, ps, h.inst_id != kInvalid, h, nullptr, sq);
        if (more) more = ++ps.bounce < max_depth;
        if (more) {
            wf_store<N>(b, slot, ps);
            b.queue[cur ^ 1u][queue_push(&b.count[cur ^ 1u])] = slot;
        } else {
            b.L[slot] = make_float4(ps.L.x, ps.L.y, ps.L.z, 0.0f);
        }
        if (sq.valid) {
            const uint32_t k = queue_push(&b.count[2]);
            b.sh_o[k] = make_float4(sq.o.x, sq.o.y, sq.o.z, sq.tmax);
            b.sh_d[k] = make_float4(sq.d.x, sq.d.y, sq.d.z, __uint_as_float(slot | (more ? 0u : 0x80000000u)));
            b.sh_c[k] = make_float4(sq.c.x, sq.c.y, sq.c.z, 0.0f);
        } else if (!more) {
            radiance[base + slot] = make_float4(ps.L.x, ps.L.y, ps.L.z, 1.0f);
        }
    }
}

// Shadow queries of the bounce: add the contribution when unoccluded; write
// the radiance of paths that ended at this bounce.
__global__ void __launch_bounds__(128) k_wf_shadow(const __grid_constant__ DeviceScene s, const __grid_constant__ WfBuffers b, uint64_t base, float4 *radiance) {
    const uint32_t n = b.count[2];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 o = b.sh_o[i], d = b.sh_d[i];
        const uint32_t tag = __float_as_uint(d.w);
        const uint32_t slot = tag & 0x7fffffffu;
        const bool occluded = trace_any(s, precompute_ray(make3(o.x, o.y, o.z), make3(d.x, d.y, d.z)), o.w);
        float4 L = b.L[slot];
        if (!occluded) {
            const float4 c = b.sh_c[i];
            f3 l = make3(L.x, L.y, L.z);
            l += make3(c.x, c.y, c.z);
            L = make_float4(l.x, l.y, l.z, 0.0f);
            b.L[slot] = L;
        }
        if (tag & 0x80000000u) radiance[base + slot] = make_float4(L.x, L.y, L.z, 1.0f);
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

template <int N>
cudaError_t wave_loop(const DeviceScene &s, uint32_t frame_begin, uint64_t paths, float4 *radiance,
                      const WfBuffers &b, cudaStream_t st, unsigned *launches) {
    static std::atomic<int> g_gen[64], g_ext[64], g_shade[64], g_shadow[64];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    unsigned grid_gen, grid_ext, grid_shade, grid_shadow;
    if ((e = resident_grid(k_wf_generate<N>, dev, g_gen[dev], &grid_gen)) != cudaSuccess) return e;
    if ((e = resident_grid(k_wf_extend, dev, g_ext[dev], &grid_ext)) != cudaSuccess) return e;
    if ((e = resident_grid(k_wf_shade<N>, dev, g_shade[dev], &grid_shade)) != cudaSuccess) return e;
    if ((e = resident_grid(k_wf_shadow, dev, g_shadow[dev], &grid_shadow)) != cudaSuccess) return e;
    unsigned n_launch = 0;
    for (uint64_t base = 0; base < paths; base += b.capacity) {
        const uint32_t n = static_cast<uint32_t>(std::min<uint64_t>(b.capacity, paths - base));
        const unsigned g = std::min<unsigned>(grid_gen, (n + 127u) / 128u);
        k_wf_generate<N><<<g, 128, 0, st>>>(s, b, frame_begin, base, n, radiance);
        ++n_launch;
        for (uint32_t bounce = 0; bounce < s.ip.max_depth; ++bounce) {
            const uint32_t cur = bounce & 1u;
            k_wf_extend<<<grid_ext, 128, 0, st>>>(s, b, cur);
            k_wf_shade<N><<<grid_shade, 128, 0, st>>>(s, b, cur, base, radiance);
            k_wf_shadow<<<grid_shadow, 128, 0, st>>>(s, b, base, radiance);
            n_launch += 3;
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (launches) *launches = n_launch;
    return cudaSuccess;
}

}  // namespace

cudaError_t launch_render_wavefront(const DeviceScene &s, uint32_t frame_begin, uint32_t frame_count,
                                    float4 *radiance, const WfBuffers &b, cudaStream_t st, unsigned *launches) {
    if (launches) *launches = 0;
    const uint64_t paths = static_cast<uint64_t>(s.cam.width) * s.cam.height * frame_count;
    if (paths == 0) return cudaSuccess;
    if (b.capacity == 0 || b.capacity > 0x7fffffffu) return cudaErrorInvalidValue;
    switch (s.ip.spectrum_dim) {
        case 1: return wave_loop<1>(s, frame_begin, paths, radiance, b, st, launches);
        case 2: return wave_loop<2>(s, frame_begin, paths, radiance, b, st, launches);
        case 3: return wave_loop<3>(s, frame_begin, paths, radiance, b, st, launches);
        case 4: return wave_loop<4>(s, frame_begin, paths, radiance, b, st, launches);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t upload_spectral_consts_wf(const float *x, const float *y, const float *z, const float *d65,
                                      float y_integral) {
    return upload_spectral_consts_tu(x, y, z, d65, y_integral);
}

}  // namespace vs

// sm_100a kernels of the path-tracing hot path:
//   k_trace_closest  - seeded closest-hit batches (parity hook)
//   k_render         - megakernel: one camera path per thread, radiance to a
//                      per-sample buffer
//   k_render_regen   - the same paths in a persistent grid that refills
//                      finished lanes (path regeneration)
//   k_film_*         - film accumulation in the reference's frame order
//                      (FP32 running mean) or as FP64 sums
#include "vs_integrator.cuh"
#include "vs_launch.h"

#include <algorithm>
#include <atomic>

namespace vs {

static std::atomic<unsigned long long> g_launches{0};
unsigned long long launch_count() { return g_launches.load(); }
void add_launches(unsigned n) { g_launches += n; }

__global__ void __launch_bounds__(128) k_trace_closest(const __grid_constant__ DeviceScene s, const float *rays,
                                                       uint32_t n, Hit *hits, float *t_out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 *r4 = reinterpret_cast<const float4 *>(rays) + 2u * i;
    float4 a = r4[0], b = r4[1];
    RayPre rp = precompute_ray(make3(a.x, a.y, a.z), make3(b.x, b.y, b.z));
    float tmax = b.w;
    Hit h;
    float t;
    if (trace_closest(s, rp, tmax, h, t)) {
        hits[i] = h;
        t_out[i] = t;
    } else {
        hits[i] = Hit{kInvalid, kInvalid, 0.0f, 0.0f};
        t_out[i] = -1.0f;
    }
}

__global__ void __launch_bounds__(128) k_trace_any(const __grid_constant__ DeviceScene s, const float *rays,
                                                   uint32_t n, uint32_t *occ) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 *r4 = reinterpret_cast<const float4 *>(rays) + 2u * i;
    float4 a = r4[0], b = r4[1];
    RayPre rp = precompute_ray(make3(a.x, a.y, a.z), make3(b.x, b.y, b.z));
    occ[i] = trace_any(s, rp, b.w) ? 1u : 0u;
}

// Paths are numbered frame-major: path p covers pixel p % (w*h) of frame
// frame_begin + p / (w*h), so neighbouring threads trace neighbouring pixels.
template <int N>
#ifndef VS_RENDER_MIN_BLOCKS
#define VS_RENDER_MIN_BLOCKS 1
#endif
__global__ void __launch_bounds__(128, VS_RENDER_MIN_BLOCKS)
    k_render(const __grid_constant__ DeviceScene s, uint32_t frame_begin, uint64_t path_count, float4 *radiance) {
    uint64_t p = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= path_count) return;
    uint32_t npix = s.cam.width * s.cam.height;
    uint32_t frame = frame_begin + static_cast<uint32_t>(p / npix);
    uint32_t pix = static_cast<uint32_t>(p % npix);
    uint32_t px = pix % s.cam.width, py = pix / s.cam.width;
    f3 L = trace_path<N>(s, px, py, frame);
    radiance[p] = make_float4(L.x, L.y, L.z, 1.0f);
}

// Persistent form of k_render with path regeneration.  A camera path ends
// after a data-dependent number of bounces (Russian roulette, misses), so a
// warp that traces one path per lane idles its finished lanes until the
// longest path ends.  Here each warp keeps 32 paths in flight: after every
// bounce the lanes whose path ended write its radiance and claim the next
// unclaimed path indices with one atomicAdd per warp on `next_path` (zero at
// launch).  Each path is still traced from its own sampler stream and written
// to radiance[p], so the output equals k_render's bit for bit.  Needs
// max_depth >= 1.
template <int N>
__global__ void __launch_bounds__(128, VS_RENDER_MIN_BLOCKS)
    k_render_regen(const __grid_constant__ DeviceScene s, uint32_t frame_begin, uint64_t path_count, float4 *radiance,
                   unsigned long long *next_path) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t npix = s.cam.width * s.cam.height;
    const uint32_t max_depth = s.ip.max_depth;
    PathState<N> ps;
    uint64_t p = 0;
    bool active = false;
    bool drained = false;  // warp-uniform: every path index has been claimed
    for (;;) {
        if (!drained) {
            const unsigned need = __ballot_sync(0xffffffffu, !active);
            if (need) {
                const int leader = __ffs(need) - 1;
                const unsigned count = static_cast<unsigned>(__popc(need));
                unsigned long long base = 0;
                if (static_cast<int>(lane) == leader) base = atomicAdd(next_path, static_cast<unsigned long long>(count));
                base = __shfl_sync(0xffffffffu, base, leader);
                if (base + count >= path_count) drained = true;
                if (!active) {
                    const uint64_t q = base + static_cast<unsigned>(__popc(need & ((1u << lane) - 1u)));
                    if (q < path_count) {
                        p = q;
                        const uint32_t frame = frame_begin + static_cast<uint32_t>(q / npix);
                        const uint32_t pix = static_cast<uint32_t>(q % npix);
                        path_start<N>(s, s.cam, pix % s.cam.width, pix / s.cam.width, frame, ps);
                        active = true;
                    }
                }
            }
        }
        if (!__any_sync(0xffffffffu, active)) break;
        if (active) {
            bool more = path_bounce<N>(s, ps, nullptr);
            if (more) more = ++ps.bounce < max_depth;
            if (!more) {
                const f3 Lw = ps.L * ps.filter_w;
                radiance[p] = make_float4(Lw.x, Lw.y, Lw.z, 1.0f);
                active = false;
            }
        }
    }
}

// NormalRadianceCollector::add_sample (normal.cpp:87-101) for frame_count
// consecutive frames: zero_if_nan_inf, then the running mean
// lerp(1 / (frame + 1), prev, value), in frame order.
__global__ void k_film_running_mean(const float4 *radiance, uint32_t npix, uint32_t frame_begin, uint32_t frame_count,
                                    float4 *film) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    float4 acc = frame_begin == 0 ? make_float4(0, 0, 0, 0) : film[i];
    for (uint32_t f = 0; f < frame_count; ++f) {
        float4 v = radiance[static_cast<size_t>(f) * npix + i];
        bool bad = isnan(v.x) || isnan(v.y) || isnan(v.z) || isinf(v.x) || isinf(v.y) || isinf(v.z);
        if (bad) v = make_float4(0, 0, 0, 0);
        float a = 1.0f / static_cast<float>(frame_begin + f + 1u);
        acc.x = acc.x + a * (v.x - acc.x);
        acc.y = acc.y + a * (v.y - acc.y);
        acc.z = acc.z + a * (v.z - acc.z);
        acc.w = acc.w + a * (v.w - acc.w);
    }
    film[i] = acc;
}

// FP64 film: per-pixel sums of the sanitised samples and the sample count,
// and (when sq4 is given) the sums of their squares, from which the
// per-pixel variance of the estimate follows.
__global__ void k_film_sum64(const float4 *radiance, uint32_t npix, uint32_t frame_begin, uint32_t frame_count,
                             double *sum4, double *sq4) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    double4 acc = frame_begin == 0 ? make_double4(0, 0, 0, 0) : reinterpret_cast<double4 *>(sum4)[i];
    double4 sq = make_double4(0, 0, 0, 0);
    if (sq4 && frame_begin != 0) sq = reinterpret_cast<double4 *>(sq4)[i];
    for (uint32_t f = 0; f < frame_count; ++f) {
        float4 v = radiance[static_cast<size_t>(f) * npix + i];
        bool bad = isnan(v.x) || isnan(v.y) || isnan(v.z) || isinf(v.x) || isinf(v.y) || isinf(v.z);
        if (bad) v = make_float4(0, 0, 0, 1);
        acc.x += v.x;
        acc.y += v.y;
        acc.z += v.z;
        acc.w += 1.0;
        sq.x += static_cast<double>(v.x) * v.x;
        sq.y += static_cast<double>(v.y) * v.y;
        sq.z += static_cast<double>(v.z) * v.z;
    }
    reinterpret_cast<double4 *>(sum4)[i] = acc;
    if (sq4) reinterpret_cast<double4 *>(sq4)[i] = sq;
}

// The tone mappers of tonemappers/impl.cpp: linear (identity), ACES (the
// fitted curve x(2.51x + 0.03) / (x(2.43x + 0.59) + 0.14), saturated) and
// Reinhard x / (x + 1).
__device__ __forceinline__ float tone_map(float x, uint32_t tm) {
    if (tm == kToneAces) return __saturatef((x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f));
    if (tm == kToneReinhard) return x / (x + 1.0f);
    return x;
}

// sRGB transfer function (IEC 61966-2-1), the gamma of the final picture.
__device__ __forceinline__ float linear_to_srgb(float v) {
    return v <= 0.0031308f ? 12.92f * v : 1.055f * powf(v, 1.0f / 2.4f) - 0.055f;
}

// The pictures of the linear film: exposure 1 - exp(-L * exposure)
// (RadianceCollector::apply_exposure, radiance_collector.cpp:24-26) and the
// tone mapper give the collector's output buffer (normal.cpp:86-101); the
// final picture maps that once more and applies the sRGB gamma unless the
// output is HDR (Postprocessor::tone_mapping, postprocessor.cpp:13-22;
// Pipeline::final_picture, pipeline.cpp:313-329).  8-bit output rounds the
// clamped value to the nearest of 255 steps.  One pixel per thread, float4
// in, float4 or uchar4 out.
__global__ void k_film_picture(const float4 *film, uint32_t npix, float exposure, uint32_t tm, uint32_t passes,
                               bool gamma, float4 *out, uchar4 *out8) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    const float4 v = film[i];
    float c[3] = {1.0f - expf(-v.x * exposure), 1.0f - expf(-v.y * exposure), 1.0f - expf(-v.z * exposure)};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        for (uint32_t p = 0; p < passes; ++p) c[k] = tone_map(c[k], tm);
        if (gamma) c[k] = linear_to_srgb(c[k]);
    }
    if (out8) {
        auto q = [](float x) { return static_cast<unsigned char>(__float2int_rn(__saturatef(x) * 255.0f)); };
        out8[i] = make_uchar4(q(c[0]), q(c[1]), q(c[2]), 255);
    } else {
        out[i] = make_float4(c[0], c[1], c[2], 1.0f);
    }
}

cudaError_t upload_spectral_consts(const float *x, const float *y, const float *z, const float *d65, float y_integral) {
    return upload_spectral_consts_tu(x, y, z, d65, y_integral);
}

cudaError_t launch_trace_closest(const DeviceScene &s, const float *rays, uint32_t n, Hit *hits, float *t,
                                 cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_trace_closest<<<(n + 127) / 128, 128, 0, st>>>(s, rays, n, hits, t);
    g_launches++;
    return cudaGetLastError();
}

// Sampler streams (parity hook): stream i starts at keys[i] = (px, py,
// sample, dim) and writes `draws` consecutive draws to out[i * draws ...].
__global__ void __launch_bounds__(128) k_sampler_stream(const uint4 *keys, uint32_t count, uint32_t draws,
                                                        uint32_t kind, uint32_t seed, float *out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    uint4 k = keys[i];
    Sampler smp;
    smp.start(k.x, k.y, k.z, k.w, kind, seed);
    float *o = out + static_cast<uint64_t>(i) * draws;
    for (uint32_t j = 0; j < draws; ++j) o[j] = smp.next();
}

cudaError_t launch_sampler_stream(const uint4 *keys, uint32_t count, uint32_t draws, uint32_t kind, uint32_t seed,
                                  float *out, cudaStream_t st) {
    if (count == 0 || draws == 0) return cudaSuccess;
    k_sampler_stream<<<(count + 127) / 128, 128, 0, st>>>(keys, count, draws, kind, seed, out);
    g_launches++;
    return cudaGetLastError();
}

cudaError_t launch_trace_any(const DeviceScene &s, const float *rays, uint32_t n, uint32_t *occ, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_trace_any<<<(n + 127) / 128, 128, 0, st>>>(s, rays, n, occ);
    g_launches++;
    return cudaGetLastError();
}

cudaError_t launch_render(const DeviceScene &s, uint32_t frame_begin, uint32_t frame_count, float4 *radiance,
                          cudaStream_t st, unsigned long long *path_counter) {
    uint64_t paths = static_cast<uint64_t>(s.cam.width) * s.cam.height * frame_count;
    if (paths == 0) return cudaSuccess;
    uint64_t blocks = (paths + 127) / 128;
    if (blocks > 0x7fffffffull) return cudaErrorInvalidValue;
    if (s.ip.spectrum_dim < 1 || s.ip.spectrum_dim > 4) return cudaErrorInvalidValue;
    if (path_counter && s.ip.max_depth > 0) {
        // One resident wave: SMs x blocks per SM, capped by the work.
        static std::atomic<int> resident[64][5];
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
        const int n = static_cast<int>(s.ip.spectrum_dim);
        int wave = resident[dev][n].load();
        if (wave == 0) {
            int sms = 0, per_sm = 0;
            e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (e != cudaSuccess) return e;
            switch (n) {
                case 1: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_render_regen<1>, 128, 0); break;
                case 2: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_render_regen<2>, 128, 0); break;
                case 3: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_render_regen<3>, 128, 0); break;
                default: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_render_regen<4>, 128, 0); break;
            }
            if (e != cudaSuccess) return e;
            wave = sms * (per_sm > 0 ? per_sm : 1);
            resident[dev][n].store(wave);
        }
        unsigned grid = static_cast<unsigned>(std::min<uint64_t>(blocks, static_cast<uint64_t>(wave)));
        e = cudaMemsetAsync(path_counter, 0, sizeof(unsigned long long), st);
        if (e != cudaSuccess) return e;
        switch (n) {
            case 1: k_render_regen<1><<<grid, 128, 0, st>>>(s, frame_begin, paths, radiance, path_counter); break;
            case 2: k_render_regen<2><<<grid, 128, 0, st>>>(s, frame_begin, paths, radiance, path_counter); break;
            case 3: k_render_regen<3><<<grid, 128, 0, st>>>(s, frame_begin, paths, radiance, path_counter); break;
            default: k_render_regen<4><<<grid, 128, 0, st>>>(s, frame_begin, paths, radiance, path_counter); break;
        }
        g_launches++;
        return cudaGetLastError();
    }
    switch (s.ip.spectrum_dim) {
        case 1: k_render<1><<<static_cast<unsigned>(blocks), 128, 0, st>>>(s, frame_begin, paths, radiance); break;
        case 2: k_render<2><<<static_cast<unsigned>(blocks), 128, 0, st>>>(s, frame_begin, paths, radiance); break;
        case 3: k_render<3><<<static_cast<unsigned>(blocks), 128, 0, st>>>(s, frame_begin, paths, radiance); break;
        default: k_render<4><<<static_cast<unsigned>(blocks), 128, 0, st>>>(s, frame_begin, paths, radiance); break;
    }
    g_launches++;
    return cudaGetLastError();
}

cudaError_t launch_film(const float4 *radiance, uint32_t npix, uint32_t frame_begin, uint32_t frame_count, float4 *film32,
                        double *film64, cudaStream_t st, double *film64sq) {
    unsigned blocks = (npix + 255) / 256;
    if (film32) {
        k_film_running_mean<<<blocks, 256, 0, st>>>(radiance, npix, frame_begin, frame_count, film32);
        g_launches++;
    }
    if (film64) {
        k_film_sum64<<<blocks, 256, 0, st>>>(radiance, npix, frame_begin, frame_count, film64, film64sq);
        g_launches++;
    }
    return cudaGetLastError();
}

cudaError_t launch_picture(const float4 *film, uint32_t npix, float exposure, uint32_t tone_mapper, uint32_t passes,
                           bool gamma, float4 *out, uchar4 *out8, cudaStream_t st) {
    k_film_picture<<<(npix + 255) / 256, 256, 0, st>>>(film, npix, exposure, tone_mapper, passes, gamma, out, out8);
    g_launches++;
    return cudaGetLastError();
}

}  // namespace vs

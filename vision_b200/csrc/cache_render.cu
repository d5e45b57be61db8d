// Cache-terminated path tracing with the radiance-cache MLP (mlp.cu).
//
// Per frame:
//   k_cache_paths    one camera path per pixel through `query_depth` bounces
//                    (emission with MIS and next-event estimation as in
//                    IlluminationIntegrator::Li, integrator.cpp:134-283); at
//                    the next surface it writes the vertex's encoded features
//                    and its path state instead of continuing.  Every
//                    `train_stride`-th pixel (offset per frame) is a training
//                    path: it goes on for `suffix_depth` more bounces,
//                    gathering the suffix radiance with the throughput
//                    restarted at the query vertex, and writes the features of
//                    the suffix end.
//   mlp_infer        the cache at every query vertex and every suffix end
//   k_cache_resolve  pixel radiance = gathered radiance + throughput times the
//                    cache's radiance at the path's three hero wavelengths
//                    into the film; training target = suffix radiance +
//                    suffix throughput times the cache at the suffix end
//                    (self-training), per wavelength.
// The cache predicts spectral radiance at the path's three hero wavelengths
// (its three outputs), leaving a vertex toward the previous one, without the
// vertex's own emission (which the path adds with its MIS weight): the path
// multiplies it by its own spectral throughput, so no RGB round trip enters
// the estimate.
// Features (64): position in the scene bounds, sin/cos(2^k pi p) for k = 0..7
// on each axis (48); outgoing direction (3); shading normal (3); roughness (1);
// albedo (3); sin/cos(2^k pi u) of the hero wavelength u = (lambda_0 - 360) /
// 470 for k = 0..2 (6).
#include "vs_cache_render.h"
#include "vs_wavefront.cuh"
#include "vs_launch.h"

#include <cuda_bf16.h>

#include <algorithm>

namespace vs {

namespace {

constexpr int CN = 3;  // hero wavelengths of cache-rendered scenes = cache outputs
using CSpec = Spec<CN>;
using CWl = Wavelengths<CN>;

__device__ __forceinline__ uint32_t bf2(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t *>(&h);
}

__device__ void encode(const CacheFrameParams &p, const Interaction &it, float lambda0, uint16_t *out) {
    float f[64];
    const float pos[3] = {clampf((it.pos.x - p.bmin.x) * p.binv.x, 0.0f, 1.0f),
                          clampf((it.pos.y - p.bmin.y) * p.binv.y, 0.0f, 1.0f),
                          clampf((it.pos.z - p.bmin.z) * p.binv.z, 0.0f, 1.0f)};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float scale = 1.0f;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            float sn, cs;
            sincospif(scale * pos[a], &sn, &cs);
            f[16 * a + 2 * k] = sn;
            f[16 * a + 2 * k + 1] = cs;
            scale *= 2.0f;
        }
    }
    const float4 m = __ldg(&p.mat[it.mat]);
    const f3 n = it.shading.z;
    const float wo[3] = {it.wo.x, it.wo.y, it.wo.z};
    f[48] = wo[0];
    f[49] = wo[1];
    f[50] = wo[2];
    f[51] = n.x;
    f[52] = n.y;
    f[53] = n.z;
    f[54] = m.w;
    f[55] = m.x;
    f[56] = m.y;
    f[57] = m.z;
    const float u = (lambda0 - 360.0f) * (1.0f / 470.0f);
    sincospif(u, &f[58], &f[59]);
    sincospif(2.0f * u, &f[60], &f[61]);
    sincospif(4.0f * u, &f[62], &f[63]);
    uint4 *dst = reinterpret_cast<uint4 *>(out);
#pragma unroll
    for (int c = 0; c < 8; ++c)
        dst[c] = make_uint4(bf2(f[8 * c], f[8 * c + 1]), bf2(f[8 * c + 2], f[8 * c + 3]),
                            bf2(f[8 * c + 4], f[8 * c + 5]), bf2(f[8 * c + 6], f[8 * c + 7]));
}

__device__ __forceinline__ float4 spec4(const CSpec &s, float w) { return make_float4(s.v[0], s.v[1], s.v[2], w); }
__device__ __forceinline__ CSpec spec_of(float4 v) {
    CSpec s;
    s.v[0] = v.x;
    s.v[1] = v.y;
    s.v[2] = v.z;
    return s;
}
// Cache output: spectral radiance at the three hero wavelengths (negative
// predictions clamped to zero).
__device__ __forceinline__ CSpec cache_radiance(float4 o) {
    CSpec s;
    s.v[0] = fmaxf(o.x, 0.0f);
    s.v[1] = fmaxf(o.y, 0.0f);
    s.v[2] = fmaxf(o.z, 0.0f);
    return s;
}
__device__ __forceinline__ float4 wl4(const CWl &w, bool pdf) {
    return pdf ? make_float4(w.pdf[0], w.pdf[1], w.pdf[2], 0.0f) : make_float4(w.lambda[0], w.lambda[1], w.lambda[2], 0.0f);
}

}  // namespace

__global__ void __launch_bounds__(128) k_cache_paths(const __grid_constant__ DeviceScene s,
                                                     const __grid_constant__ CacheFrameParams p) {
    const uint32_t npix = s.cam.width * s.cam.height;
    const uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= npix) return;
    const uint32_t px = pix % s.cam.width, py = pix / s.cam.width;
    const IntegratorParams &ip = s.ip;
    // Training path?  Samples j = 0 .. n_train-1 sit at pixels offset + j * stride.
    bool train = false;
    uint32_t tj = 0;
    if (p.n_train && pix >= p.train_offset && (pix - p.train_offset) % p.train_stride == 0) {
        tj = (pix - p.train_offset) / p.train_stride;
        train = tj < p.n_train;
    }
    Sampler smp;
    smp.start(px, py, p.frame, 0xffffffffu, ip.sampler, ip.seed);
    CWl wl = ip.srgb ? rgb_wavelengths<CN>() : sample_wavelengths<CN>(smp.next());
    smp.start(px, py, p.frame, 0u, ip.sampler, ip.seed);
    f2 p_film;
    f3 ro, rd;
    const float filter_w = camera_ray(s, s.cam, smp, px, py, p_film, ro, rd);

    CSpec throughput = CSpec::fill(1.0f);
    f3 ret = make3(0.0f);               // radiance before the query vertex (linear sRGB)
    CSpec suffix = CSpec::fill(0.0f);   // training suffix radiance at the hero wavelengths,
                                        // throughput restarted at the query vertex
    bool in_suffix = false;
    float scatter_pdf = 1e16f;
    float eta_scale = 1.0f;
    CacheQueryRec rec;
    rec.l_valid = make_float4(0, 0, 0, 0);
    bool wrote_query = false;
    const uint32_t end_depth = p.query_depth + p.suffix_depth;
    // Adds a spectral contribution (already weighted by the throughput) to the
    // pixel radiance or, inside a training suffix, to the suffix radiance.
    auto gather = [&](const CSpec &c) {
        if (in_suffix) suffix = suffix + c;
        else ret += linear_srgb<CN>(c, wl);
    };
    for (uint32_t bounce = 0; bounce <= end_depth; ++bounce) {
        RayPre rp = precompute_ray(ro, rd);
        Hit hit;
        float t_hit;
        const bool hit_any = trace_closest(s, rp, 3.402823466e+38f, hit, t_hit);
        if (!hit_any) {
            if (s.has_env) {
                CSpec Le;
                float lpdf;
                env_eval<CN>(s, normalize((ro + rd) - ro), wl, Le, lpdf);
                lpdf *= light_pmf<CN>(s, s.env_index);
                float weight = scatter_pdf / (scatter_pdf + lpdf);
                if (ip.mis_mode == 2u) weight = 1.0f;
                else if (ip.mis_mode == 1u) weight = bounce == 0 ? weight : 0.0f;
                gather(Le * throughput * weight);
            }
            break;
        }
        Interaction it = surface_interaction(s, hit, rd, true);
        if (it.light != kInvalid) {
            CSpec Le;
            float lpdf;
            eval_hit_light<CN>(s, it, ro, wl, Le, lpdf);
            float weight = scatter_pdf / (scatter_pdf + lpdf);
            if (ip.mis_mode == 2u) weight = 1.0f;
            else if (ip.mis_mode == 1u) weight = bounce == 0 ? weight : 0.0f;
            gather(Le * throughput * weight);
        }
        if (bounce == p.query_depth) {
            encode(p, it, wl.lambda[0], p.q_feat + static_cast<size_t>(pix) * 64u);
            rec.t = spec4(throughput, filter_w);
            rec.lambda = wl4(wl, false);
            rec.pdf = wl4(wl, true);
            rec.l_valid = make_float4(ret.x, ret.y, ret.z, 1.0f);
            wrote_query = true;
            if (!train) break;
            encode(p, it, wl.lambda[0], p.t_feat + static_cast<size_t>(tj) * 64u);
            in_suffix = true;
            throughput = CSpec::fill(1.0f);
        }
        if (bounce == end_depth) {
            // Suffix end: the cache continues from here.
            encode(p, it, wl.lambda[0], p.b_feat + static_cast<size_t>(tj) * 64u);
            CacheTrainRec tr;
            tr.suffix_valid = spec4(suffix, 1.0f);
            tr.t = spec4(throughput, 0.0f);
            tr.lambda = wl4(wl, false);
            tr.pdf = wl4(wl, true);
            p.t_rec[tj] = tr;
            in_suffix = false;
            break;
        }
        float u_light = smp.next();
        f2 u_surf = smp.next2();
        LightSample<CN> ls = sample_light<CN>(s, it, u_light, u_surf, wl);
        Ray sh = spawn_ray_to(it.pos, it.ng, ls.p_light);
        bool occluded = trace_any(s, precompute_ray(sh.o, sh.d), sh.tmax);
        Material mat = s.materials[it.mat];
        Bsdf<CN> bsdf = make_bsdf<CN>(s, mat, it.shading, it.ng, it.wo, it.uv, wl);
        if (bsdf.dispersive) invalidate_secondary<CN>(wl);
        f3 wi_light = normalize(ls.p_light - it.pos);
        BsdfEval<CN> se = bsdf.evaluate(it.wo, wi_light, nullptr);
        BsdfSample<CN> bs = bsdf.sample(it.wo, smp);
        CSpec Ld = CSpec::fill(0.0f);
        const bool delta = ls.pdf < 0.0f;
        const float l_pdf = delta ? -ls.pdf : ls.pdf;
        float w_mis = delta ? 1.0f : ls.pdf / (ls.pdf + se.pdf);
        if (ip.mis_mode == 1u) w_mis = 1.0f;
        if (!occluded && se.valid() && l_pdf > 0.0f) Ld = ls.L * se.f * (w_mis / l_pdf);
        if (ip.mis_mode != 2u) gather(throughput * Ld);
        eta_scale *= sqr(bs.eta);
        float lum = throughput.max();
        if (!bs.eval.valid() || lum == 0.0f) break;
        throughput = throughput * bs.eval.throughput();
        if (eta_scale * lum < ip.rr_threshold && bounce >= ip.min_depth) {
            float q = fminf(0.95f, lum);
            float rr = smp.next();
            if (q < rr) break;
            throughput = throughput * (1.0f / q);
        }
        if (throughput.all_zero()) break;
        scatter_pdf = bs.eval.pdf;
        Ray nr = spawn_ray(it.pos, it.ng, bs.wi);
        ro = nr.o;
        rd = nr.d;
    }
    if (!wrote_query) rec.l_valid = make_float4(ret.x * filter_w, ret.y * filter_w, ret.z * filter_w, 0.0f);
    p.q_rec[pix] = rec;
    if (train && (in_suffix || !wrote_query)) {
        // The suffix ended before its last vertex (no bootstrap term), or the
        // path before the query vertex (an empty sample with zero features).
        CacheTrainRec tr;
        tr.suffix_valid = spec4(suffix, 0.0f);
        tr.t = make_float4(0, 0, 0, 0);
        tr.lambda = wl4(wl, false);
        tr.pdf = wl4(wl, true);
        p.t_rec[tj] = tr;
        uint4 *b = reinterpret_cast<uint4 *>(p.b_feat + static_cast<size_t>(tj) * 64u);
        uint4 *a = reinterpret_cast<uint4 *>(p.t_feat + static_cast<size_t>(tj) * 64u);
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            b[c] = make_uint4(0, 0, 0, 0);
            if (!wrote_query) a[c] = make_uint4(0, 0, 0, 0);
        }
    }
}

namespace {

__device__ __forceinline__ CWl wl_of(float4 lambda, float4 pdf) {
    CWl w;
    w.lambda[0] = lambda.x;
    w.lambda[1] = lambda.y;
    w.lambda[2] = lambda.z;
    w.pdf[0] = pdf.x;
    w.pdf[1] = pdf.y;
    w.pdf[2] = pdf.z;
    return w;
}

__device__ __forceinline__ bool bad3(f3 v) {
    return isnan(v.x) || isnan(v.y) || isnan(v.z) || isinf(v.x) || isinf(v.y) || isinf(v.z);
}

}  // namespace

// Pixel radiance into the film (running mean of frame film_index, optional
// FP64 sums) and the training targets.
// `ended` (wavefront frames): radiance of the paths that ended before their
// query vertex, whose query records stay zero; null when the records carry it.
__global__ void k_cache_resolve(const __grid_constant__ DeviceScene s, const __grid_constant__ CacheFrameParams p,
                                float4 *film32, double *film64, uint32_t film_index, const float4 *ended) {
    const uint32_t npix = s.cam.width * s.cam.height;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < npix) {
        CacheQueryRec r = p.q_rec[i];
        f3 L = make3(r.l_valid.x, r.l_valid.y, r.l_valid.z);
        if (ended && r.l_valid.w == 0.0f) L = make3(ended[i].x, ended[i].y, ended[i].z);
        if (r.l_valid.w != 0.0f) {
            CWl wl = wl_of(r.lambda, r.pdf);
            L += linear_srgb<CN>(spec_of(r.t) * cache_radiance(p.q_out[i]), wl);
            L = L * r.t.w;  // the camera sample's filter weight
        }
        if (bad3(L)) L = make3(0.0f);
        float4 acc = film_index == 0 ? make_float4(0, 0, 0, 0) : film32[i];
        float a = 1.0f / static_cast<float>(film_index + 1u);
        acc.x = acc.x + a * (L.x - acc.x);
        acc.y = acc.y + a * (L.y - acc.y);
        acc.z = acc.z + a * (L.z - acc.z);
        acc.w = acc.w + a * (1.0f - acc.w);
        film32[i] = acc;
        if (film64) {
            double4 d = film_index == 0 ? make_double4(0, 0, 0, 0) : reinterpret_cast<double4 *>(film64)[i];
            d.x += L.x;
            d.y += L.y;
            d.z += L.z;
            d.w += 1.0;
            reinterpret_cast<double4 *>(film64)[i] = d;
        }
    }
    if (i < p.n_train) {
        CacheTrainRec r = p.t_rec[i];
        CSpec T = spec_of(r.suffix_valid);
        if (r.suffix_valid.w != 0.0f) T = T + spec_of(r.t) * cache_radiance(p.b_out[i]);
        f3 v = make3(T.v[0], T.v[1], T.v[2]);
        if (bad3(v)) v = make3(0.0f);
        p.targets[i] = make_float4(v.x, v.y, v.z, 0.0f);
    }
}

cudaError_t upload_spectral_consts_cache(const float *x, const float *y, const float *z, const float *d65,
                                         float y_integral) {
    return upload_spectral_consts_tu(x, y, z, d65, y_integral);
}

cudaError_t launch_cache_frame(const DeviceScene &s, const CacheFrameParams &p, const MlpState &mlp, float4 *film32,
                               double *film64, uint32_t film_index, cudaStream_t st, unsigned *launches) {
    const uint32_t npix = s.cam.width * s.cam.height;
    unsigned n = 0;
    k_cache_paths<<<(npix + 127) / 128, 128, 0, st>>>(s, p);
    ++n;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = mlp_infer(mlp, p.q_feat, npix, p.q_out, st);
    ++n;
    if (e == cudaSuccess && p.n_train) {
        e = mlp_infer(mlp, p.b_feat, p.n_train, p.b_out, st);
        ++n;
    }
    if (e == cudaSuccess) {
        uint32_t m = npix > p.n_train ? npix : p.n_train;
        k_cache_resolve<<<(m + 255) / 256, 256, 0, st>>>(s, p, film32, film64, film_index, nullptr);
        ++n;
        e = cudaGetLastError();
    }
    if (launches) *launches = n;
    return e;
}

// ---------------------------------------------------------------------------
// Wavefront form of the cache-terminated frame.  The two bounces before the
// query vertex run as wavefront passes (closest hit, material-sorted
// shading, shadow rays); k_cache_query adds the query vertex's emission,
// encodes it and writes its record; k_cache_suffix traces the training
// suffixes of the (compacted) training paths, so a warp no longer carries one
// training lane through two extra bounces.  Every path makes the same sampler
// draws and sums in the same order as k_cache_paths, so the records, features
// and targets are those of k_cache_paths.
// ---------------------------------------------------------------------------
namespace {

struct CacheScene {
    const DeviceScene *s;
    __device__ __forceinline__ const DeviceScene &operator()(uint32_t) const { return *s; }
};

// Training sample of pixel `pix`, or n_train when it is not a training pixel.
__device__ __forceinline__ uint32_t train_index(const CacheFrameParams &p, uint32_t pix) {
    if (!p.n_train || pix < p.train_offset || (pix - p.train_offset) % p.train_stride != 0) return p.n_train;
    const uint32_t tj = (pix - p.train_offset) / p.train_stride;
    return tj < p.n_train ? tj : p.n_train;
}

}  // namespace

__global__ void __launch_bounds__(128) k_cw_generate(const __grid_constant__ DeviceScene s,
                                                     const __grid_constant__ WfBuffers b, uint32_t frame, uint32_t n,
                                                     float4 *ended) {
    wf::generate<CN>(s, s.cam, b, frame, 0, n, ended);
}

template <int L>
__global__ void __launch_bounds__(128) k_cw_extend(const __grid_constant__ DeviceScene s,
                                                   const __grid_constant__ WfBuffers b, uint32_t cur) {
    wf::extend<L>(CacheScene{&s}, b, cur);
}

template <uint32_t C>
__global__ void __launch_bounds__(128) k_cw_shade(const __grid_constant__ DeviceScene s,
                                                  const __grid_constant__ WfBuffers b, uint32_t cur, float4 *ended) {
    wf::shade<CN, C>(CacheScene{&s}, b, cur, 0, ended);
}

template <int L>
__global__ void __launch_bounds__(128) k_cw_shadow(const __grid_constant__ DeviceScene s,
                                                   const __grid_constant__ WfBuffers b, float4 *ended) {
    wf::shadow<L>(CacheScene{&s}, b, 0, ended);
}

// Query vertices (the hits of the bounce-`query_depth` rays of queue `cur`).
__global__ void __launch_bounds__(128) k_cache_query(const __grid_constant__ DeviceScene s,
                                                     const __grid_constant__ CacheFrameParams p,
                                                     const __grid_constant__ WfBuffers b, uint32_t cur, float4 *ended,
                                                     uint32_t *suffix_list, uint32_t *suffix_count) {
    const uint32_t n = b.count[cur];
    const uint32_t *q = b.queue[cur];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t slot = q[i];
        PathState<CN> ps;
        wf::load<CN>(CacheScene{&s}, b, slot, ps);
        const Hit h = b.hit[slot];
        if (h.inst_id == kInvalid) {
            miss_emission<CN>(s, ps, RgbAcc<CN>{});
            const f3 Lw = ps.L * ps.filter_w;
            ended[slot] = make_float4(Lw.x, Lw.y, Lw.z, 1.0f);
            continue;
        }
        const Interaction it = surface_interaction(s, h, ps.rd, true);
        hit_emission<CN>(s, ps, it, RgbAcc<CN>{});
        encode(p, it, ps.wl.lambda[0], p.q_feat + static_cast<size_t>(slot) * 64u);
        CacheQueryRec rec;
        rec.t = spec4(ps.throughput, ps.filter_w);
        rec.lambda = wl4(ps.wl, false);
        rec.pdf = wl4(ps.wl, true);
        rec.l_valid = make_float4(ps.L.x, ps.L.y, ps.L.z, 1.0f);
        p.q_rec[slot] = rec;
        const uint32_t tj = train_index(p, slot);
        if (tj < p.n_train) {
            encode(p, it, ps.wl.lambda[0], p.t_feat + static_cast<size_t>(tj) * 64u);
            suffix_list[wf::queue_push(suffix_count)] = slot;
        }
    }
}

// Training suffixes: `suffix_depth` more bounces from the query vertex with the
// throughput restarted there, gathered per hero wavelength, then the
// features of the suffix end (bootstrap vertex).
__global__ void __launch_bounds__(128) k_cache_suffix(const __grid_constant__ DeviceScene s,
                                                      const __grid_constant__ CacheFrameParams p,
                                                      const __grid_constant__ WfBuffers b,
                                                      const uint32_t *suffix_list, const uint32_t *suffix_count) {
    const uint32_t n = *suffix_count;
    const uint32_t end_depth = p.query_depth + p.suffix_depth;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t slot = suffix_list[k];
        const uint32_t tj = train_index(p, slot);
        PathState<CN> ps;
        wf::load<CN>(CacheScene{&s}, b, slot, ps);
        CSpec suffix = CSpec::fill(0.0f);
        const SpecAcc<CN> acc{&suffix};
        ps.throughput = CSpec::fill(1.0f);
        ShadowQuery sq;
        bool more = path_shade_acc<CN, true, kAllMaterials>(s, ps, true, b.hit[slot], nullptr, sq, acc, false);
        bool complete = false;
        while (more) {
            ++ps.bounce;
            Hit h;
            float t_hit;
            const bool hit_any = trace_closest(s, precompute_ray(ps.ro, ps.rd), 3.402823466e+38f, h, t_hit);
            if (ps.bounce == end_depth) {
                if (!hit_any) {
                    miss_emission<CN>(s, ps, acc);
                    break;
                }
                const Interaction it = surface_interaction(s, h, ps.rd, true);
                hit_emission<CN>(s, ps, it, acc);
                encode(p, it, ps.wl.lambda[0], p.b_feat + static_cast<size_t>(tj) * 64u);
                complete = true;
                break;
            }
            more = path_shade_acc<CN, true, kAllMaterials>(s, ps, hit_any, h, nullptr, sq, acc, true);
        }
        CacheTrainRec tr;
        tr.suffix_valid = spec4(suffix, complete ? 1.0f : 0.0f);
        tr.t = complete ? spec4(ps.throughput, 0.0f) : make_float4(0, 0, 0, 0);
        tr.lambda = wl4(ps.wl, false);
        tr.pdf = wl4(ps.wl, true);
        p.t_rec[tj] = tr;
    }
}

namespace {

template <typename K>
unsigned wave_grid(K kernel) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 128, 0);
    return static_cast<unsigned>(std::max(1, sms * std::max(per_sm, 1)));
}

template <uint32_t C>
void cw_shade(uint32_t mask, const DeviceScene &s, const WfBuffers &b, uint32_t cur, float4 *ended, cudaStream_t st,
              unsigned &n) {
    static unsigned grid = 0;
    if (!((mask >> C) & 1u)) return;
    if (!grid) grid = wave_grid(k_cw_shade<C>);
    k_cw_shade<C><<<grid, 128, 0, st>>>(s, b, cur, ended);
    ++n;
}

}  // namespace

cudaError_t launch_cache_frame_wavefront(const DeviceScene &s, const CacheFrameParams &p, const MlpState &mlp,
                                         float4 *film32, double *film64, uint32_t film_index, const WfBuffers &b,
                                         uint32_t class_mask, float4 *ended, uint32_t *suffix_list,
                                         uint32_t *suffix_count, cudaStream_t st, unsigned *launches) {
    const uint32_t npix = s.cam.width * s.cam.height;
    if (npix > b.capacity) return cudaErrorInvalidValue;
    static unsigned g_gen = 0, g_ext = 0, g_shadow = 0, g_query = 0, g_suffix = 0, g_ext2 = 0, g_shadow2 = 0;
    if (!g_gen) {
        g_gen = wave_grid(k_cw_generate);
        g_ext = wave_grid(k_cw_extend<kLevelsFlat>);
        g_shadow = wave_grid(k_cw_shadow<kLevelsFlat>);
        g_ext2 = wave_grid(k_cw_extend<kLevelsTwo>);
        g_shadow2 = wave_grid(k_cw_shadow<kLevelsTwo>);
        g_query = wave_grid(k_cache_query);
        g_suffix = wave_grid(k_cache_suffix);
    }
    // The prefix ends at the query vertex, not at the scene's depth limit
    // (k_cache_paths does not apply it either).
    DeviceScene sv = s;
    sv.ip.max_depth = 0xffffffffu;
    const bool two = s.two_level != 0u;
    auto extend = [&](uint32_t cur) {
        if (two) k_cw_extend<kLevelsTwo><<<g_ext2, 128, 0, st>>>(sv, b, cur);
        else k_cw_extend<kLevelsFlat><<<g_ext, 128, 0, st>>>(sv, b, cur);
    };
    cudaError_t e = cudaMemsetAsync(p.q_rec, 0, sizeof(CacheQueryRec) * npix, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(suffix_count, 0, sizeof(uint32_t), st);
    if (e == cudaSuccess && p.n_train) {
        e = cudaMemsetAsync(p.t_rec, 0, sizeof(CacheTrainRec) * p.n_train, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(p.t_feat, 0, 128ull * p.n_train, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(p.b_feat, 0, 128ull * p.n_train, st);
    }
    if (e != cudaSuccess) return e;
    unsigned n = 0;
    const uint32_t mask = class_mask | 1u;
    k_cw_generate<<<std::min<unsigned>(g_gen, (npix + 127) / 128), 128, 0, st>>>(sv, b, p.frame, npix, ended);
    ++n;
    for (uint32_t bounce = 0; bounce < p.query_depth; ++bounce) {
        const uint32_t cur = bounce & 1u;
        extend(cur);
        cw_shade<0>(mask, sv, b, cur, ended, st, n);
        cw_shade<1>(mask, sv, b, cur, ended, st, n);
        cw_shade<2>(mask, sv, b, cur, ended, st, n);
        cw_shade<3>(mask, sv, b, cur, ended, st, n);
        cw_shade<4>(mask, sv, b, cur, ended, st, n);
        cw_shade<5>(mask, sv, b, cur, ended, st, n);
        cw_shade<6>(mask, sv, b, cur, ended, st, n);
        if (two) k_cw_shadow<kLevelsTwo><<<g_shadow2, 128, 0, st>>>(sv, b, ended);
        else k_cw_shadow<kLevelsFlat><<<g_shadow, 128, 0, st>>>(sv, b, ended);
        n += 2;
    }
    const uint32_t cur = p.query_depth & 1u;
    extend(cur);
    k_cache_query<<<g_query, 128, 0, st>>>(sv, p, b, cur, ended, suffix_list, suffix_count);
    n += 2;
    if (p.n_train) {
        k_cache_suffix<<<std::min<unsigned>(g_suffix, (p.n_train + 127) / 128), 128, 0, st>>>(sv, p, b, suffix_list,
                                                                                           suffix_count);
        ++n;
    }
    e = cudaGetLastError();
    if (e == cudaSuccess) e = mlp_infer(mlp, p.q_feat, npix, p.q_out, st);
    ++n;
    if (e == cudaSuccess && p.n_train) {
        e = mlp_infer(mlp, p.b_feat, p.n_train, p.b_out, st);
        ++n;
    }
    if (e == cudaSuccess) {
        const uint32_t m = npix > p.n_train ? npix : p.n_train;
        k_cache_resolve<<<(m + 255) / 256, 256, 0, st>>>(s, p, film32, film64, film_index, ended);
        ++n;
        e = cudaGetLastError();
    }
    if (launches) *launches = n;
    return e;
}

}  // namespace vs

// Per-path integrator of the megakernel: surface interaction, area-light
// sampling, BSDF evaluation/sampling and the bounce loop of
// IlluminationIntegrator::Li (src/base/integrator.cpp:134-283).
#pragma once

#include "vs_device.cuh"
#include "vs_bsdf.cuh"
#include "vs_env.cuh"

namespace vs {

// Geometry::compute_surface_interaction (src/base/mgr/geometry.cpp:78-165).
// Positions and vertex normals are stored in world space, so the instance
// transform of the reference is folded into the scene build.  The shading
// frame follows PartialDerivative::update (interaction.h:87-110) and is kept
// orthonormal.
struct Interaction {
    f3 pos;
    f3 ng;
    f3 wo;
    Frame shading;
    f2 uv;
    float prim_area;
    uint32_t prim;
    uint32_t inst;
    uint32_t mat;
    uint32_t light;
};

__device__ __forceinline__ f3 ld3(const float4 &v) { return {v.x, v.y, v.z}; }

__device__ __forceinline__ void load_triangle(const DeviceScene &s, uint32_t prim, uint4 &idx, float4 a[2],
                                              float4 b[2], float4 c[2]) {
    idx = __ldg(&s.prims[prim]);
    a[0] = __ldg(&s.vtx[2u * idx.x]); a[1] = __ldg(&s.vtx[2u * idx.x + 1u]);
    b[0] = __ldg(&s.vtx[2u * idx.y]); b[1] = __ldg(&s.vtx[2u * idx.y + 1u]);
    c[0] = __ldg(&s.vtx[2u * idx.z]); c[1] = __ldg(&s.vtx[2u * idx.z + 1u]);
}

__device__ __forceinline__ Interaction surface_interaction(const DeviceScene &s, const Hit &hit, f3 ray_dir,
                                                           bool complete) {
    Interaction it;
    uint4 idx;
    float4 A[2], B[2], C[2];
    load_triangle(s, hit.prim_id, idx, A, B, C);
    f3 p0 = ld3(A[0]), p1 = ld3(B[0]), p2 = ld3(C[0]);
    float w = 1.0f - hit.u - hit.v;
    it.pos = p0 * w + p1 * hit.u + p2 * hit.v;
    f3 dp02 = p0 - p2, dp12 = p1 - p2;
    f3 ng_un = cross(dp02, dp12);
    it.prim_area = 0.5f * length(ng_un);
    it.ng = normalize(ng_un);
    f2 uv0 = {A[0].w, A[1].w}, uv1 = {B[0].w, B[1].w}, uv2 = {C[0].w, C[1].w};
    it.uv = {uv0.x * w + uv1.x * hit.u + uv2.x * hit.v, uv0.y * w + uv1.y * hit.u + uv2.y * hit.v};
    it.prim = hit.prim_id;
    it.inst = idx.w;
    Instance inst = s.instances[idx.w];
    it.mat = inst.mat_id;
    it.light = inst.light_id;
    it.wo = normalize(-ray_dir);
    if (complete) {
        f2 duv02 = uv0 - uv2, duv12 = uv1 - uv2;
        float det = duv02.x * duv12.y - duv02.y * duv12.x;
        f3 dp_dv;
        if (fabsf(det) < 1e-8f) {
            dp_dv = normalize(p2 - p0);
        } else {
            float inv_det = 1.0f / det;
            dp_dv = (dp12 * duv02.x - dp02 * duv12.x) * inv_det;
        }
        f3 n = ld3(A[1]) * w + ld3(B[1]) * hit.u + ld3(C[1]) * hit.v;
        f3 ns = is_zero(n) ? it.ng : normalize(n);
        f3 x = normalize(cross(ns, dp_dv));
        f3 y = normalize(cross(ns, x));
        it.shading = {x, y, ns};
    }
    return it;
}

// Light sample (LightSampler::sample_wi, lightsampler.cpp:210-216 and
// AreaLight::sample_wi, area.cpp:120-149).
template <int N>
struct LightSample {
    Spec<N> L;
    float pdf;
    f3 p_light;
};

__device__ __forceinline__ uint32_t alias_sample(const AliasEntry *table, uint32_t size, float u,
                                                 float *u_remapped) {
    u = u * static_cast<float>(size);
    uint32_t idx = min(static_cast<uint32_t>(u), size - 1u);
    u = fminf(u - static_cast<float>(idx), kOneMinusEpsilon);
    AliasEntry e = table[idx];
    bool keep = u < e.prob;
    if (u_remapped)
        *u_remapped = keep ? fminf(u / e.prob, kOneMinusEpsilon) : fminf((1.0f - u) / (1.0f - e.prob), kOneMinusEpsilon);
    return keep ? idx : e.alias;
}

// PDF_wi (src/math/warp.h:88-94) with the inf/nan guard of AreaLight::PDF_wi.
__device__ __forceinline__ float pdf_wi_from_area(float pdf_pos, f3 ng, f3 w_un) {
    float cos_t = fabsf(dot(ng, normalize(w_un)));
    float r = pdf_pos * length_sq(w_un) / cos_t;
    return (isinf(r) || isnan(r)) ? 0.0f : r;
}

template <int N>
__device__ __forceinline__ float light_pmf(const DeviceScene &s, uint32_t light) {
    if (s.ip.light_sampler == kLightSamplerPower) return s.light_pmf[light];
    return 1.0f / static_cast<float>(s.ip.light_count);
}

// SpotLight::falloff (spot.cpp:47-55): ((cos - cos_angle) / (cos_start -
// cos_angle))^4 with cos clamped to [cos_angle, cos_start]; a cone without a
// falloff range is a hard edge.
__device__ __forceinline__ float spot_falloff(const AreaLight &L, float cos_theta) {
    const float c = clampf(cos_theta, L.cos_angle, L.cos_start);
    const float range = L.cos_start - L.cos_angle;
    const float f = range > 0.0f ? (c - L.cos_angle) / range : (cos_theta >= L.cos_start ? 1.0f : 0.0f);
    const float f2 = f * f;
    return f2 * f2;
}

// Projector::Le (projector.cpp:112-125): the reference point in the light's
// frame, its squared distance there, and the colour slot at the projected uv
// when it falls inside the frustum (zero outside and behind).
template <int N>
__device__ __forceinline__ Spec<N> projector_L(const DeviceScene &s, const AreaLight &L, f3 p_ref,
                                               const Wavelengths<N> &wl) {
    const float *b = s.spd + L.alias_offset;
    const f3 p = {b[0] * p_ref.x + b[1] * p_ref.y + b[2] * p_ref.z + b[3],
                  b[4] * p_ref.x + b[5] * p_ref.y + b[6] * p_ref.z + b[7],
                  b[8] * p_ref.x + b[9] * p_ref.y + b[10] * p_ref.z + b[11]};
    const float d2 = length_sq(p);
    const float u = (p.x / p.z + b[12]) / (2.0f * b[12]);
    const float v = (p.y / p.z + b[13]) / (2.0f * b[13]);
    Spec<N> r = Spec<N>::fill(0.0f);
    if (!(p.z > 0.0f && u >= 0.0f && u <= 1.0f && v >= 0.0f && v <= 1.0f)) return r;
    const uint32_t tex = __float_as_uint(b[14]);
    if (tex == kInvalid) return emitter_spectrum<N>(L, wl) * (1.0f / d2);
    const f3 t = texture_rgb(s, tex, make2(u, v));
    const f3 rgb = {t.x * L.coef[0], t.y * L.coef[1], t.z * L.coef[2]};
    if (is_rgb(wl)) {
        const float ch[3] = {rgb.x, rgb.y, rgb.z};
#pragma unroll
        for (int i = 0; i < N; ++i) r.v[i] = ch[i < 3 ? i : 2] * L.scale / d2;
        return r;
    }
    float c[4];
    rgb2spec_unbound(s.rgb2spec, rgb, c);
#pragma unroll
    for (int i = 0; i < N; ++i)
        r.v[i] = sigmoid_poly(c[0], c[1], c[2], wl.lambda[i]) * c[3] * cie_spd(c_spec.d65, wl.lambda[i]) * L.scale / d2;
    return r;
}

// Radiance of a delta-position light at p_ref (PointLight::Le, point.cpp:36-41;
// SpotLight::Le, spot.cpp:47-67; Projector::Le).
template <int N>
__device__ __forceinline__ Spec<N> delta_light_L(const DeviceScene &s, const AreaLight &L, f3 p_ref,
                                                 const Wavelengths<N> &wl) {
    if (L.shape == kLightProjector) return projector_L<N>(s, L, p_ref, wl);
    const f3 lp = make3(L.pos[0], L.pos[1], L.pos[2]);
    const f3 w_un = p_ref - lp;
    float g = 1.0f / length_sq(w_un);
    if (L.shape == kLightSpot) g *= spot_falloff(L, dot(make3(L.dir[0], L.dir[1], L.dir[2]), normalize(w_un)));
    return emitter_spectrum<N>(L, wl) * g;
}

template <int N>
__device__ VS_OUTLINE LightSample<N> sample_light(const DeviceScene &s, const Interaction &it, float u_light,
                                                       f2 u, const Wavelengths<N> &wl) {
    LightSample<N> ls;
    uint32_t n = s.ip.light_count;
    uint32_t li;
    float pmf_light;
    if (s.ip.light_sampler == kLightSamplerPower) {
        li = alias_sample(s.light_alias, n, u_light, nullptr);
        pmf_light = s.light_pmf[li];
    } else {
        li = static_cast<uint32_t>(fminf(u_light * static_cast<float>(n), static_cast<float>(n) - 1.0f));
        pmf_light = 1.0f / static_cast<float>(n);
    }
    if (s.has_env && li == s.env_index) {
        // SphericalMap::sample_wi (spherical.cpp:180-186).
        env_sample<N>(s, it.pos, u, wl, ls.L, ls.pdf, ls.p_light);
        ls.pdf *= pmf_light;
        return ls;
    }
    const AreaLight &L = s.lights[li];
    if (L.shape != kLightArea) {
        // IPointLight::sample_wi (light.cpp:42-51) with PointLight::Le /
        // SpotLight::Le: colour * scale / distance^2, times the spot's
        // falloff.  A negative pdf marks the delta light (direct_lighting,
        // integrator.cpp:29-31: MIS weight 1, pdf = the light's pmf).
        ls.L = delta_light_L<N>(s, L, it.pos, wl);
        ls.pdf = -pmf_light;
        ls.p_light = make3(L.pos[0], L.pos[1], L.pos[2]);
        return ls;
    }
    float ux = u.x;
    uint32_t local = alias_sample(s.prim_alias + L.alias_offset, L.prim_count, u.x, &ux);
    float pmf_prim = s.prim_pmf[L.alias_offset + local];
    float su0 = sqrtf(ux);
    Hit h;
    h.prim_id = L.first_prim + local;
    h.u = 1.0f - su0;
    h.v = u.y * su0;
    // LightEvalContext: position, geometric normal and area of the sampled point.
    uint4 idx;
    float4 A[2], B[2], C[2];
    load_triangle(s, h.prim_id, idx, A, B, C);
    f3 p0 = ld3(A[0]), p1 = ld3(B[0]), p2 = ld3(C[0]);
    float w = 1.0f - h.u - h.v;
    f3 pos = p0 * w + p1 * h.u + p2 * h.v;
    f3 ng_un = cross(p0 - p2, p1 - p2);
    float area = 0.5f * length(ng_un);
    f3 ng = normalize(ng_un);
    float pdf_pos = (1.0f / area) * pmf_prim;
    f3 w_ref = it.pos - pos;
    bool front = dot(w_ref, ng) > 0.0f || L.two_sided;
    ls.L = front ? emitter_spectrum<N>(L, wl) : Spec<N>::fill(0.0f);
    ls.pdf = pdf_wi_from_area(pdf_pos, ng, w_ref) * pmf_light;
    f3 n_off = dot(ng, w_ref) > 0.0f ? ng : -ng;
    ls.p_light = offset_ray_origin(pos, n_off);
    return ls;
}

// LightSampler::evaluate_hit_wi (lightsampler.cpp:252-267) for a path that hit
// an emissive primitive; p_ref is the ray origin.
template <int N>
__device__ VS_OUTLINE void eval_hit_light(const DeviceScene &s, const Interaction &it, f3 p_ref,
                                               const Wavelengths<N> &wl, Spec<N> &L, float &pdf) {
    AreaLight light = s.lights[it.light];
    float pmf_prim = s.prim_pmf[light.alias_offset + (it.prim - light.first_prim)];
    float pdf_pos = (1.0f / it.prim_area) * pmf_prim;
    f3 w = p_ref - it.pos;
    bool front = dot(w, it.ng) > 0.0f || light.two_sided;
    L = front ? emitter_spectrum<N>(light, wl) : Spec<N>::fill(0.0f);
    pdf = pdf_wi_from_area(pdf_pos, it.ng, w) * light_pmf<N>(s, it.light);
}

// sample_linear / sample_tent (math/warp.h:132-145): the tent filter's offset.
__device__ __forceinline__ float sample_linear(float u, float a, float b) {
    float x = u * (a + b) / (a + sqrtf(lerpf(u, a * a, b * b)));
    x = fminf(x, kOneMinusEpsilon);
    return (u == 0.0f && a == 0.0f) ? 0.0f : x;
}
__device__ __forceinline__ float sample_tent(float u, float r) {
    return u < 0.5f ? -r * sample_linear((0.5f - u) * 2.0f, 1.0f, 0.0f) : r * sample_linear((u - 0.5f) * 2.0f, 1.0f, 0.0f);
}

__device__ __forceinline__ float sign_of(float v) { return v > 0.0f ? 1.0f : (v < 0.0f ? -1.0f : 0.0f); }

// FilterSampler::sample (fitted_curve.h:72-80): the tabulated filter's offset
// in [-1, 1]^2 (times the radius by the caller) and weight.
__device__ __forceinline__ f2 fitted_filter_sample(const DeviceScene &s, f2 u, float &weight) {
    const uint32_t n = kFilterTable;
    u = make2(u.x * 2.0f - 1.0f, u.y * 2.0f - 1.0f);
    const float *lut = s.filter_tab;
    const float *marginal_func = s.filter_tab + n * n;
    const float *cond_func = marginal_func + n;
    uint32_t iv, iu;
    const float fv = alias_continuous(s.filter_alias, n, fabsf(u.y), iv);
    const float pdf_v = s.filter_integral > 0.0f ? __ldg(&marginal_func[iv]) / s.filter_integral : 0.0f;
    const float fu = alias_continuous(s.filter_alias + n + static_cast<size_t>(iv) * n, n, fabsf(u.x), iu);
    const float integral_u = __ldg(&marginal_func[iv]);
    const float pdf_u = integral_u > 0.0f ? __ldg(&cond_func[iv * n + iu]) / integral_u : 0.0f;
    const float pdf = pdf_u * pdf_v;
    weight = __ldg(&lut[iv * n + iu]) / pdf;
    return make2(fu * sign_of(u.x), fv * sign_of(u.y));
}

// Sampler::sensor_sample (sampler.h:65-73) with the scene's filter (box.cpp,
// triangle.cpp, fitted_curve.h) and Sensor::generate_ray (sensor.cpp:44-56,
// 63-76; ThinLensCamera::generate_ray_in_local_space, thin_lens.cpp:36-43):
// raster -> screen -> camera -> world.  Draws 2 (filter) + 2 (lens) + 1
// (time) numbers.  Returns the filter weight the path's radiance is scaled by.
__device__ __forceinline__ float camera_ray(const DeviceScene &s, const Camera &cam, Sampler &smp, uint32_t px,
                                            uint32_t py, f2 &p_film, f3 &ro, f3 &rd) {
    f2 uf = smp.next2();
    float fx, fy, weight = 1.0f;
    if (cam.filter == kFilterBox) {
        fx = lerpf(uf.x, -cam.filter_rx, cam.filter_rx);
        fy = lerpf(uf.y, -cam.filter_ry, cam.filter_ry);
    } else if (cam.filter == kFilterTriangle) {
        fx = sample_tent(uf.x, cam.filter_rx);
        fy = sample_tent(uf.y, cam.filter_ry);
    } else {
        f2 q = fitted_filter_sample(s, uf, weight);
        fx = q.x * cam.filter_rx;
        fy = q.y * cam.filter_ry;
    }
    const f2 u_lens = smp.next2();
    (void)smp.next();
    float film_x = static_cast<float>(px) + 0.5f + fx;
    float film_y = static_cast<float>(py) + 0.5f + fy;
    p_film = {film_x, film_y};
    float sx = cam.screen_lo_x + film_x / static_cast<float>(cam.width) * cam.screen_span_x;
    float sy = cam.screen_hi_y - film_y / static_cast<float>(cam.height) * cam.screen_span_y;
    f3 dir_cam = normalize(make3(sx * cam.tan_half_fov, sy * cam.tan_half_fov, 1.0f));
    if (cam.thin_lens) {
        const f2 pl = square_to_disk(u_lens);
        const f3 o_lens = make3(pl.x * cam.lens_radius, pl.y * cam.lens_radius, 0.0f);
        const float ft = cam.focal_distance / dir_cam.z;
        const f3 p_focus = dir_cam * ft;
        const f3 d_lens = normalize(p_focus - o_lens);
        ro = xform_point(cam.c2w, o_lens);
        rd = normalize(xform_vector(cam.c2w, d_lens));
    } else {
        ro = xform_point(cam.c2w, make3(0.0f));
        rd = normalize(xform_vector(cam.c2w, dir_cam));
    }
    return weight;
}

// Mutable state of one camera path between bounces: the sampler, the hero
// wavelengths, the next ray with the pdf of the direction it was sampled
// with, the throughput, the radiance gathered so far, the accumulated
// relative-IOR factor of Russian roulette, the bounce index and the camera
// sample's filter weight.
template <int N>
struct PathState {
    Sampler smp;
    Wavelengths<N> wl;
    f3 ro, rd;
    Spec<N> throughput;
    f3 L;
    float scatter_pdf;
    float eta_scale;
    uint32_t bounce;
    float filter_w;  // the camera sample's filter weight (radiance scale at the end)
};

// Shadow ray of one bounce and the radiance it adds when unoccluded (linear
// sRGB, already weighted by the throughput and the MIS weight).
struct ShadowQuery {
    f3 o, d;
    float tmax;
    f3 c;
    bool valid;  // false: no contribution possible, no ray to trace
};

// One iteration of the bounce loop of IlluminationIntegrator::Li
// (integrator.cpp:134-283) after the closest-hit query: add the emission of
// the hit (or the environment on a miss) to ps.L, prepare the next-event
// estimate as a shadow query, sample the BSDF and set the next ray.  The caller
// traces `sq` and adds sq.c when it is unoccluded; a query whose contribution
// would be zero (no valid BSDF value or light pdf, or mis_mode 2) is not
// issued, which leaves the sum unchanged.  Returns false where the
// reference's loop breaks (miss, invalid BSDF sample, Russian roulette, zero
// throughput).  `first`, when non-null, receives the interaction of the first
// surface hit (the HitContext of the reference).
//
// kTraceShadow: trace the shadow ray in place, right after the light sample
// (the megakernel: nothing of the query stays live across the BSDF code), and
// add its contribution to ps.L; sq then stays invalid.  M: the material types
// compiled in (kAllMaterials, or one class for the material-sorted wavefront
// kernels, whose hits all have that type); M = 0 compiles the miss only.
//
// path_shade_acc generalises the gathering: every contribution (spectral,
// already weighted) goes through acc(ps, c) — RgbAcc adds its linear sRGB to
// ps.L, SpecAcc sums the spectrum — and emit = false skips the emission of
// the hit (a path suffix that starts at a vertex whose emission belongs to
// the prefix).  Deferred shadow queries carry linear sRGB, so a spectral
// accumulator needs kTraceShadow.
template <int N>
struct RgbAcc {
    __device__ __forceinline__ void operator()(PathState<N> &ps, const Spec<N> &c) const {
        ps.L += linear_srgb<N>(c, ps.wl);
    }
};
template <int N>
struct SpecAcc {
    Spec<N> *sum;
    __device__ __forceinline__ void operator()(PathState<N> &, const Spec<N> &c) const { *sum = *sum + c; }
};

// IlluminationIntegrator::evaluate_miss (integrator.cpp:111-132): the
// environment seen by a ray that left the scene, MIS-weighted against the
// pdf of the direction it was sampled with.
template <int N, class Acc>
__device__ __forceinline__ void miss_emission(const DeviceScene &s, PathState<N> &ps, const Acc &acc) {
    if (!s.has_env) return;
    const IntegratorParams &ip = s.ip;
    Spec<N> Le;
    float lpdf;
    env_eval<N>(s, normalize((ps.ro + ps.rd) - ps.ro), ps.wl, Le, lpdf);
    lpdf *= light_pmf<N>(s, s.env_index);
    float weight = ps.scatter_pdf / (ps.scatter_pdf + lpdf);
    if (ip.mis_mode == 2u) weight = 1.0f;
    else if (ip.mis_mode == 1u) weight = ps.bounce == 0 ? weight : 0.0f;
    acc(ps, Le * ps.throughput * weight);
}

// Emission of the surface a ray hit (integrator.cpp:192-203), MIS-weighted.
template <int N, class Acc>
__device__ __forceinline__ void hit_emission(const DeviceScene &s, PathState<N> &ps, const Interaction &it,
                                             const Acc &acc) {
    if (it.light == kInvalid) return;
    const IntegratorParams &ip = s.ip;
    Spec<N> Le;
    float lpdf;
    eval_hit_light<N>(s, it, ps.ro, ps.wl, Le, lpdf);
    float weight = ps.scatter_pdf / (ps.scatter_pdf + lpdf);
    if (ip.mis_mode == 2u) weight = 1.0f;
    else if (ip.mis_mode == 1u) weight = ps.bounce == 0 ? weight : 0.0f;
    acc(ps, Le * ps.throughput * weight);
}

template <int N, bool kTraceShadow, uint32_t M, class Acc>
__device__ __forceinline__ bool path_shade_acc(const DeviceScene &s, PathState<N> &ps, bool hit_any, const Hit &hit,
                                               Interaction *first, ShadowQuery &sq, const Acc &acc, bool emit) {
    const IntegratorParams &ip = s.ip;
    const uint32_t bounce = ps.bounce;
    sq.valid = false;
    if (!hit_any || M == 0u) {
        miss_emission<N>(s, ps, acc);
        return false;
    }
    Interaction it = surface_interaction(s, hit, ps.rd, true);
    if (first && bounce == 0) *first = it;
    if (emit) hit_emission<N>(s, ps, it, acc);
    // Light sample: 1 draw for the light, 2 for the surface point.
    float u_light = ps.smp.next();
    f2 u_surf = ps.smp.next2();
    LightSample<N> ls = sample_light<N>(s, it, u_light, u_surf, ps.wl);
    Ray sh = spawn_ray_to(it.pos, it.ng, ls.p_light);
    bool occluded = false;
    if (kTraceShadow) occluded = trace_any(s, precompute_ray(sh.o, sh.d), sh.tmax);
    // Material evaluation + BSDF sample (direct_lighting, integrator.cpp:20-44).
    Material mat = s.materials[it.mat];
    const typename ShadeBsdf<N, M>::type bsdf = ShadeBsdf<N, M>::make(s, mat, it.shading, it.ng, it.wo, it.uv, ps.wl);
    if (bsdf.dispersive) invalidate_secondary<N>(ps.wl);
    f3 wi_light = normalize(ls.p_light - it.pos);
    BsdfEval<N> se = bsdf.evaluate(it.wo, wi_light, nullptr);
    BsdfSample<N> bs = bsdf.sample(it.wo, ps.smp);
    const bool delta = ls.pdf < 0.0f;
    const float l_pdf = delta ? -ls.pdf : ls.pdf;
    float w_mis = delta ? 1.0f : ls.pdf / (ls.pdf + se.pdf);
    if (ip.mis_mode == 1u) w_mis = 1.0f;
    if (kTraceShadow) {
        Spec<N> Ld = Spec<N>::fill(0.0f);
        if (!occluded && se.valid() && l_pdf > 0.0f) Ld = ls.L * se.f * (w_mis / l_pdf);
        if (ip.mis_mode != 2u) acc(ps, ps.throughput * Ld);
    } else if (ip.mis_mode != 2u && se.valid() && l_pdf > 0.0f) {
        Spec<N> Ld = ls.L * se.f * (w_mis / l_pdf);
        sq.o = sh.o;
        sq.d = sh.d;
        sq.tmax = sh.tmax;
        sq.c = linear_srgb<N>(ps.throughput * Ld, ps.wl);
        sq.valid = true;
    }
    ps.eta_scale *= sqr(bs.eta);
    float lum = ps.throughput.max();
    if (!bs.eval.valid() || lum == 0.0f) return false;
    ps.throughput = ps.throughput * bs.eval.throughput();
    if (ps.eta_scale * lum < ip.rr_threshold && bounce >= ip.min_depth) {
        float q = fminf(0.95f, lum);
        float rr = ps.smp.next();
        if (q < rr) return false;
        ps.throughput = ps.throughput * (1.0f / q);
    }
    // A path whose throughput is exactly zero adds nothing from here on.
    if (ps.throughput.all_zero()) return false;
    ps.scatter_pdf = bs.eval.pdf;
    Ray nr = spawn_ray(it.pos, it.ng, bs.wi);
    ps.ro = nr.o;
    ps.rd = nr.d;
    return true;
}

template <int N, bool kTraceShadow, uint32_t M = kAllMaterials>
__device__ __forceinline__ bool path_shade(const DeviceScene &s, PathState<N> &ps, bool hit_any, const Hit &hit,
                                           Interaction *first, ShadowQuery &sq) {
    return path_shade_acc<N, kTraceShadow, M>(s, ps, hit_any, hit, first, sq, RgbAcc<N>{}, true);
}

// One iteration of the bounce loop: closest hit, shading, shadow ray.
template <int N>
__device__ __forceinline__ bool path_bounce(const DeviceScene &s, PathState<N> &ps, Interaction *first) {
    RayPre rp = precompute_ray(ps.ro, ps.rd);
    Hit hit;
    float t_hit;
    const bool hit_any = trace_closest(s, rp, 3.402823466e+38f, hit, t_hit);
    ShadowQuery sq;
    return path_shade<N, true>(s, ps, hit_any, hit, first, sq);
}

// The bounce loop of IlluminationIntegrator::Li (integrator.cpp:134-283) from
// ray (ro, rd) with the given scatter pdf and throughput.  Returns linear sRGB
// radiance; smp and wl carry the sampler position and the (possibly
// invalidated) wavelengths back to the caller.
template <int N>
__device__ __forceinline__ f3 path_li(const DeviceScene &s, Sampler &smp, Wavelengths<N> &wl, f3 ro, f3 rd,
                                      float scatter_pdf, Spec<N> throughput, uint32_t max_depth,
                                      Interaction *first) {
    PathState<N> ps;
    ps.smp = smp;
    ps.wl = wl;
    ps.ro = ro;
    ps.rd = rd;
    ps.throughput = throughput;
    ps.L = make3(0.0f);
    ps.scatter_pdf = scatter_pdf;
    ps.eta_scale = 1.0f;
    ps.filter_w = 1.0f;
    for (ps.bounce = 0; ps.bounce < max_depth; ++ps.bounce)
        if (!path_bounce<N>(s, ps, first)) break;
    smp = ps.smp;
    wl = ps.wl;
    return ps.L;
}

// Start of one camera path (PathTracingIntegrator kernel body, pt.cpp:53-72)
// through sensor `cam`: wavelengths from their own sampler stream
// (RenderEnv::initial, integrator.cpp:49-58), then the camera ray from the
// pixel's stream.
template <int N>
__device__ __forceinline__ void path_start(const DeviceScene &s, const Camera &cam, uint32_t px, uint32_t py,
                                           uint32_t frame, PathState<N> &ps) {
    const IntegratorParams &ip = s.ip;
    ps.smp.start(px, py, frame, 0xffffffffu, ip.sampler, ip.seed);
    ps.wl = ip.srgb ? rgb_wavelengths<N>() : sample_wavelengths<N>(ps.smp.next());
    ps.smp.start(px, py, frame, 0u, ip.sampler, ip.seed);
    f2 p_film;
    ps.filter_w = camera_ray(s, cam, ps.smp, px, py, p_film, ps.ro, ps.rd);
    ps.throughput = Spec<N>::fill(1.0f);
    ps.L = make3(0.0f);
    ps.scatter_pdf = 1e16f;
    ps.eta_scale = 1.0f;
    ps.bounce = 0;
}

// One camera path through sensor `cam`.  Returns linear sRGB radiance times
// the filter weight.
template <int N>
__device__ __forceinline__ f3 trace_path_cam(const DeviceScene &s, const Camera &cam, uint32_t px, uint32_t py,
                                             uint32_t frame) {
    PathState<N> ps;
    path_start<N>(s, cam, px, py, frame, ps);
    const uint32_t max_depth = s.ip.max_depth;
    for (; ps.bounce < max_depth; ++ps.bounce)
        if (!path_bounce<N>(s, ps, nullptr)) break;
    return ps.L * ps.filter_w;
}

template <int N>
__device__ f3 trace_path(const DeviceScene &s, uint32_t px, uint32_t py, uint32_t frame) {
    return trace_path_cam<N>(s, s.cam, px, py, frame);
}

}  // namespace vs

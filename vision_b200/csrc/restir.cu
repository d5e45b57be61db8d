// sm_100a kernels of the real-time ReSTIR frame (RealTimeIntegrator::render,
// src/render_core/integrators/rt.cpp:144-160):
//   k_rt_reset        - default surfaces and reservoirs (ReSTIRDI/GI::prepare)
//   k_di_primary .. k_di_temporal
//                     - the direct pass (direct.cpp:519-557) in six stages:
//                       primary hit with its near-specular chain and motion
//                       vector, RIS over M_light light candidates, the BSDF
//                       candidate's ray, its evaluation, visibility, temporal
//                       reuse; k_di_candidates does it in one kernel (used when
//                       M_bsdf > 1)
//   k_di_sp_*         - spatial reuse and shading (direct.cpp:638-674) in three
//                       stages (combine, shading rays, shading)
//   k_gi_wf_*         - one path suffix per pixel from the direct pass's BSDF
//                       direction (indirect.cpp:83-111) as wavefront passes;
//                       k_gi_initial does it in one kernel (grid and
//                       persistent schedules)
//   k_gi_temporal     - GI temporal reuse (indirect.cpp:205-236)
//   k_gi_sp_*         - GI spatial reuse and shading (indirect.cpp:238-332) in
//                       three stages (neighbours, visibility rays, combine)
//   k_rt_combine      - direct * di + indirect * ii into the film (rt.cpp:118-126)
// One thread per pixel, 16 x 8 pixel tiles.  Spectral work runs on 3 hero
// wavelengths: the reference's ReSTIR code moves spectra through float3
// (SampledSpectrum::vec3, SampledSpectrum(Float3)), which is only defined for
// three channels.
#include "vs_wavefront.cuh"
#include "vs_launch.h"
#include "vs_restir.h"

#include <algorithm>

// The material types compiled into this copy of the ReSTIR kernels and the
// namespace that holds them: restir.cu builds the general copy (every
// material); restir_diffuse.cu includes this file again for scenes made of
// diffuse surfaces and emitters only, whose candidate loops then carry no
// code for the other materials (the reference's DSL likewise compiles a
// scene's kernels for the materials it has).
#ifndef VS_RT_MATERIALS
#define VS_RT_MATERIALS kAllMaterials
#define VS_RT_NS rt_all
#endif

namespace vs {
namespace VS_RT_NS {

namespace {

constexpr int RN = 3;
using RSpec = Spec<RN>;
using RWl = Wavelengths<RN>;

constexpr uint32_t kFlagNearSpec = 1u << 6;  // BxDFFlag::NearSpec (sample.h:31)
constexpr float kAlphaThreshold = 0.022f;    // alpha_threshold_ of metal.cpp:46, glass.cpp:178

__device__ __forceinline__ f3 vec3(const RSpec &s) { return {s.v[0], s.v[1], s.v[2]}; }
__device__ __forceinline__ RSpec spec3(f3 v) {
    RSpec r;
    r.v[0] = v.x;
    r.v[1] = v.y;
    r.v[2] = v.z;
    return r;
}
// ocarina::luminance: Rec.709 luma of a float3.
__device__ __forceinline__ float lum3(f3 v) { return linear_srgb_to_y(v); }
__device__ __forceinline__ bool bad(float x) { return isnan(x) || isinf(x); }
__device__ __forceinline__ f3 zero_if_nan_inf(f3 v) {
    return {bad(v.x) ? 0.0f : v.x, bad(v.y) ? 0.0f : v.y, bad(v.z) ? 0.0f : v.z};
}
__device__ __forceinline__ f3 ld3p(const float *p) { return {p[0], p[1], p[2]}; }
__device__ __forceinline__ void st3(float *p, f3 v) {
    p[0] = v.x;
    p[1] = v.y;
    p[2] = v.z;
}

// DIReservoir::safe_weight / cal_weight (reservoir.h:73-86).
__device__ __forceinline__ float cal_weight(float mis, float p_hat, float W) { return mis * p_hat * W; }
__device__ __forceinline__ float safe_weight(float mis, float p_hat, float W) {
    float r = cal_weight(mis, p_hat, W);
    return isnan(r) ? 0.0f : r;
}
// balance_heuristic with integer counts (warp.h:148-154,186-199).
__device__ __forceinline__ float mis_n(int nf, float f, int ng, float g) {
    return (static_cast<float>(nf) * f) / (static_cast<float>(nf) * f + static_cast<float>(ng) * g);
}

// DIReservoir update / truncation / process_occluded / cal_W (reservoir.h:89-115).
__device__ __forceinline__ bool di_update(DiReservoir &r, float u, const DiReservoir &v, float weight,
                                          float new_C = 1.0f) {
    r.weight_sum += static_cast<double>(weight);
    r.C += new_C;
    bool take = static_cast<double>(u) * r.weight_sum < static_cast<double>(weight);
    if (take) {
        r.light_index = v.light_index;
        r.prim_id = v.prim_id;
        r.bary_u = v.bary_u;
        r.bary_v = v.bary_v;
        r.age = v.age;
        r.p_hat = v.p_hat;
        r.pos[0] = v.pos[0];
        r.pos[1] = v.pos[1];
        r.pos[2] = v.pos[2];
    }
    return take;
}
__device__ __forceinline__ void di_update_W(DiReservoir &r, float p_hat) {
    r.W = p_hat == 0.0f ? 0.0f : static_cast<float>(r.weight_sum / static_cast<double>(p_hat));
}
__device__ __forceinline__ DiReservoir di_empty() {
    DiReservoir r{};
    r.light_index = kInvalid;
    return r;
}

// GIReservoir update / truncation / cal_W (reservoir.h:195-221).
__device__ __forceinline__ void gi_copy_sample(GiReservoir &r, const GiReservoir &v) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        r.sp_pos[i] = v.sp_pos[i];
        r.sp_ng[i] = v.sp_ng[i];
        r.Lo[i] = v.Lo[i];
    }
    r.age = v.age;
}
__device__ __forceinline__ bool gi_update(GiReservoir &r, float u, const GiReservoir &v, float weight,
                                          float new_C = 1.0f) {
    r.weight_sum += static_cast<double>(weight);
    r.C += new_C;
    bool take = static_cast<double>(u) * r.weight_sum < static_cast<double>(weight) || r.weight_sum == 0.0;
    if (take) gi_copy_sample(r, v);
    return take;
}
__device__ __forceinline__ void gi_truncation(GiReservoir &r, float limit) {
    float factor = limit / r.C;
    r.C = fminf(limit, r.C);
    if (factor < 1.0f) r.weight_sum = r.weight_sum * static_cast<double>(factor);
}
__device__ __forceinline__ void gi_update_W(GiReservoir &r, float p_hat) {
    r.W = p_hat == 0.0f ? 0.0f
                        : static_cast<float>(r.weight_sum / (static_cast<double>(p_hat) * static_cast<double>(r.C)));
}

__device__ __forceinline__ uint32_t pixel_index(const RtParams &p, uint32_t x, uint32_t y) { return y * p.width + x; }

// Float -> integer conversions of the reference's make_uint2 / make_int2 on
// float vectors: round toward zero, saturating (NaN -> 0).
__device__ __forceinline__ uint32_t f2u(float x) { return __float2uint_rz(x); }
__device__ __forceinline__ int f2i(float x) { return __float2int_rz(x); }

__device__ __forceinline__ f2 square_to_disk2(f2 u) {
    float r = sqrtf(u.x);
    float theta = 2.0f * kPi * u.y;
    return {r * cosf(theta), r * sinf(theta)};
}

// Sensor::prev_raster_coord (sensor.cpp:105-110) in closed form: the inverse
// of the raster -> camera mapping of camera_ray().
__device__ __forceinline__ f2 prev_raster(const RtParams &p, f3 world) {
    f3 c = xform_point(p.prev_w2c, world);
    float a = c.x / c.z, b = c.y / c.z;
    const Camera &k = p.prev_cam;
    float sx = a / k.tan_half_fov, sy = b / k.tan_half_fov;
    return {(sx - k.screen_lo_x) / k.screen_span_x * static_cast<float>(k.width),
            (k.screen_hi_y - sy) / k.screen_span_y * static_cast<float>(k.height)};
}

// is_valid_neighbor (common.h:72-80).
__device__ __forceinline__ bool valid_neighbor(const RtSurface &c, const RtSurface &o, float dot_thr, float depth_thr,
                                               float diff_thr) {
    bool c0 = fabsf(c.nx * o.nx + c.ny * o.ny + c.nz * o.nz) > dot_thr;
    bool c1 = (fabsf(c.depth - o.depth) / c.depth) < depth_thr;
    bool c2 = fabsf(c.diffuse - o.diffuse) / c.diffuse < diff_thr;
    return c0 && c1 && c2 && c.hit.inst_id != kInvalid && o.hit.inst_id != kInvalid;
}

// Geometry::compute_surface_interaction(hit, view_pos) (geometry.h:59-63).
__device__ __forceinline__ Interaction it_at(const DeviceScene &s, const Hit &h, f3 view_pos) {
    Interaction it = surface_interaction(s, h, make3(0.0f, 0.0f, 1.0f), true);
    it.wo = normalize(view_pos - it.pos);
    return it;
}

// MaterialEvaluator creation plus SampledWavelengths::check_dispersive.
__device__ __forceinline__ Bsdf<RN, VS_RT_MATERIALS> bsdf_at(const DeviceScene &s, const Interaction &it, RWl &wl) {
    Material m = s.materials[it.mat];
    Bsdf<RN, VS_RT_MATERIALS> b = make_bsdf<RN, VS_RT_MATERIALS>(s, m, it.shading, it.ng, it.wo, it.uv, wl);
    if (b.dispersive) invalidate_secondary<RN>(wl);
    return b;
}

// Lobe-set flag and diffuse factor of a material (SurfaceData flag / pos_diff.w):
// metal and glass carry NearSpec below alpha 0.022 and Glossy above
// (metal.cpp:146-148, glass.cpp:250-252); their diffuse factors are
// sqrt(sqrt(ax * ay)) (MicrofacetLobe, lobe.cpp:212-214) and sqrt(ax)
// (DielectricLobe, lobe.cpp:427-429); diffuse, black body and principled
// lobe sets keep the default factor 1 (lobe.h:84).
__device__ __forceinline__ void classify(const Material &m, uint32_t &flag, float &diffuse) {
    diffuse = 1.0f;
    if (m.type == kMatMetal) {
        flag = fminf(m.p[0], m.p[1]) < kAlphaThreshold ? kFlagNearSpec : kFlagGlossy;
        diffuse = sqrtf(sqrtf(m.p[0] * m.p[1]));
    } else if (m.type == kMatGlass) {
        flag = fminf(m.p[0], m.p[1]) < kAlphaThreshold ? kFlagNearSpec : kFlagGlossy;
        diffuse = sqrtf(m.p[0]);
    } else if (m.type == kMatSubstrate && (m.flags & kMatFlagPlastic)) {
        // PlasticLobe: NearSpec below alpha 0.022 (plastic.cpp:120-121), the
        // microfacet lobe's diffuse factor.
        flag = fminf(m.p[0], m.p[1]) < kAlphaThreshold ? kFlagNearSpec : kFlagGlossy;
        diffuse = sqrtf(sqrtf(m.p[0] * m.p[1]));
    } else if (m.type == kMatSubstrate) {
        // SubstrateLobe: always Glossy (substrate.cpp:147), diffuse factor
        // sqrt of the microfacet lobe's (substrate.cpp:74-80).
        flag = kFlagGlossy;
        diffuse = sqrtf(sqrtf(sqrtf(m.p[0] * m.p[1])));
    } else if (m.type == kMatDiffuse) {
        flag = kFlagDiffRefl;
    } else if (m.type == kMatBlackBody) {
        flag = kFlagDiffuse;
    } else {
        flag = kFlagGlossyRefl | kFlagDiffRefl;
    }
}

// MaterialEvaluator::sample_delta (material.cpp:154-160) of a near-specular
// conductor (MicrofacetLobe::sample_delta_local, lobe.cpp:223-230: mirror
// direction, uncompensated BxDF) or dielectric (DielectricLobe::sample_delta_local,
// lobe.cpp:404-425: one draw picks mirror reflection or refraction).
__device__ VS_OUTLINE BsdfSample<RN> sample_delta(const Bsdf<RN, VS_RT_MATERIALS> &b, f3 wo_w, Sampler &smp) {
    BsdfSample<RN> bs;
    bs.eta = 1.0f;
    f3 wo = b.frame.to_local(wo_w);
    f3 wi;
    if (b.type == kMatMetal || b.type == kMatSubstrate) {
        // Metal, mirror, and a near-specular plastic: the microfacet
        // reflection BxDF of the lobe (kr 1 for plastic).
        wi = make3(-wo.x, -wo.y, wo.z);
        MfLobe<RN> l = b.mf[0];
        l.compensate = false;
        l.eval_local(wo, wi, b.luts, bs.eval.f, bs.eval.pdf);
        bs.eval.flags = kFlagGlossyRefl;
    } else {
        const DielLobe<RN> &d = b.dl;
        RSpec F = d.F(fabsf(wo.z));
        float uc = smp.next();
        if (uc < d.refl_prob(F)) {
            wi = make3(-wo.x, -wo.y, wo.z);
        } else {
            f3 n = face_forward(make3(0.0f, 0.0f, 1.0f), wo);
            if (!refract_dir(wo, n, d.eta.v[0], wi)) wi = make3(0.0f, 0.0f, 0.0f);
        }
        d.eval_local(wo, wi, b.luts, bs.eval.f, bs.eval.pdf, bs.eval.flags, bs.eta);
    }
    bs.eval.f = bs.eval.f * fabsf(wi.z);
    bs.wi = b.frame.to_world(wi);
    return bs;
}

// LightEvalContext of a point on an area light (Geometry::compute_light_eval_context,
// geometry.cpp:226-236): position, geometric normal and the primitive's area.
struct LightPoint {
    f3 pos;
    f3 ng;
    float area;
};
__device__ __forceinline__ LightPoint light_point(const DeviceScene &s, uint32_t prim, float bu, float bv) {
    uint4 idx;
    float4 A[2], B[2], C[2];
    load_triangle(s, prim, idx, A, B, C);
    f3 p0 = ld3(A[0]), p1 = ld3(B[0]), p2 = ld3(C[0]);
    float w = 1.0f - bu - bv;
    LightPoint lp;
    lp.pos = p0 * w + p1 * bu + p2 * bv;
    f3 ng_un = cross(p0 - p2, p1 - p2);
    lp.area = 0.5f * length(ng_un);
    lp.ng = normalize(ng_un);
    return lp;
}

// AreaLight::L for a point seen from p_ref (area.cpp:91-101).
__device__ __forceinline__ RSpec area_Le(const AreaLight &L, const LightPoint &lp, f3 p_ref, const RWl &wl) {
    bool front = dot(p_ref - lp.pos, lp.ng) > 0.0f || L.two_sided;
    return front ? emitter_spectrum<RN>(L, wl) : RSpec::fill(0.0f);
}

// Light::G (light.h:126-129).
__device__ __forceinline__ float light_G(f3 p_ref, const LightPoint &lp) {
    f3 w = p_ref - lp.pos;
    return dot(normalize(w), lp.ng) / length_sq(w);
}

__device__ __forceinline__ float light_select_pmf(const DeviceScene &s, uint32_t light) {
    return s.ip.light_sampler == kLightSamplerPower ? s.light_pmf[light]
                                                    : 1.0f / static_cast<float>(s.ip.light_count);
}

// LightSampler::evaluate_point (lightsampler.cpp:230-240) of a stored light
// sample, multiplied by the light's selection pmf:
//  * area light (AreaLight::evaluate_point, area.cpp:157-167): L = Le * G, pdf
//    in area measure = PDF_pos * PMF(prim), and the robust light position;
//  * point or spot light (IPointLight::evaluate_point, light.h:237-246): L =
//    Le at p_ref, pdf = -1 (the delta marker), the light's position;
//  * environment (SphericalMap::evaluate_point, spherical.cpp:134-141): the
//    map coordinates in (bary_u, bary_v) give the direction, L and the
//    solid-angle pdf; the point lies world_diameter along the direction.
// lp carries the LightEvalContext (compute_light_eval_context) that
// Light::PDF_point reads: the point and its normal.
enum : uint32_t { kPointArea = 0u, kPointDelta = 1u, kPointEnv = 2u };
struct PointEval {
    RSpec L;
    float pdf;
    f3 p_light;
    LightPoint lp;
    uint32_t kind;
};
__device__ __forceinline__ PointEval eval_light_point(const DeviceScene &s, f3 p_ref, uint32_t light, uint32_t prim,
                                                      float bu, float bv, const RWl &wl) {
    PointEval e;
    const float pmf = light_select_pmf(s, light);
    if (s.has_env && light == s.env_index) {
        f3 wd;
        env_eval_uv<RN>(s, bu, bv, wl, e.L, e.pdf, wd);
        e.pdf *= pmf;
        e.p_light = p_ref + wd * s.env.world_diameter;
        e.lp.pos = e.p_light;
        e.lp.ng = -wd;
        e.lp.area = 0.0f;
        e.kind = kPointEnv;
        return e;
    }
    AreaLight L = s.lights[light];
    if (L.shape != kLightArea) {
        const f3 lpos = make3(L.pos[0], L.pos[1], L.pos[2]);
        e.L = delta_light_L<RN>(s, L, p_ref, wl);
        e.pdf = -1.0f * pmf;
        e.p_light = lpos;
        e.lp.pos = lpos;
        e.lp.ng = normalize(p_ref - lpos);
        e.lp.area = 0.0f;
        e.kind = kPointDelta;
        return e;
    }
    e.lp = light_point(s, L.first_prim + prim, bu, bv);
    e.L = area_Le(L, e.lp, p_ref, wl) * light_G(p_ref, e.lp);
    float pmf_prim = s.prim_pmf[L.alias_offset + prim];
    e.pdf = (1.0f / e.lp.area) * pmf_prim * pmf;
    f3 w = p_ref - e.lp.pos;
    e.p_light = offset_ray_origin(e.lp.pos, dot(e.lp.ng, w) > 0.0f ? e.lp.ng : -e.lp.ng);
    e.kind = kPointArea;
    return e;
}

// vision::PDF_point (warp.h:101-105) with Light::PDF_point's inf guard (light.h:141-146).
__device__ __forceinline__ float pdf_point(float pdf_wi, f3 ng, f3 w_un) {
    float cos_t = fabsf(dot(ng, normalize(w_un)));
    float r = pdf_wi * cos_t / length_sq(w_un);
    return isinf(r) ? 0.0f : r;
}

// ReSTIRDI::Li evaluated for a stored light sample (direct.cpp:116-158) and
// its p_hat = luminance(f.vec3()).  Optionally returns the BSDF pdf of the
// point in area measure and the evaluated light sample.
__device__ VS_OUTLINE float di_p_hat(const DeviceScene &s, const Interaction &it, const Bsdf<RN, VS_RT_MATERIALS> &bsdf,
                                     const DiReservoir &smp, const RWl &wl, float *bsdf_pdf_point, PointEval *out,
                                     RSpec *f_out) {
    PointEval e;
    e.L = RSpec::fill(0.0f);
    e.pdf = 0.0f;
    e.p_light = make3(0.0f);
    e.lp.pos = make3(0.0f);
    e.lp.ng = make3(0.0f);
    e.lp.area = 0.0f;
    e.kind = kPointArea;
    bool valid = smp.light_index != kInvalid;
    if (valid) e = eval_light_point(s, it.pos, smp.light_index, smp.prim_id, smp.bary_u, smp.bary_v, wl);
    f3 wi = normalize(e.p_light - it.pos);
    BsdfEval<RN> ev = bsdf.evaluate(it.wo, wi, nullptr);
    RSpec f = ev.f * e.L;
    // LightSampler::PDF_point: the environment keeps the solid-angle pdf
    // (spherical.cpp:143-146); area and delta lights convert it to area
    // measure at their LightEvalContext (light.h:141-146).
    if (bsdf_pdf_point)
        *bsdf_pdf_point = !valid ? 0.0f : e.kind == kPointEnv ? ev.pdf : pdf_point(ev.pdf, e.lp.ng, it.pos - e.lp.pos);
    if (out) *out = e;
    if (f_out) *f_out = f;
    return lum3(vec3(f));
}

// compute_p_hat(it, nullptr, sample): a fresh evaluator at `it`.
__device__ __forceinline__ float di_p_hat_at(const DeviceScene &s, const Interaction &it, const DiReservoir &smp,
                                             RWl &wl) {
    Bsdf<RN, VS_RT_MATERIALS> b = bsdf_at(s, it, wl);
    return di_p_hat(s, it, b, smp, wl, nullptr, nullptr, nullptr);
}

__device__ __forceinline__ bool occluded_to(const DeviceScene &s, const Interaction &it, f3 p) {
    Ray sh = spawn_ray_to(it.pos, it.ng, p);
    return trace_any(s, precompute_ray(sh.o, sh.d), sh.tmax);
}

// ReSTIRDI::compute_hit (direct.cpp:353-400): primary hit and its chain of
// near-specular vertices (at most max_recursion surfaces).
struct PrimaryHit {
    RtSurface surf;
    RtSurfaceExt ext;
    Interaction it;
    f3 last_d;  // direction of the ray that found `it`
    bool hit;
};
__device__ VS_OUTLINE PrimaryHit compute_hit(const DeviceScene &s, const RtParams &p, Sampler &smp, RWl &wl,
                                             f3 cam_o, f3 cam_d) {
    PrimaryHit r;
    r.surf = RtSurface{};
    r.surf.hit.inst_id = kInvalid;
    r.surf.hit.prim_id = kInvalid;
    r.surf.flag = kFlagUnset;
    r.ext = RtSurfaceExt{1.0f, 1.0f, 1.0f, cam_o.x, cam_o.y, cam_o.z, 0.0f, 0u};
    f3 ro = cam_o, rd = cam_d;
    uint32_t counter = 0;
    for (;;) {
        Hit h;
        float t;
        r.hit = trace_closest(s, precompute_ray(ro, rd), 3.402823466e+38f, h, t);
        if (!r.hit) {
            r.surf.hit.inst_id = kInvalid;
            r.surf.hit.prim_id = kInvalid;
            r.surf.hit.u = r.surf.hit.v = 0.0f;
            break;
        }
        r.surf.hit = h;
        r.it = surface_interaction(s, h, rd, true);
        r.last_d = rd;
        r.ext.t_max += length(r.it.pos - ro) / length(rd);
        f3 v_pos = cam_o + cam_d * r.ext.t_max;
        Material m = s.materials[r.it.mat];
        uint32_t flag;
        float diff;
        classify(m, flag, diff);
        r.surf.flag = flag;
        r.surf.diffuse = diff;
        bool near_spec = flag == kFlagNearSpec;
        f3 w = make3(0.0f);
        if (near_spec) {
            Bsdf<RN, VS_RT_MATERIALS> b = make_bsdf<RN, VS_RT_MATERIALS>(s, m, r.it.shading, r.it.ng, r.it.wo, r.it.uv, wl);
            BsdfSample<RN> bs = sample_delta(b, r.it.wo, smp);
            w = bs.wi;
            RSpec tp = bs.eval.throughput();
            r.ext.tx *= tp.v[0];
            r.ext.ty *= tp.v[1];
            r.ext.tz *= tp.v[2];
        }
        if (counter == 0) {
            f3 c = xform_point(p.w2c, v_pos);
            r.surf.depth = c.z;
            r.surf.nx = r.it.shading.z.x;
            r.surf.ny = r.it.shading.z.y;
            r.surf.nz = r.it.shading.z.z;
            r.surf.px = r.it.pos.x;
            r.surf.py = r.it.pos.y;
            r.surf.pz = r.it.pos.z;
        }
        counter += 1;
        if (counter >= p.max_recursion) break;
        if (!near_spec) break;
        r.ext.vx = r.it.pos.x;
        r.ext.vy = r.it.pos.y;
        r.ext.vz = r.it.pos.z;
        Ray nr = spawn_ray(r.it.pos, r.it.ng, w);
        ro = nr.o;
        rd = nr.d;
        r.surf.is_replaced = 1u;
    }
    return r;
}

// Alias sampling with the remapped remainder (alias.h:124-146).
__device__ __forceinline__ uint32_t select_light(const DeviceScene &s, float u) {
    uint32_t n = s.ip.light_count;
    if (s.ip.light_sampler == kLightSamplerPower) return alias_sample(s.light_alias, n, u, nullptr);
    return static_cast<uint32_t>(fminf(u * static_cast<float>(n), static_cast<float>(n) - 1.0f));
}

// ReSTIRDI::RIS (direct.cpp:161-233).
__device__ __forceinline__ DiReservoir di_ris_lights(const DeviceScene &s, const RtParams &p, const Interaction &it,
                                                     Sampler &smp, RWl &wl, float lum_tp,
                                                     const Bsdf<RN, VS_RT_MATERIALS> &bsdf) {
    DiReservoir ret = di_empty();
    float Ml = static_cast<float>(p.M_light), Mb = static_cast<float>(p.M_bsdf);
    // LightSampler::sample_only (lightsampler.cpp:218-228): one light candidate
    // from its three draws, with its target pdf and RIS weight.  The
    // light-surface point is AreaLight::sample_only's primitive and
    // barycentrics (area.cpp:134-140), the environment's map coordinates
    // (spherical.cpp:127-132), or Light::sample_only's raw pair for a point or
    // spot light (light.h:177-182).  A delta light's negative pdf selects the
    // MIS weight 1 / M_light (direct.cpp:180-186).
    auto candidate = [&](float u_sel, f2 u, DiReservoir &cand, float &weight) {
        cand = di_empty();
        uint32_t li = select_light(s, u_sel);
        cand.light_index = li;
        cand.prim_id = 0u;
        if (s.has_env && li == s.env_index) {
            const f2 uv = env_sample_uv(s, u);
            cand.bary_u = uv.x;
            cand.bary_v = uv.y;
        } else {
            AreaLight L = s.lights[li];
            if (L.shape == kLightArea) {
                float ux = u.x;
                uint32_t local = alias_sample(s.prim_alias + L.alias_offset, L.prim_count, u.x, &ux);
                float su0 = sqrtf(ux);
                cand.prim_id = local;
                cand.bary_u = 1.0f - su0;
                cand.bary_v = u.y * su0;
            } else {
                cand.bary_u = u.x;
                cand.bary_v = u.y;
            }
        }
        PointEval ls;
        float bsdf_pdf_point = 0.0f;
        cand.p_hat = di_p_hat(s, it, bsdf, cand, wl, &bsdf_pdf_point, &ls, nullptr);
        st3(cand.pos, ls.p_light);
        const bool delta = ls.pdf < 0.0f;
        const float light_pdf = delta ? -ls.pdf : ls.pdf;
        const float mis = delta ? 1.0f / Ml : light_pdf / (Ml * light_pdf + Mb * bsdf_pdf_point);
        weight = safe_weight(mis, cand.p_hat, 1.0f / light_pdf) * lum_tp;
    };
    // Candidates in pairs: the draws of a pair are taken in the reference's
    // order (selection, surface point, reservoir update of the first, then
    // of the second) before either candidate is evaluated, so the two
    // candidates' dependent fetches (light table, primitive table, vertices)
    // are in flight together; the reservoir sees them in the same order.
    uint32_t i = 0;
    for (; i + 1 < p.M_light; i += 2) {
        const float s0 = smp.next();
        const f2 u0 = smp.next2();
        const float r0 = smp.next();
        const float s1 = smp.next();
        const f2 u1 = smp.next2();
        const float r1 = smp.next();
        DiReservoir c0, c1;
        float w0, w1;
        candidate(s0, u0, c0, w0);
        candidate(s1, u1, c1, w1);
        di_update(ret, r0, c0, w0);
        di_update(ret, r1, c1, w1);
    }
    if (i < p.M_light) {
        const float s0 = smp.next();
        const f2 u0 = smp.next2();
        DiReservoir c0;
        float w0;
        candidate(s0, u0, c0, w0);
        di_update(ret, smp.next(), c0, w0);
    }
    return ret;
}

// The BSDF candidate of ReSTIRDI::Li (direct.cpp:39-114), part one: the BSDF
// sample (recorded as the pixel's HitBSDF) and the ray that looks for an
// emitter along it.
__device__ __forceinline__ Ray di_bsdf_ray(const Interaction &it, const Bsdf<RN, VS_RT_MATERIALS> &bsdf,
                                           Sampler &smp, RtHitBsdf &hb) {
    BsdfSample<RN> bs = bsdf.sample(it.wo, smp);
    Ray ray = spawn_ray(it.pos, it.ng, bs.wi);
    hb.wx = bs.wi.x;
    hb.wy = bs.wi.y;
    hb.wz = bs.wi.z;
    hb.fx = bs.eval.f.v[0];
    hb.fy = bs.eval.f.v[1];
    hb.fz = bs.eval.f.v[2];
    hb.pdf = bs.eval.pdf;
    return ray;
}

// Part two: the candidate from what the ray hit (an emitter or nothing) and
// its RIS weight.
__device__ __forceinline__ void di_bsdf_candidate(const DeviceScene &s, const RtParams &p, const Interaction &it,
                                                  const RWl &wl, const RtHitBsdf &hb, bool hit, const Hit &h,
                                                  f3 ray_d, float lum_tp, DiReservoir &cand, float &weight) {
    const float Ml = static_cast<float>(p.M_light), Mb = static_cast<float>(p.M_bsdf);
    cand = di_empty();
    float pdf = hb.pdf;
    float eval_pdf = hb.pdf;
    RSpec eval_f;
    eval_f.v[0] = hb.fx;
    eval_f.v[1] = hb.fy;
    eval_f.v[2] = hb.fz;
    float light_pdf_point = 0.0f;
    RSpec f = RSpec::fill(0.0f);
    if (hit) {
        Interaction nit = surface_interaction(s, h, ray_d, false);
        if (nit.light != kInvalid) {
            // LightSampler::evaluate_hit_point (lightsampler.cpp:269-300).
            AreaLight L = s.lights[nit.light];
            LightPoint lp{nit.pos, nit.ng, nit.prim_area};
            RSpec Le = area_Le(L, lp, it.pos, wl) * light_G(it.pos, lp);
            float le_pdf = pdf_point(pdf, nit.ng, it.pos - nit.pos);
            uint32_t local = nit.prim - L.first_prim;
            light_pdf_point = (1.0f / nit.prim_area) * s.prim_pmf[L.alias_offset + local] *
                              light_select_pmf(s, nit.light);
            cand.light_index = nit.light;
            cand.prim_id = local;
            cand.bary_u = h.u;
            cand.bary_v = h.v;
            f3 w = it.pos - nit.pos;
            st3(cand.pos, offset_ray_origin(nit.pos, dot(nit.ng, w) > 0.0f ? nit.ng : -nit.ng));
            eval_pdf = le_pdf;
            f = eval_f * Le;
        }
    } else if (s.has_env) {
        // LightSampler::evaluate_miss_point (lightsampler.cpp:315-327): the
        // environment along the BSDF direction; the candidate keeps the
        // BSDF's solid-angle pdf and stores the direction's map coordinates
        // and the point world_diameter along it.
        const f3 wd = make3(hb.wx, hb.wy, hb.wz);
        const f3 pl = it.pos + wd * s.env.world_diameter;
        RSpec Le;
        float env_pdf;
        env_eval<RN>(s, normalize(pl - it.pos), wl, Le, env_pdf);
        light_pdf_point = env_pdf * light_select_pmf(s, s.env_index);
        const f2 uv = env_dir_uv(s, wd);
        cand.light_index = s.env_index;
        cand.prim_id = 0u;
        cand.bary_u = uv.x;
        cand.bary_v = uv.y;
        st3(cand.pos, pl);
        f = eval_f * Le;
    }
    cand.p_hat = lum3(vec3(f));
    float bp = eval_pdf;
    weight = safe_weight(bp / (Ml * light_pdf_point + Mb * bp), cand.p_hat, 1.0f / bp) * lum_tp;
}

// ReSTIRDI::RIS (direct.cpp:161-233): M_light light candidates, then M_bsdf
// BSDF candidates, each found by tracing its ray.
__device__ VS_OUTLINE DiReservoir di_ris(const DeviceScene &s, const RtParams &p, const Interaction &it,
                                         Sampler &smp, RWl &wl, f3 throughput, RtHitBsdf &hb) {
    Bsdf<RN, VS_RT_MATERIALS> bsdf = bsdf_at(s, it, wl);
    float lum_tp = lum3(throughput);
    DiReservoir ret = di_ris_lights(s, p, it, smp, wl, lum_tp, bsdf);
    for (uint32_t i = 0; i < p.M_bsdf; ++i) {
        Ray ray = di_bsdf_ray(it, bsdf, smp, hb);
        Hit h;
        float t;
        bool hit = trace_closest(s, precompute_ray(ray.o, ray.d), ray.tmax, h, t);
        DiReservoir cand;
        float weight;
        di_bsdf_candidate(s, p, it, wl, hb, hit, h, ray.d, lum_tp, cand, weight);
        di_update(ret, smp.next(), cand, weight);
    }
    di_update_W(ret, ret.p_hat);
    ret.C = fminf(1.0f, ret.C);
    return ret;
}

// ReSTIRDI::combine_temporal (direct.cpp:327-371).
__device__ VS_OUTLINE DiReservoir di_combine_temporal(const DeviceScene &s, const RtParams &p, const DiReservoir &cur,
                                                      const RtSurface &cs, DiReservoir other, f3 view_pos,
                                                      f3 prev_view_pos, Sampler &smp, RWl &wl) {
    other.age += 1u;
    Interaction it = it_at(s, cs.hit, view_pos);
    float p_n_at_n, mis_cur, mis_prev;
    if (p.di.t_mis) {
        it.wo = normalize(prev_view_pos - it.pos);
        float p_c_at_n = di_p_hat_at(s, it, cur, wl);
        p_n_at_n = di_p_hat_at(s, it, other, wl);
        it.wo = normalize(view_pos - it.pos);
        float p_c_at_c = di_p_hat_at(s, it, cur, wl);
        float p_n_at_c = di_p_hat_at(s, it, other, wl);
        mis_cur = mis_n(static_cast<int>(cur.C), p_c_at_c, static_cast<int>(other.C), p_c_at_n);
        mis_prev = mis_n(static_cast<int>(other.C), p_n_at_n, static_cast<int>(cur.C), p_n_at_c);
    } else {
        it.wo = normalize(prev_view_pos - it.pos);
        p_n_at_n = di_p_hat_at(s, it, other, wl);
        mis_cur = cur.C / (cur.C + other.C);
        mis_prev = other.C / (other.C + cur.C);
    }
    DiReservoir ret = di_empty();
    di_update(ret, 0.5f, cur, safe_weight(mis_cur, cur.p_hat, cur.W), cur.C);
    DiReservoir os = other;
    os.p_hat = p_n_at_n;
    di_update(ret, smp.next(), os, safe_weight(mis_prev, p_n_at_n, other.W), other.C);
    di_update_W(ret, ret.p_hat);
    return ret;
}

// ReSTIRDI::temporal_reuse (direct.cpp:373-432).
__device__ VS_OUTLINE DiReservoir di_temporal(const DeviceScene &s, const RtParams &p, const RtBuffers &b,
                                              DiReservoir rsv, const RtSurface &cs, const RtSurfaceExt &cext,
                                              f2 mv, f2 p_film, Sampler &smp, RWl &wl) {
    const uint32_t prev = p.frame & 1u;
    f2 pp = p_film - mv;
    float limit = rsv.C * static_cast<float>(p.di.history_limit);
    f3 view_pos = cs.is_replaced ? make3(cext.vx, cext.vy, cext.vz) : p.view_pos;
    f3 prev_view_pos = p.prev_view_pos;
    int ix = f2i(pp.x), iy = f2i(pp.y);
    bool in_screen = ix >= 0 && iy >= 0 && ix < static_cast<int>(p.width) && iy < static_cast<int>(p.height);
    if (!(in_screen && p.di.temporal)) return rsv;
    auto fetch = [&](uint32_t x, uint32_t y, RtSurface &ps, DiReservoir &pr) {
        uint32_t idx = pixel_index(p, x, y);
        pr = b.di[prev][idx];
        pr.C = fminf(limit, pr.C);
        ps = b.surf[prev][idx];
        if (ps.is_replaced) {
            RtSurfaceExt e = b.ext[prev][idx];
            prev_view_pos = make3(e.vx, e.vy, e.vz);
        }
    };
    uint32_t px = min(f2u(pp.x), p.width - 1u), py = min(f2u(pp.y), p.height - 1u);
    RtSurface ps;
    DiReservoir pr;
    fetch(px, py, ps, pr);
    if (valid_neighbor(cs, ps, p.di.t_dot, p.di.t_depth, p.di.diff_factor) && pr.age < p.di.max_age) {
        return di_combine_temporal(s, p, rsv, cs, pr, view_pos, prev_view_pos, smp, wl);
    }
    for (uint32_t i = 0; i < p.di.t_count; ++i) {
        f2 d = square_to_disk2(smp.next2());
        uint32_t qx = min(f2u(d.x * p.di.t_radius + pp.x), p.width - 1u);
        uint32_t qy = min(f2u(d.y * p.di.t_radius + pp.y), p.height - 1u);
        fetch(qx, qy, ps, pr);
        if (valid_neighbor(cs, ps, p.di.t_dot, p.di.t_depth, p.di.diff_factor) && pr.age < p.di.max_age) {
            return di_combine_temporal(s, p, rsv, cs, pr, view_pos, prev_view_pos, smp, wl);
        }
    }
    return rsv;
}

__device__ __forceinline__ bool tile_pixel(const RtParams &p, uint32_t &x, uint32_t &y) {
    x = blockIdx.x * blockDim.x + threadIdx.x;
    y = blockIdx.y * blockDim.y + threadIdx.y;
    return x < p.width && y < p.height;
}

__device__ __forceinline__ RWl pixel_wavelengths(const DeviceScene &s, uint32_t x, uint32_t y, uint32_t frame) {
    Sampler w;
    if (s.ip.srgb) return rgb_wavelengths<RN>();
    w.start(x, y, frame, 0xffffffffu, s.ip.sampler, s.ip.seed);
    return sample_wavelengths<RN>(w.next());
}

}  // namespace

__global__ void k_rt_reset(uint32_t npix, const __grid_constant__ RtBuffers b) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    RtSurface sf{};
    sf.hit.inst_id = kInvalid;
    sf.hit.prim_id = kInvalid;
    sf.flag = kFlagUnset;
    RtSurfaceExt ex = RtSurfaceExt{1.0f, 1.0f, 1.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0u};
    DiReservoir dr = di_empty();
    GiReservoir gr{};
    RtHitBsdf hb{};
    hb.pdf = -1.0f;
    for (int k = 0; k < 2; ++k) {
        b.surf[k][i] = sf;
        b.ext[k][i] = ex;
        b.di[k][i] = dr;
        b.gi[k][i] = gr;
    }
    b.di_pass[i] = dr;
    b.gi_pass[i] = gr;
    b.gi_init[i] = gr;
    b.hit_bsdf[i] = hb;
    b.motion[i] = make_float2(0.0f, 0.0f);
    b.di_radiance[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    b.gi_radiance[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

// Minimum resident blocks per SM of the candidate and spatial kernels (a
// register budget).  3 blocks of 128 (at most 170 registers) measured 5 %
// faster on the many-light frame than the compiler's own 207 registers
// (2 blocks), despite the spills it caused in the one-kernel spatial pass.
#ifndef VS_RT_MIN_BLOCKS
#define VS_RT_MIN_BLOCKS 3
#endif
// The light-candidate pass waits on dependent loads (light table, primitive
// table, vertices) at a quarter occupancy; its own register budget.
#ifndef VS_RT_LIGHTS_MIN_BLOCKS
#define VS_RT_LIGHTS_MIN_BLOCKS VS_RT_MIN_BLOCKS
#endif

// ReSTIRDI shader0 (direct.cpp:519-557).
__global__ void __launch_bounds__(128, VS_RT_MIN_BLOCKS)
    k_di_candidates(const __grid_constant__ DeviceScene s, const __grid_constant__ RtParams p,
                    const __grid_constant__ RtBuffers b) {
    uint32_t x, y;
    if (!tile_pixel(p, x, y)) return;
    const uint32_t idx = pixel_index(p, x, y);
    const uint32_t cur = (p.frame + 1u) & 1u;
    RWl wl = pixel_wavelengths(s, x, y, p.frame);
    Sampler smp;
    smp.start(x, y, p.frame, 0u, s.ip.sampler, s.ip.seed);
    f2 p_film;
    f3 ro, rd;
    (void)camera_ray(s, s.cam, smp, x, y, p_film, ro, rd);
    PrimaryHit ph = compute_hit(s, p, smp, wl, ro, rd);
    b.surf[cur][idx] = ph.surf;
    if (ph.surf.is_replaced) b.ext[cur][idx] = ph.ext;
    f3 tp = make3(ph.ext.tx, ph.ext.ty, ph.ext.tz);
    RtHitBsdf hb{};
    hb.pdf = -1.0f;
    DiReservoir rsv = di_empty();
    if (ph.hit) {
        rsv = di_ris(s, p, ph.it, smp, wl, tp, hb);
    } else {
        di_update_W(rsv, rsv.p_hat);
        rsv.C = fminf(1.0f, rsv.C);
    }
    b.hit_bsdf[idx] = hb;
    // FrameBuffer::compute_motion_vec (frame_buffer.cpp:325-333).
    f2 mv = make2(0.0f, 0.0f);
    if (ph.hit) {
        f2 pr = prev_raster(p, ro + rd * ph.ext.t_max);
        mv = p_film - pr;
    }
    b.motion[idx] = make_float2(mv.x, mv.y);
    if (ph.hit) {
        if (occluded_to(s, ph.it, ld3p(rsv.pos))) {
            rsv.W = 0.0f;
            rsv.weight_sum = 0.0;
        }
    }
    rsv = di_temporal(s, p, b, rsv, ph.surf, ph.ext, mv, p_film, smp, wl);
    b.di_pass[idx] = rsv;
}

// ---------------------------------------------------------------------------
// The same direct pass as k_di_candidates in stages, so that its three
// traversals (primary chain, BSDF candidate, visibility) run in small kernels
// and the candidate loop runs without traversal code beside it.  Per pixel the
// stages pass the sampler state, wavelengths, film position and the direction
// that found the primary surface through b.di_stage; the hit pixels are
// listed in b.di_list.  Every pixel makes the same draws in the same order as
// in k_di_candidates.  Used when M_bsdf <= 1.
// ---------------------------------------------------------------------------
namespace {

__device__ __forceinline__ void stage_store(const RtBuffers &b, uint32_t idx, f3 last_d, f2 p_film, const RWl &wl,
                                            const Sampler &smp, bool hit) {
    float4 *st = b.di_stage + 4ull * idx;
    st[0] = make_float4(last_d.x, last_d.y, last_d.z, p_film.x);
    st[1] = make_float4(p_film.y, wl.lambda[0], wl.lambda[1], wl.lambda[2]);
    st[2] = make_float4(wl.pdf[0], wl.pdf[1], wl.pdf[2], hit ? 1.0f : 0.0f);
    st[3] = make_float4(__uint_as_float(static_cast<uint32_t>(smp.state)),
                        __uint_as_float(static_cast<uint32_t>(smp.state >> 32)), 0.0f, 0.0f);
}

// Sampler state, wavelengths and film position of a pixel; returns the
// direction that found its primary surface.
__device__ __forceinline__ f3 stage_load(const DeviceScene &s, const RtBuffers &b, uint32_t idx, RWl &wl,
                                         Sampler &smp, f2 &p_film) {
    const float4 *st = b.di_stage + 4ull * idx;
    const float4 a = st[0], c = st[1], d = st[2], e = st[3];
    p_film = make2(a.w, c.x);
    wl.lambda[0] = c.y;
    wl.lambda[1] = c.z;
    wl.lambda[2] = c.w;
    wl.pdf[0] = d.x;
    wl.pdf[1] = d.y;
    wl.pdf[2] = d.z;
    smp.kind = s.ip.sampler;
    smp.seed = s.ip.seed;
    smp.state = static_cast<uint64_t>(__float_as_uint(e.x)) | (static_cast<uint64_t>(__float_as_uint(e.y)) << 32);
    return make3(a.x, a.y, a.z);
}

__device__ __forceinline__ void stage_sampler(const RtBuffers &b, uint32_t idx, const Sampler &smp) {
    b.di_stage[4ull * idx + 3] = make_float4(__uint_as_float(static_cast<uint32_t>(smp.state)),
                                             __uint_as_float(static_cast<uint32_t>(smp.state >> 32)), 0.0f, 0.0f);
}

// The primary surface of a listed pixel (compute_hit's interaction) and the
// throughput of its near-specular chain.
__device__ __forceinline__ Interaction stage_surface(const DeviceScene &s, const RtParams &p, const RtBuffers &b,
                                                     uint32_t idx, f3 last_d, f3 &tp) {
    const uint32_t cur = (p.frame + 1u) & 1u;
    const RtSurface cs = b.surf[cur][idx];
    tp = make3(1.0f);
    if (cs.is_replaced) {
        const RtSurfaceExt e = b.ext[cur][idx];
        tp = make3(e.tx, e.ty, e.tz);
    }
    return surface_interaction(s, cs.hit, last_d, true);
}

}  // namespace

// Stage 1: camera ray, primary chain, motion vector; pixels that see nothing
// get their (empty) reservoir here.
__global__ void __launch_bounds__(128) k_di_primary(const __grid_constant__ DeviceScene s,
                                                    const __grid_constant__ RtParams p,
                                                    const __grid_constant__ RtBuffers b) {
    uint32_t x, y;
    if (!tile_pixel(p, x, y)) return;
    const uint32_t idx = pixel_index(p, x, y);
    const uint32_t cur = (p.frame + 1u) & 1u;
    RWl wl = pixel_wavelengths(s, x, y, p.frame);
    Sampler smp;
    smp.start(x, y, p.frame, 0u, s.ip.sampler, s.ip.seed);
    f2 p_film;
    f3 ro, rd;
    (void)camera_ray(s, s.cam, smp, x, y, p_film, ro, rd);
    PrimaryHit ph = compute_hit(s, p, smp, wl, ro, rd);
    b.surf[cur][idx] = ph.surf;
    if (ph.surf.is_replaced) b.ext[cur][idx] = ph.ext;
    // FrameBuffer::compute_motion_vec (frame_buffer.cpp:325-333).
    f2 mv = make2(0.0f, 0.0f);
    if (ph.hit) {
        f2 pr = prev_raster(p, ro + rd * ph.ext.t_max);
        mv = p_film - pr;
    }
    b.motion[idx] = make_float2(mv.x, mv.y);
    stage_store(b, idx, ph.last_d, p_film, wl, smp, ph.hit);
    if (ph.hit) {
        b.di_list[wf::queue_push(b.di_count)] = idx;
    } else {
        RtHitBsdf hb{};
        hb.pdf = -1.0f;
        b.hit_bsdf[idx] = hb;
        DiReservoir rsv = di_empty();
        di_update_W(rsv, rsv.p_hat);
        rsv.C = fminf(1.0f, rsv.C);
        b.di_pass[idx] = rsv;
    }
}

// Stage 2: the light candidates and the BSDF candidate's ray.
__global__ void __launch_bounds__(128, VS_RT_LIGHTS_MIN_BLOCKS)
    k_di_lights(const __grid_constant__ DeviceScene s, const __grid_constant__ RtParams p,
                const __grid_constant__ RtBuffers b) {
    const uint32_t n = *b.di_count;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t idx = b.di_list[k];
        RWl wl;
        Sampler smp;
        f2 p_film;
        const f3 last_d = stage_load(s, b, idx, wl, smp, p_film);
        f3 tp;
        const Interaction it = stage_surface(s, p, b, idx, last_d, tp);
        Bsdf<RN, VS_RT_MATERIALS> bsdf = bsdf_at(s, it, wl);
        DiReservoir rsv = di_ris_lights(s, p, it, smp, wl, lum3(tp), bsdf);
        RtHitBsdf hb{};
        hb.pdf = -1.0f;
        if (p.M_bsdf == 1u) {
            const Ray ray = di_bsdf_ray(it, bsdf, smp, hb);
            b.di_ray[2ull * idx] = make_float4(ray.o.x, ray.o.y, ray.o.z, ray.tmax);
            b.di_ray[2ull * idx + 1] = make_float4(ray.d.x, ray.d.y, ray.d.z, 0.0f);
        } else {
            di_update_W(rsv, rsv.p_hat);
            rsv.C = fminf(1.0f, rsv.C);
        }
        b.hit_bsdf[idx] = hb;
        b.di_pass[idx] = rsv;
        stage_store(b, idx, last_d, p_film, wl, smp, true);
    }
}

// Stage 3: the BSDF candidates' closest hits (warps refill finished lanes,
// as the wavefront traversal kernels do).
__global__ void __launch_bounds__(128) k_di_bsdf_trace(const __grid_constant__ DeviceScene s,
                                                       const __grid_constant__ RtParams p,
                                                       const __grid_constant__ RtBuffers b) {
    if (p.M_bsdf != 1u) return;
    const uint32_t n = *b.di_count;
    uint2 stack[kStackSize];
    bool active = false, drained = false;
    uint32_t idx = 0;
    RayPre r;
    TravState t;
    for (;;) {
        if (!drained) {
            const uint32_t k = wf::refill(b.di_count + 1, n, active, drained);
            if (k < n) {
                idx = b.di_list[k];
                const float4 o = b.di_ray[2ull * idx], d = b.di_ray[2ull * idx + 1];
                r = precompute_ray(make3(o.x, o.y, o.z), make3(d.x, d.y, d.z));
                trav_init(t, r, o.w);
                active = true;
            }
        }
        if (!__any_sync(0xffffffffu, active)) break;
        if (active && closest_step(s, r, t, stack)) {
            b.di_hit[idx] = trav_hit(s, t);
            active = false;
        }
    }
}

// Stage 4: the BSDF candidate, the reservoir's weight, and the visibility ray
// towards the chosen sample.
__global__ void __launch_bounds__(128, VS_RT_MIN_BLOCKS)
    k_di_bsdf_eval(const __grid_constant__ DeviceScene s, const __grid_constant__ RtParams p,
                   const __grid_constant__ RtBuffers b) {
    const uint32_t n = *b.di_count;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t idx = b.di_list[k];
        RWl wl;
        Sampler smp;
        f2 p_film;
        const f3 last_d = stage_load(s, b, idx, wl, smp, p_film);
        f3 tp;
        const Interaction it = stage_surface(s, p, b, idx, last_d, tp);
        DiReservoir rsv = b.di_pass[idx];
        if (p.M_bsdf == 1u) {
            const Hit h = b.di_hit[idx];
            const float4 d = b.di_ray[2ull * idx + 1];
            DiReservoir cand;
            float weight;
            di_bsdf_candidate(s, p, it, wl, b.hit_bsdf[idx], h.inst_id != kInvalid, h, make3(d.x, d.y, d.z), lum3(tp),
                              cand, weight);
            di_update(rsv, smp.next(), cand, weight);
            di_update_W(rsv, rsv.p_hat);
            rsv.C = fminf(1.0f, rsv.C);
            b.di_pass[idx] = rsv;
            stage_sampler(b, idx, smp);
        }
        const Ray sh = spawn_ray_to(it.pos, it.ng, ld3p(rsv.pos));
        b.di_ray[2ull * idx] = make_float4(sh.o.x, sh.o.y, sh.o.z, sh.tmax);
        b.di_ray[2ull * idx + 1] = make_float4(sh.d.x, sh.d.y, sh.d.z, 0.0f);
    }
}

// Stage 5: visibility of the chosen samples (an occluded sample keeps its
// history count but loses its weight), with ray replacement.
__global__ void __launch_bounds__(128) k_di_visibility(const __grid_constant__ DeviceScene s,
                                                       const __grid_constant__ RtBuffers b) {
    const uint32_t n = *b.di_count;
    uint2 stack[kStackSize];
    bool active = false, drained = false;
    uint32_t idx = 0;
    RayPre r;
    TravState t;
    for (;;) {
        if (!drained) {
            const uint32_t k = wf::refill(b.di_count + 2, n, active, drained);
            if (k < n) {
                idx = b.di_list[k];
                const float4 o = b.di_ray[2ull * idx], d = b.di_ray[2ull * idx + 1];
                r = precompute_ray(make3(o.x, o.y, o.z), make3(d.x, d.y, d.z));
                trav_init(t, r, o.w);
                active = true;
            }
        }
        if (!__any_sync(0xffffffffu, active)) break;
        bool occluded = false;
        if (active && any_step(s, r, t, stack, occluded)) {
            if (occluded) {
                DiReservoir rsv = b.di_pass[idx];
                rsv.W = 0.0f;
                rsv.weight_sum = 0.0;
                b.di_pass[idx] = rsv;
            }
            active = false;
        }
    }
}

// Stage 6: temporal reuse for every pixel.
__global__ void __launch_bounds__(128, VS_RT_MIN_BLOCKS)
    k_di_temporal(const __grid_constant__ DeviceScene s, const __grid_constant__ RtParams p,
                  const __grid_constant__ RtBuffers b) {
    uint32_t x, y;
    if (!tile_pixel(p, x, y)) return;
    const uint32_t idx = pixel_index(p, x, y);
    const uint32_t cur = (p.frame + 1u) & 1u;
    RWl wl;
    Sampler smp;
    f2 p_film;
    (void)stage_load(s, b, idx, wl, smp, p_film);
    const RtSurface cs = b.surf[cur][idx];
    RtSurfaceExt cext{};
    if (cs.is_replaced) cext = b.ext[cur][idx];
    const float2 m = b.motion[idx];
    DiReservoir rsv = di_temporal(s, p, b, b.di_pass[idx], cs, cext, make2(m.x, m.y), p_film, smp, wl);
    b.di_pass[idx] = rsv;
}

namespace {

// ReSTIRDI::neighbor_pairwise_MIS / canonical_pairwise_MIS / pairwise_combine
// (direct.cpp:235-282) and constant_combine (:284-300).
__device__ VS_OUTLINE DiReservoir di_combine_spatial(const DeviceScene &s, const RtParams &p, const RtBuffers &b,
                                                     const DiReservoir &canon, const RtSurface &cs, f3 view_pos,
                                                     const uint32_t *nb, uint32_t count, Sampler &smp, RWl &wl) {
    const uint32_t cur = (p.frame + 1u) & 1u;
    Interaction cit = it_at(s, cs.hit, view_pos);
    DiReservoir ret = di_empty();
    if (p.pairwise) {
        float canonical_weight = 0.0f;
        uint32_t M = count + 1u;
        float num = static_cast<float>(M - 1u);
        for (uint32_t k = 0; k < count; ++k) {
            DiReservoir nr = b.di_pass[nb[k]];
            RtSurface ns = b.surf[cur][nb[k]];
            Interaction nit = it_at(s, ns.hit, view_pos);
            float p_c_at_c = di_p_hat_at(s, cit, canon, wl);
            float p_c_at_n = di_p_hat_at(s, nit, canon, wl);
            float p_n_at_n = di_p_hat_at(s, nit, nr, wl);
            float p_n_at_c = di_p_hat_at(s, cit, nr, wl);
            float mi = mis_n(1, p_n_at_n, static_cast<int>(num), p_n_at_c);
            di_update(ret, smp.next(), nr, safe_weight(mi, nr.p_hat, nr.W), nr.C);
            float cw = mis_n(1, p_c_at_c, static_cast<int>(num), p_c_at_n) / num;
            canonical_weight += isnan(cw) ? 0.0f : cw;
        }
        canonical_weight = canonical_weight == 0.0f ? 1.0f : canonical_weight;
        di_update(ret, smp.next(), canon, safe_weight(canonical_weight, canon.p_hat, canon.W), canon.C);
        di_update_W(ret, ret.p_hat);
        return ret;
    }
    float inv_n = 1.0f / static_cast<float>(count + 1u);
    di_update(ret, 0.5f, canon, cal_weight(inv_n, canon.p_hat, canon.W), canon.C);
    for (uint32_t k = 0; k < count; ++k) {
        DiReservoir nr = b.di_pass[nb[k]];
        nr.p_hat = di_p_hat_at(s, cit, nr, wl);
        di_update(ret, smp.next(), nr, cal_weight(inv_n, nr.p_hat, nr.W), nr.C);
    }
    di_update_W(ret, ret.p_hat);
    return ret;
}


}  // namespace


// ReSTIRDI shader1 (direct.cpp:638-674) in stages, so the shading ray runs in
// a small traversal kernel: k_di_sp_combine (neighbours and combine; pixels
// that see nothing or an emitter are shaded here), k_di_sp_vis (the shading
// rays of the others), k_di_sp_shade (ReSTIRDI::shading with that
// visibility).  The shading rays and the listed pixels reuse the direct
// pass's ray and list buffers; the wavelengths pass through b.di_stage.
__global__ void __launch_bounds__(128, VS_RT_MIN_BLOCKS)
    k_di_sp_combine(const __grid_constant__ DeviceScene s, const __grid_constant__ RtParams p,
                    const __grid_constant__ RtBuffers b) {
    uint32_t x, y;
    if (!tile_pixel(p, x, y)) return;
    const uint32_t idx = pixel_index(p, x, y);
    const uint32_t cur = (p.frame + 1u) & 1u;
    RWl wl = pixel_wavelengths(s, x, y, p.frame);
    Sampler smp;
    smp.start(x, y, p.frame, 0u, s.ip.sampler, s.ip.seed);
    f2 p_film;
    f3 ro, rd;
    (void)camera_ray(s, s.cam, smp, x, y, p_film, ro, rd);
    smp.start(x, y, p.frame, 1u, s.ip.sampler, s.ip.seed);
    RtSurface cs = b.surf[cur][idx];
    DiReservoir rsv = b.di_pass[idx];
    f3 view_pos = p.view_pos;
    if (cs.is_replaced) {
        RtSurfaceExt e = b.ext[cur][idx];
        view_pos = make3(e.vx, e.vy, e.vz);
    }
    if (p.di.spatial) {
        uint32_t nb[kMaxSpatialNeighbours];
        uint32_t count = 0;
        for (uint32_t i = 0; i < p.di.s_count; ++i) {
            f2 d = square_to_disk2(smp.next2());
            int qx = static_cast<int>(x) + f2i(roundf(d.x * p.di.s_radius));
            int qy = static_cast<int>(y) + f2i(roundf(d.y * p.di.s_radius));
            qx = min(max(qx, 0), static_cast<int>(p.width) - 1);
            qy = min(max(qy, 0), static_cast<int>(p.height) - 1);
            uint32_t q = pixel_index(p, static_cast<uint32_t>(qx), static_cast<uint32_t>(qy));
            RtSurface os = b.surf[cur][q];
            if (valid_neighbor(cs, os, p.di.s_dot, p.di.s_depth, p.di.diff_factor)) nb[count++] = q;
        }
        if (cs.hit.inst_id != kInvalid) rsv = di_combine_spatial(s, p, b, rsv, cs, view_pos, nb, count, smp, wl);
    }
    b.di[cur][idx] = rsv;
    f3 L = make3(0.0f);
    if (cs.hit.inst_id != kInvalid) {
        Interaction it = it_at(s, cs.hit, view_pos);
        if (it.light != kInvalid) {
            AreaLight Ls = s.lights[it.light];
            LightPoint lp{it.pos, it.ng, it.prim_area};
            RSpec Le = area_Le(Ls, lp, p.view_pos, wl);
            L = linear_srgb<RN>(RSpec::fill(0.0f) + Le, wl);
        } else {
            const Ray sh = spawn_ray_to(it.pos, it.ng, ld3p(rsv.pos));
            b.di_ray[2ull * idx] = make_float4(sh.o.x, sh.o.y, sh.o.z, sh.tmax);
            b.di_ray[2ull * idx + 1] = make_float4(sh.d.x, sh.d.y, sh.d.z, 0.0f);
            float4 *st = b.di_stage + 4ull * idx;
            st[0] = make_float4(wl.lambda[0], wl.lambda[1], wl.lambda[2], wl.pdf[0]);
            st[1] = make_float4(wl.pdf[1], wl.pdf[2], 0.0f, 0.0f);
            b.di_list[wf::queue_push(b.di_count)] = idx;
            return;
        }
    } else if (s.has_env) {
        // LightSampler::evaluate_miss_wi along the camera ray (direct.cpp:659-668).
        RSpec Le;
        float env_pdf;
        env_eval<RN>(s, normalize((ro + rd) - ro), wl, Le, env_pdf);
        L = linear_srgb<RN>(Le, wl);
    }
    b.di_radiance[idx] = make_float4(L.x, L.y, L.z, 1.0f);
}

// Shading rays of the listed pixels (ray replacement); w of the direction
// record becomes 1 when the ray is occluded.
__global__ void __launch_bounds__(128) k_di_sp_vis(const __grid_constant__ DeviceScene s,
                                                   const __grid_constant__ RtBuffers b) {
    const uint32_t n = *b.di_count;
    uint2 stack[kStackSize];
    bool active = false, drained = false;
    uint32_t idx = 0;
    RayPre r;
    TravState t;
    for (;;) {
        if (!drained) {
            const uint32_t k = wf::refill(b.di_count + 1, n, active, drained);
            if (k < n) {
                idx = b.di_list[k];
                const float4 o = b.di_ray[2ull * idx], d = b.di_ray[2ull * idx + 1];
                r = precompute_ray(make3(o.x, o.y, o.z), make3(d.x, d.y, d.z));
                trav_init(t, r, o.w);
                active = true;
            }
        }
        if (!__any_sync(0xffffffffu, active)) break;
        bool occluded = false;
        if (active && any_step(s, r, t, stack, occluded)) {
            b.di_ray[2ull * idx + 1].w = occluded ? 1.0f : 0.0f;
            active = false;
        }
    }
}

// ReSTIRDI::shading (direct.cpp:583-636) of the listed pixels.  The
// BSDF-sampled emission the reference computes there is overwritten before
// use, so it is not traced.
__global__ void __launch_bounds__(128, VS_RT_MIN_BLOCKS)
    k_di_sp_shade(const __grid_constant__ DeviceScene s, const __grid_constant__ RtParams p,
                  const __grid_constant__ RtBuffers b) {
    const uint32_t n = *b.di_count;
    const uint32_t cur = (p.frame + 1u) & 1u;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t idx = b.di_list[k];
        const RtSurface cs = b.surf[cur][idx];
        DiReservoir rsv = b.di[cur][idx];
        const float4 *st = b.di_stage + 4ull * idx;
        const float4 s0 = st[0], s1 = st[1];
        RWl wl;
        wl.lambda[0] = s0.x;
        wl.lambda[1] = s0.y;
        wl.lambda[2] = s0.z;
        wl.pdf[0] = s0.w;
        wl.pdf[1] = s1.x;
        wl.pdf[2] = s1.y;
        f3 view_pos = p.view_pos;
        f3 tp = make3(1.0f);
        if (cs.is_replaced) {
            RtSurfaceExt e = b.ext[cur][idx];
            tp = make3(e.tx, e.ty, e.tz);
            view_pos = make3(e.vx, e.vy, e.vz);
        }
        Interaction it = it_at(s, cs.hit, view_pos);
        Bsdf<RN, VS_RT_MATERIALS> bsdf = bsdf_at(s, it, wl);
        RSpec f;
        di_p_hat(s, it, bsdf, rsv, wl, nullptr, nullptr, &f);
        RSpec value = f * spec3(tp) * (1.0f / lum3(tp));
        if (b.di_ray[2ull * idx + 1].w != 0.0f) {
            rsv.W = 0.0f;
            rsv.weight_sum = 0.0;
        }
        value = value * rsv.W;
        const f3 L = linear_srgb<RN>(value + RSpec::fill(0.0f), wl);
        b.di_radiance[idx] = make_float4(L.x, L.y, L.z, 1.0f);
    }
}

namespace {

// GISample::p_hat with ReSTIRGI::eval_bsdf (indirect.cpp:113-128,
// reservoir.h:166-170): luminance(Lo * f.vec3()) toward the sample point.
__device__ __forceinline__ f3 gi_f(const DeviceScene &s, const Interaction &it, const GiReservoir &g, RWl &wl) {
    Bsdf<RN, VS_RT_MATERIALS> bsdf = bsdf_at(s, it, wl);
    f3 wi = normalize(ld3p(g.sp_pos) - it.pos);
    return vec3(bsdf.evaluate(it.wo, wi, nullptr).f);
}
__device__ __forceinline__ float gi_p_hat(const DeviceScene &s, const Interaction &it, const GiReservoir &g,
                                          RWl &wl) {
    return lum3(ld3p(g.Lo) * gi_f(s, it, g, wl));
}

// ReSTIRGI::Jacobian_det (indirect.cpp:14-30).
__device__ __forceinline__ float jacobian(f3 cur_pos, f3 nb_pos, const GiReservoir &g) {
    f3 sp = ld3p(g.sp_pos), n = ld3p(g.sp_ng);
    f3 cv = cur_pos - sp, nv = nb_pos - sp;
    float cc = fabsf(dot(normalize(cv), n));
    float cn = fabsf(dot(normalize(nv), n));
    float r = (cc * length_sq(nv)) / (cn * length_sq(cv));
    if (bad(r)) r = 0.0f;
    return clampf(r, 0.6f, 1.0f / 0.6f);
}

// ReSTIRGI::combine_temporal (indirect.cpp:130-153).
__device__ VS_OUTLINE GiReservoir gi_combine_temporal(const DeviceScene &s, const GiReservoir &cur,
                                                      const RtSurface &cs, GiReservoir other, const RtSurface *ns,
                                                      f3 view_pos, f3 prev_view_pos, Sampler &smp, RWl &wl) {
    other.age += 1.0f;
    Interaction it = it_at(s, cs.hit, view_pos);
    GiReservoir ret{};
    float cur_p_hat = gi_p_hat(s, it, cur, wl);
    gi_update(ret, smp.next(), cur, safe_weight(cur.C, cur_p_hat, cur.W));
    float other_p_hat = gi_p_hat(s, it, other, wl);
    gi_update(ret, smp.next(), other, safe_weight(other.C, other_p_hat, other.W), other.C);
    float ph = gi_p_hat(s, it, ret, wl);
    if (ns) {
        Interaction nit = it_at(s, ns->hit, prev_view_pos);
        ph = ph * jacobian(it.pos, nit.pos, other);
    }
    gi_update_W(ret, ph);
    return ret;
}

}  // namespace

// ReSTIRGI initial samples (indirect.cpp:43-111).
__global__ void __launch_bounds__(128) k_gi_initial(const __grid_constant__ DeviceScene s,
                                                    const __grid_constant__ RtParams p,
                                                    const __grid_constant__ RtBuffers b) {
    uint32_t x, y;
    if (!tile_pixel(p, x, y)) return;
    const uint32_t idx = pixel_index(p, x, y);
    const uint32_t cur = (p.frame + 1u) & 1u;
    RWl wl = pixel_wavelengths(s, x, y, p.frame);
    RtSurface cs = b.surf[cur][idx];
    if (cs.hit.inst_id == kInvalid) {
        b.gi_radiance[idx] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        return;
    }
    f3 view_pos = p.view_pos;
    f3 tp_chain = make3(1.0f);
    if (cs.is_replaced) {
        RtSurfaceExt e = b.ext[cur][idx];
        view_pos = make3(e.vx, e.vy, e.vz);
        tp_chain = make3(e.tx, e.ty, e.tz);
    }
    Interaction it = it_at(s, cs.hit, view_pos);
    RtHitBsdf hb = b.hit_bsdf[idx];
    Sampler smp;
    smp.start(x, y, p.frame, 3u, s.ip.sampler, s.ip.seed);
    f3 wi = make3(hb.wx, hb.wy, hb.wz);
    Ray ray = spawn_ray(it.pos, it.ng, wi);
    f3 tp = zero_if_nan_inf(make3(hb.fx, hb.fy, hb.fz) / hb.pdf);
    Interaction first;
    first.pos = make3(0.0f);
    first.ng = make3(0.0f);
    f3 L = path_li<RN>(s, smp, wl, ray.o, ray.d, hb.pdf, spec3(tp), p.gi_max_depth, &first);
    L = zero_if_nan_inf(make3(L.x / tp.x, L.y / tp.y, L.z / tp.z));
    GiReservoir g{};
    st3(g.sp_pos, first.pos);
    st3(g.sp_ng, first.ng);
    st3(g.Lo, L * tp_chain);
    b.gi_init[idx] = g;
}

// ---------------------------------------------------------------------------
// The initial indirect samples in wavefront form: k_gi_initial's path suffix
// (path_li from the DI pass's BSDF sample) as wavefront passes over one slot
// per pixel (slot = pixel index; the queue counters are cleared before the
// start kernel).  k_gi_wf_start builds each path and writes the pixel's sample
// with zero radiance; k_gi_wf_first records the first
// vertex of the suffix after the bounce-0 closest hits; the bounce passes
// leave each path's radiance in `radiance`; k_gi_wf_finish divides by the
// BSDF weight as k_gi_initial does.  Same draws and sums as path_li, so the
// samples are k_gi_initial's.
// ---------------------------------------------------------------------------
namespace {

struct RtScene {
    const DeviceScene *s;
    __device__ __forceinline__ const DeviceScene &operator()(uint32_t) const { return *s; }
};

// The pixel's surface, view position and near-specular chain throughput;
// false when the camera ray left the scene.
__device__ __forceinline__ bool gi_surface(const DeviceScene &s, const RtParams &p, const RtBuffers &b,
                                           uint32_t idx, Interaction &it, f3 &tp_chain) {
    const uint32_t cur = (p.frame + 1u) & 1u;
    RtSurface cs = b.surf[cur][idx];
    if (cs.hit.inst_id == kInvalid) return false;
    f3 view_pos = p.view_pos;
    tp_chain = make3(1.0f);
    if (cs.is_replaced) {
        RtSurfaceExt e = b.ext[cur][idx];
        view_pos = make3(e.vx, e.vy, e.vz);
        tp_chain = make3(e.tx, e.ty, e.tz);
    }
    it = it_at(s, cs.hit, view_pos);
    return true;
}

}  // namespace

__global__ void __launch_bounds__(128) k_gi_wf_start(const __grid_constant__ DeviceScene s,
                                                     const __grid_constant__ RtParams p,
                                                     const __grid_constant__ RtBuffers b,
                                                     const __grid_constant__ WfBuffers w) {
    const uint32_t npix = p.width * p.height;
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < npix; idx += gridDim.x * blockDim.x) {
        const uint32_t x = idx % p.width, y = idx / p.width;
        Interaction it;
        f3 tp_chain;
        if (!gi_surface(s, p, b, idx, it, tp_chain)) {
            b.gi_radiance[idx] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            continue;
        }
        const RtHitBsdf hb = b.hit_bsdf[idx];
        PathState<RN> ps;
        ps.smp.start(x, y, p.frame, 3u, s.ip.sampler, s.ip.seed);
        ps.wl = pixel_wavelengths(s, x, y, p.frame);
        const Ray ray = spawn_ray(it.pos, it.ng, make3(hb.wx, hb.wy, hb.wz));
        const f3 tp = zero_if_nan_inf(make3(hb.fx, hb.fy, hb.fz) / hb.pdf);
        ps.ro = ray.o;
        ps.rd = ray.d;
        ps.scatter_pdf = hb.pdf;
        ps.throughput = spec3(tp);
        ps.L = make3(0.0f);
        ps.eta_scale = 1.0f;
        ps.bounce = 0;
        ps.filter_w = 1.0f;
        GiReservoir g{};
        b.gi_init[idx] = g;
        if (p.gi_max_depth == 0u) continue;
        wf::store<RN>(w, idx, ps, 0u);
        w.queue[0][wf::queue_push(&w.count[0])] = idx;
    }
}

// The first vertex of each suffix (the HitContext of path_li) after the
// bounce-0 closest hits.
__global__ void __launch_bounds__(128) k_gi_wf_first(const __grid_constant__ DeviceScene s,
                                                     const __grid_constant__ RtBuffers b,
                                                     const __grid_constant__ WfBuffers w) {
    const uint32_t n = w.count[0];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t slot = w.queue[0][i];
        const Hit h = w.hit[slot];
        if (h.inst_id == kInvalid) continue;
        const float4 d = w.d[slot];
        const Interaction it = surface_interaction(s, h, make3(d.x, d.y, d.z), true);
        GiReservoir g{};
        st3(g.sp_pos, it.pos);
        st3(g.sp_ng, it.ng);
        b.gi_init[slot] = g;
    }
}

template <uint32_t C>
__global__ void __launch_bounds__(128) k_gi_wf_shade(const __grid_constant__ DeviceScene s,
                                                     const __grid_constant__ WfBuffers w, uint32_t cur,
                                                     float4 *radiance) {
    wf::shade<RN, C>(RtScene{&s}, w, cur, 0, radiance);
}

__global__ void __launch_bounds__(128) k_gi_wf_extend(const __grid_constant__ DeviceScene s,
                                                      const __grid_constant__ WfBuffers w, uint32_t cur) {
    wf::extend<kLevelsFlat>(RtScene{&s}, w, cur);
}

__global__ void __launch_bounds__(128) k_gi_wf_shadow(const __grid_constant__ DeviceScene s,
                                                      const __grid_constant__ WfBuffers w, float4 *radiance) {
    wf::shadow<kLevelsFlat>(RtScene{&s}, w, 0, radiance);
}

// Radiance of each suffix over the BSDF weight, times the chain throughput.
__global__ void __launch_bounds__(128) k_gi_wf_finish(const __grid_constant__ DeviceScene s,
                                                      const __grid_constant__ RtParams p,
                                                      const __grid_constant__ RtBuffers b, const float4 *radiance) {
    const uint32_t npix = p.width * p.height;
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < npix; idx += gridDim.x * blockDim.x) {
        Interaction it;
        f3 tp_chain;
        if (!gi_surface(s, p, b, idx, it, tp_chain)) continue;
        const RtHitBsdf hb = b.hit_bsdf[idx];
        const f3 tp = zero_if_nan_inf(make3(hb.fx, hb.fy, hb.fz) / hb.pdf);
        f3 L = make3(0.0f);
        if (p.gi_max_depth != 0u) L = make3(radiance[idx].x, radiance[idx].y, radiance[idx].z);
        L = zero_if_nan_inf(make3(L.x / tp.x, L.y / tp.y, L.z / tp.z));
        GiReservoir g = b.gi_init[idx];
        st3(g.Lo, L * tp_chain);
        b.gi_init[idx] = g;
    }
}

// ReSTIRGI temporal pass (indirect.cpp:155-236).
__global__ void __launch_bounds__(128) k_gi_temporal(const __grid_constant__ DeviceScene s,
                                                     const __grid_constant__ RtParams p,
                                                     const __grid_constant__ RtBuffers b) {
    uint32_t x, y;
    if (!tile_pixel(p, x, y)) return;
    const uint32_t idx = pixel_index(p, x, y);
    const uint32_t cur = (p.frame + 1u) & 1u, prev = p.frame & 1u;
    RWl wl = pixel_wavelengths(s, x, y, p.frame);
    RtSurface cs = b.surf[cur][idx];
    if (cs.hit.inst_id == kInvalid) return;
    Sampler smp;
    smp.start(x, y, p.frame, 0u, s.ip.sampler, s.ip.seed);
    f2 p_film;
    f3 ro, rd;
    (void)camera_ray(s, s.cam, smp, x, y, p_film, ro, rd);
    smp.start(x, y, p.frame, 4u, s.ip.sampler, s.ip.seed);
    GiReservoir sample = b.gi_init[idx];
    RtHitBsdf hb = b.hit_bsdf[idx];
    GiReservoir rsv{};
    float ph = lum3(ld3p(sample.Lo) * make3(hb.fx, hb.fy, hb.fz));
    gi_update(rsv, 0.5f, sample, safe_weight(1.0f, ph, 1.0f / hb.pdf));
    gi_update_W(rsv, ph);
    float2 mv = b.motion[idx];
    f2 pp = make2(p_film.x - mv.x, p_film.y - mv.y);
    float limit = rsv.C * static_cast<float>(p.gi.history_limit);
    f3 view_pos = p.view_pos;
    if (cs.is_replaced) {
        RtSurfaceExt e = b.ext[cur][idx];
        view_pos = make3(e.vx, e.vy, e.vz);
    }
    f3 prev_view_pos = p.prev_view_pos;
    int ix = f2i(pp.x), iy = f2i(pp.y);
    bool in_screen = ix >= 0 && iy >= 0 && ix < static_cast<int>(p.width) && iy < static_cast<int>(p.height);
    if (in_screen && p.gi.temporal) {
        auto fetch = [&](uint32_t qx, uint32_t qy, RtSurface &ps, GiReservoir &pr) {
            uint32_t q = pixel_index(p, qx, qy);
            pr = b.gi[prev][q];
            gi_truncation(pr, limit);
            ps = b.surf[prev][q];
            if (ps.is_replaced) {
                RtSurfaceExt e = b.ext[prev][q];
                prev_view_pos = make3(e.vx, e.vy, e.vz);
            }
        };
        uint32_t px = min(f2u(pp.x), p.width - 1u), py = min(f2u(pp.y), p.height - 1u);
        RtSurface ps;
        GiReservoir pr;
        fetch(px, py, ps, pr);
        if (valid_neighbor(cs, ps, p.gi.t_dot, p.gi.t_depth, p.gi.diff_factor) && pr.age < static_cast<float>(p.gi.max_age)) {
            rsv = gi_combine_temporal(s, rsv, cs, pr, nullptr, view_pos, prev_view_pos, smp, wl);
        } else {
            for (uint32_t i = 0; i < p.gi.t_count; ++i) {
                f2 d = square_to_disk2(smp.next2());
                uint32_t qx = min(f2u(d.x * p.gi.t_radius + pp.x), p.width - 1u);
                uint32_t qy = min(f2u(d.y * p.gi.t_radius + pp.y), p.height - 1u);
                fetch(qx, qy, ps, pr);
                if (valid_neighbor(cs, ps, p.gi.t_dot, p.gi.t_depth, p.gi.diff_factor) &&
                    pr.age < static_cast<float>(p.gi.max_age)) {
                    rsv = gi_combine_temporal(s, rsv, cs, pr, &ps, view_pos, prev_view_pos, smp, wl);
                    break;
                }
            }
        }
    }
    b.gi_pass[idx] = rsv;
}

// ---------------------------------------------------------------------------
// ReSTIRGI spatial reuse and shading (indirect.cpp:238-332) in stages, so its
// visibility rays (one per neighbour) run in a small traversal kernel:
// k_gi_sp_select picks the neighbours (same draws as the reference),
// computes each one's target pdf, Jacobian and weight and queues its
// visibility ray; k_gi_sp_vis traces them; k_gi_sp_combine merges the
// neighbours in order (same draws) and shades.  Per pixel the stages pass the
// sampler state and wavelengths through b.di_stage (free after the direct
// pass) and the neighbours through b.gs_nb.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128, VS_RT_MIN_BLOCKS)
    k_gi_sp_select(const __grid_constant__ DeviceScene s, const __grid_constant__ RtParams p,
                   const __grid_constant__ RtBuffers b) {
    uint32_t x, y;
    if (!tile_pixel(p, x, y)) return;
    const uint32_t idx = pixel_index(p, x, y);
    const uint32_t cur = (p.frame + 1u) & 1u;
    RWl wl = pixel_wavelengths(s, x, y, p.frame);
    RtSurface cs = b.surf[cur][idx];
    if (cs.hit.inst_id == kInvalid) return;
    Sampler smp;
    smp.start(x, y, p.frame, 5u, s.ip.sampler, s.ip.seed);
    f3 view_pos = p.view_pos;
    if (cs.is_replaced) {
        RtSurfaceExt e = b.ext[cur][idx];
        view_pos = make3(e.vx, e.vy, e.vz);
    }
    Interaction cit = it_at(s, cs.hit, view_pos);
    uint32_t count = 0;
    if (p.gi.spatial) {
        for (uint32_t i = 0; i < p.gi.s_count; ++i) {
            f2 d = square_to_disk2(smp.next2());
            int qx = static_cast<int>(x) + f2i(roundf(d.x * p.gi.s_radius));
            int qy = static_cast<int>(y) + f2i(roundf(d.y * p.gi.s_radius));
            qx = min(max(qx, 0), static_cast<int>(p.width) - 1);
            qy = min(max(qy, 0), static_cast<int>(p.height) - 1);
            uint32_t q = pixel_index(p, static_cast<uint32_t>(qx), static_cast<uint32_t>(qy));
            RtSurface os = b.surf[cur][q];
            if (valid_neighbor(cs, os, p.gi.s_dot, p.gi.s_depth, p.gi.diff_factor)) {
                const size_t e = static_cast<size_t>(idx) * kMaxSpatialNeighbours + count;
                float w = 0.0f;
                GiReservoir nr = b.gi_pass[q];
                if (lum3(ld3p(nr.Lo)) > 0.0f) {
                    RtSurface ns = b.surf[cur][q];
                    Interaction nit = it_at(s, ns.hit, view_pos);
                    float ph = gi_p_hat(s, cit, nr, wl) * jacobian(cit.pos, nit.pos, nr);
                    w = safe_weight(nr.C, ph, nr.W);
                    const Ray sh = spawn_ray_to(cit.pos, cit.ng, ld3p(nr.sp_pos));
                    b.gs_ray[2 * e] = make_float4(sh.o.x, sh.o.y, sh.o.z, sh.tmax);
                    b.gs_ray[2 * e + 1] = make_float4(sh.d.x, sh.d.y, sh.d.z, 0.0f);
                    b.gs_vis[e] = 1u;
                    b.gs_list[wf::queue_push(b.gs_count)] = static_cast<uint32_t>(e);
                }
                b.gs_nb[e] = make_float2(__uint_as_float(q), w);
                ++count;
            }
        }
    }
    float4 *st = b.di_stage + 4ull * idx;
    st[0] = make_float4(wl.lambda[0], wl.lambda[1], wl.lambda[2], wl.pdf[0]);
    st[1] = make_float4(wl.pdf[1], wl.pdf[2], __uint_as_float(count), 0.0f);
    st[2] = make_float4(__uint_as_float(static_cast<uint32_t>(smp.state)),
                        __uint_as_float(static_cast<uint32_t>(smp.state >> 32)), 0.0f, 0.0f);
}

// Visibility of the queued neighbour samples (ray replacement).
__global__ void __launch_bounds__(128) k_gi_sp_vis(const __grid_constant__ DeviceScene s,
                                                   const __grid_constant__ RtBuffers b) {
    const uint32_t n = b.gs_count[0];
    uint2 stack[kStackSize];
    bool active = false, drained = false;
    uint32_t e = 0;
    RayPre r;
    TravState t;
    for (;;) {
        if (!drained) {
            const uint32_t k = wf::refill(b.gs_count + 1, n, active, drained);
            if (k < n) {
                e = b.gs_list[k];
                const float4 o = b.gs_ray[2ull * e], d = b.gs_ray[2ull * e + 1];
                r = precompute_ray(make3(o.x, o.y, o.z), make3(d.x, d.y, d.z));
                trav_init(t, r, o.w);
                active = true;
            }
        }
        if (!__any_sync(0xffffffffu, active)) break;
        bool occluded = false;
        if (active && any_step(s, r, t, stack, occluded)) {
            if (occluded) b.gs_vis[e] = 0u;
            active = false;
        }
    }
}

// ReSTIRGI::constant_combine (indirect.cpp:238-262) and shading (:264-278).
__global__ void __launch_bounds__(128, VS_RT_MIN_BLOCKS)
    k_gi_sp_combine(const __grid_constant__ DeviceScene s, const __grid_constant__ RtParams p,
                    const __grid_constant__ RtBuffers b) {
    uint32_t x, y;
    if (!tile_pixel(p, x, y)) return;
    const uint32_t idx = pixel_index(p, x, y);
    const uint32_t cur = (p.frame + 1u) & 1u;
    RtSurface cs = b.surf[cur][idx];
    if (cs.hit.inst_id == kInvalid) return;
    const float4 *st = b.di_stage + 4ull * idx;
    const float4 s0 = st[0], s1 = st[1], s2 = st[2];
    RWl wl;
    wl.lambda[0] = s0.x;
    wl.lambda[1] = s0.y;
    wl.lambda[2] = s0.z;
    wl.pdf[0] = s0.w;
    wl.pdf[1] = s1.x;
    wl.pdf[2] = s1.y;
    const uint32_t count = __float_as_uint(s1.z);
    Sampler smp;
    smp.kind = s.ip.sampler;
    smp.seed = s.ip.seed;
    smp.state = static_cast<uint64_t>(__float_as_uint(s2.x)) | (static_cast<uint64_t>(__float_as_uint(s2.y)) << 32);
    GiReservoir rsv = b.gi_pass[idx];
    f3 view_pos = p.view_pos;
    if (cs.is_replaced) {
        RtSurfaceExt e = b.ext[cur][idx];
        view_pos = make3(e.vx, e.vy, e.vz);
    }
    Interaction cit = it_at(s, cs.hit, view_pos);
    if (p.gi.spatial) {
        GiReservoir ret = rsv;
        for (uint32_t k = 0; k < count; ++k) {
            const size_t e = static_cast<size_t>(idx) * kMaxSpatialNeighbours + k;
            const float2 nbw = b.gs_nb[e];
            GiReservoir nr = b.gi_pass[__float_as_uint(nbw.x)];
            if (lum3(ld3p(nr.Lo)) > 0.0f) {
                float v = b.gs_vis[e] ? 1.0f : 0.0f;
                gi_update(ret, smp.next(), nr, nbw.y * v, nr.C * v);
            }
        }
        gi_update_W(ret, gi_p_hat(s, cit, ret, wl));
        rsv = ret;
    }
    f3 L = ld3p(rsv.Lo) * gi_f(s, cit, rsv, wl) * rsv.W;
    b.gi_radiance[idx] = make_float4(L.x, L.y, L.z, 1.0f);
    b.gi[cur][idx] = rsv;
}

// RealTimeIntegrator combine kernel (rt.cpp:118-126) with
// NormalRadianceCollector::add_sample (normal.cpp:87-101).
__global__ void k_rt_combine(uint32_t npix, const __grid_constant__ RtBuffers b, float di, float ii,
                             uint32_t film_index, float4 *film) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    float4 d = b.di_radiance[i], g = b.gi_radiance[i];
    f3 L = make3(d.x * di + g.x * ii, d.y * di + g.y * ii, d.z * di + g.z * ii);
    L = zero_if_nan_inf(L);
    float4 acc = film_index == 0 ? make_float4(0, 0, 0, 0) : film[i];
    float a = 1.0f / static_cast<float>(film_index + 1u);
    acc.x = acc.x + a * (L.x - acc.x);
    acc.y = acc.y + a * (L.y - acc.y);
    acc.z = acc.z + a * (L.z - acc.z);
    acc.w = acc.w + a * (1.0f - acc.w);
    film[i] = acc;
}

cudaError_t upload_spectral_consts_rt(const float *x, const float *y, const float *z, const float *d65,
                                      float y_integral) {
    return upload_spectral_consts_tu(x, y, z, d65, y_integral);
}

cudaError_t launch_rt_reset(uint32_t npix, const RtBuffers &b, cudaStream_t st) {
    k_rt_reset<<<(npix + 255) / 256, 256, 0, st>>>(npix, b);
    return cudaGetLastError();
}

namespace {

template <typename K>
unsigned rt_wave_grid(K kernel) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 128, 0);
    return static_cast<unsigned>(std::max(1, sms * std::max(per_sm, 1)));
}

}  // namespace

cudaError_t launch_rt_frame(const DeviceScene &s, const RtParams &p, const RtBuffers &b, uint32_t film_index,
                            float4 *film, const WfBuffers *wf, float4 *radiance, uint32_t class_mask, cudaStream_t st,
                            unsigned *launches) {
    dim3 block(16, 8);
    dim3 grid((p.width + 15) / 16, (p.height + 7) / 8);
    unsigned n = 0;
    if (p.M_bsdf <= 1u && b.di_stage) {
        // One resident wave of each list kernel (its own occupancy).
        static unsigned g_lights = 0, g_trace = 0, g_eval = 0, g_vis = 0;
        if (!g_lights) {
            g_lights = rt_wave_grid(k_di_lights);
            g_trace = rt_wave_grid(k_di_bsdf_trace);
            g_eval = rt_wave_grid(k_di_bsdf_eval);
            g_vis = rt_wave_grid(k_di_visibility);
        }
        cudaError_t e = cudaMemsetAsync(b.di_count, 0, 3 * sizeof(uint32_t), st);
        if (e != cudaSuccess) return e;
        k_di_primary<<<grid, block, 0, st>>>(s, p, b);
        k_di_lights<<<g_lights, 128, 0, st>>>(s, p, b);
        k_di_bsdf_trace<<<g_trace, 128, 0, st>>>(s, p, b);
        k_di_bsdf_eval<<<g_eval, 128, 0, st>>>(s, p, b);
        k_di_visibility<<<g_vis, 128, 0, st>>>(s, b);
        k_di_temporal<<<grid, block, 0, st>>>(s, p, b);
        n += 6;
    } else {
        k_di_candidates<<<grid, block, 0, st>>>(s, p, b);
        ++n;
    }
    if (p.di.open) {
        static unsigned g_vis = 0, g_shade = 0;
        if (!g_vis) {
            g_vis = rt_wave_grid(k_di_sp_vis);
            g_shade = rt_wave_grid(k_di_sp_shade);
        }
        cudaError_t e = cudaMemsetAsync(b.di_count, 0, 3 * sizeof(uint32_t), st);
        if (e != cudaSuccess) return e;
        k_di_sp_combine<<<grid, block, 0, st>>>(s, p, b);
        k_di_sp_vis<<<g_vis, 128, 0, st>>>(s, b);
        k_di_sp_shade<<<g_shade, 128, 0, st>>>(s, p, b);
        n += 3;
    }
    if (wf && radiance) {
        static unsigned g_ext = 0, g_shadow = 0, g_shade[kWfClasses] = {};
        if (!g_ext) {
            g_ext = rt_wave_grid(k_gi_wf_extend);
            g_shadow = rt_wave_grid(k_gi_wf_shadow);
            g_shade[0] = rt_wave_grid(k_gi_wf_shade<0>);
            g_shade[1] = rt_wave_grid(k_gi_wf_shade<1>);
            g_shade[2] = rt_wave_grid(k_gi_wf_shade<2>);
            g_shade[3] = rt_wave_grid(k_gi_wf_shade<3>);
            g_shade[4] = rt_wave_grid(k_gi_wf_shade<4>);
            g_shade[5] = rt_wave_grid(k_gi_wf_shade<5>);
            g_shade[6] = rt_wave_grid(k_gi_wf_shade<6>);
        }
        const uint32_t np = p.width * p.height;
        const unsigned g_pix = (np + 127) / 128;
        const uint32_t mask = class_mask | 1u;
        cudaError_t e = cudaMemsetAsync(wf->count, 0, sizeof(uint32_t) * kWfCounters, st);
        if (e != cudaSuccess) return e;
        k_gi_wf_start<<<g_pix, 128, 0, st>>>(s, p, b, *wf);
        ++n;
        for (uint32_t bounce = 0; bounce < p.gi_max_depth; ++bounce) {
            const uint32_t cur = bounce & 1u;
            k_gi_wf_extend<<<g_ext, 128, 0, st>>>(s, *wf, cur);
            ++n;
            if (bounce == 0) {
                k_gi_wf_first<<<g_ext, 128, 0, st>>>(s, b, *wf);
                ++n;
            }
            if (mask & 1u) { k_gi_wf_shade<0><<<g_shade[0], 128, 0, st>>>(s, *wf, cur, radiance); ++n; }
            if (mask & 2u) { k_gi_wf_shade<1><<<g_shade[1], 128, 0, st>>>(s, *wf, cur, radiance); ++n; }
            if (mask & 4u) { k_gi_wf_shade<2><<<g_shade[2], 128, 0, st>>>(s, *wf, cur, radiance); ++n; }
            if (mask & 8u) { k_gi_wf_shade<3><<<g_shade[3], 128, 0, st>>>(s, *wf, cur, radiance); ++n; }
            if (mask & 16u) { k_gi_wf_shade<4><<<g_shade[4], 128, 0, st>>>(s, *wf, cur, radiance); ++n; }
            if (mask & 32u) { k_gi_wf_shade<5><<<g_shade[5], 128, 0, st>>>(s, *wf, cur, radiance); ++n; }
            if (mask & 64u) { k_gi_wf_shade<6><<<g_shade[6], 128, 0, st>>>(s, *wf, cur, radiance); ++n; }
            k_gi_wf_shadow<<<g_shadow, 128, 0, st>>>(s, *wf, radiance);
            ++n;
        }
        k_gi_wf_finish<<<g_pix, 128, 0, st>>>(s, p, b, radiance);
        ++n;
    } else {
        k_gi_initial<<<grid, block, 0, st>>>(s, p, b);
        ++n;
    }
    k_gi_temporal<<<grid, block, 0, st>>>(s, p, b);
    {
        static unsigned g_vis = 0;
        if (!g_vis) g_vis = rt_wave_grid(k_gi_sp_vis);
        cudaError_t e = cudaMemsetAsync(b.gs_count, 0, 2 * sizeof(uint32_t), st);
        if (e != cudaSuccess) return e;
        k_gi_sp_select<<<grid, block, 0, st>>>(s, p, b);
        k_gi_sp_vis<<<g_vis, 128, 0, st>>>(s, b);
        k_gi_sp_combine<<<grid, block, 0, st>>>(s, p, b);
        n += 2;
    }
    n += 2;
    uint32_t npix = p.width * p.height;
    k_rt_combine<<<(npix + 255) / 256, 256, 0, st>>>(npix, b, p.di_factor, p.gi_factor, film_index, film);
    ++n;
    if (launches) *launches = n;
    return cudaGetLastError();
}

}  // namespace VS_RT_NS
}  // namespace vs

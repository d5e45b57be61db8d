// BSDFs of the in-scope material plugins, evaluated and sampled in world space
// the way MaterialEvaluator does with individual shading normals
// (src/base/scattering/material.cpp:132-184): each lobe works in its local
// frame and multiplies f by |cos theta_i|; the evaluator zeroes the pdf when
// wi and wo lie on sides of the geometric normal that contradict the lobes'
// reflection/transmission flags.
//
// Materials: diffuse (diffuse.cpp), black_body (black_body.cpp), metal
// (metal.cpp: GGX conductor with complex Fresnel and albedo compensation),
// glass (glass.cpp: rough dielectric, optionally dispersive, compensated) and
// principled_bsdf (principled_bsdf.cpp: the lobe set sheen (LTC), coat,
// metallic F82, transmission, Schlick specular and diffuse, layered by
// albedo).
#pragma once

#include "vs_texture.cuh"
#include "vs_microfacet.h"

namespace vs {

// BxDFFlag (src/base/sample.h:24-49).
constexpr uint32_t kFlagUnset = 1u;
constexpr uint32_t kFlagReflection = 1u << 1;
constexpr uint32_t kFlagTransmission = 1u << 2;
constexpr uint32_t kFlagDiffuse = 1u << 3;
constexpr uint32_t kFlagGlossy = 1u << 4;
constexpr uint32_t kFlagSpecular = 1u << 5;
constexpr uint32_t kFlagDiffRefl = kFlagDiffuse | kFlagReflection;
constexpr uint32_t kFlagGlossyRefl = kFlagGlossy | kFlagReflection;
constexpr uint32_t kFlagGlossyTrans = kFlagGlossy | kFlagTransmission;

template <int N>
struct BsdfEval {
    Spec<N> f;
    float pdf;  // the reference keeps one scatter pdf broadcast to all channels
    uint32_t flags;
    __device__ __forceinline__ bool valid() const { return pdf > 0.0f; }
    __device__ __forceinline__ Spec<N> throughput() const { return f * (1.0f / pdf); }
};

template <int N>
struct BsdfSample {
    BsdfEval<N> eval;
    f3 wi;
    float eta;
};

// SampledWavelengths::invalidation_secondary (src/base/color/spectrum.cpp:21-31).
template <int N>
__device__ __forceinline__ void invalidate_secondary(Wavelengths<N> &w) {
    bool all_valid = N > 1;
#pragma unroll
    for (int i = 1; i < N; ++i) all_valid = all_valid && (w.pdf[i] != 0.0f);
    if (all_valid) {
#pragma unroll
        for (int i = 1; i < N; ++i) w.pdf[i] = 0.0f;
    }
}

// square_to_cosine_hemisphere (src/math/warp.h:24-47).
__device__ __forceinline__ f3 cosine_hemisphere(f2 u) {
    f2 d = square_to_disk(u);
    float z = sqrtf(fmaxf(0.0f, 1.0f - d.x * d.x - d.y * d.y));
    return {d.x, d.y, z};
}

template <int N>
__device__ __forceinline__ float avg(const Spec<N> &s) {
    float a = 0.0f;
#pragma unroll
    for (int i = 0; i < N; ++i) a += s.v[i];
    return a * (1.0f / N);
}

// Fresnel variants of the microfacet lobes (src/base/scattering/fresnel.h).
enum FresnelKind : uint32_t { kFresnelConductor = 0, kFresnelSchlick = 1, kFresnelF82 = 2, kFresnelConstant = 3,
                               kFresnelDielectric = 4 };

// One microfacet reflection lobe: MicrofacetReflection + Fresnel, with the
// PureReflectionLobe albedo compensation when `compensate` is set.
template <int N>
struct MfLobe {
    float ax, ay;
    uint32_t fresnel;
    bool compensate;
    Spec<N> kr;
    Spec<N> fa, fb;  // conductor: eta, k;  Schlick: F0, -;  F82: F0, B
    float eta0;      // Schlick: eta[0]

    __device__ __forceinline__ Spec<N> F(float c) const {
        Spec<N> r;
        if (fresnel == kFresnelConductor) {
#pragma unroll
            for (int i = 0; i < N; ++i) r.v[i] = fresnel_complex(c, fa.v[i], fb.v[i]);
        } else if (fresnel == kFresnelSchlick) {
            // FresnelSchlick::evaluate (fresnel.h:60-67).
            float f_real = fresnel_dielectric(c, eta0);
            float f0_real = schlick_F0_from_ior(eta0);
            float t = clampf((f_real - f0_real) / (1.0f - f0_real), 0.0f, 1.0f);
#pragma unroll
            for (int i = 0; i < N; ++i) r.v[i] = fa.v[i] + t * (1.0f - fa.v[i]);
        } else if (fresnel == kFresnelF82) {
            // FresnelF82Tint::evaluate (fresnel.h:117-124).
            float mu = clampf(1.0f - c, 0.0f, 1.0f);
            float mu2 = mu * mu;
            float mu5 = mu2 * mu2 * mu;
#pragma unroll
            for (int i = 0; i < N; ++i) {
                float fs = fa.v[i] + mu5 * (1.0f - fa.v[i]);
                r.v[i] = clampf(fs - fb.v[i] * c * mu5 * mu, 0.0f, 1.0f);
            }
        } else if (fresnel == kFresnelDielectric) {
            // FresnelDielectric (fresnel.h:74-90) with one eta for every channel.
            const float fr = fresnel_dielectric(c, eta0);
#pragma unroll
            for (int i = 0; i < N; ++i) r.v[i] = fr;
        } else {
            r = Spec<N>::fill(1.0f);
        }
        return r;
    }

    // MicrofacetLobe::evaluate_local_impl -> BxDF::safe_evaluate (bxdf.cpp:30-43),
    // MicrofacetReflection::f / PDF (bxdf.cpp:56-70), compensation (lobe.cpp:716-735).
    __device__ __forceinline__ void eval_local(f3 wo, f3 wi, const float *luts, Spec<N> &f, float &pdf) const {
        bool s = wo.z * wi.z > 0.0f;
        if (!s) {
            f = Spec<N>::fill(0.0f);
            pdf = 0.0f;
            return;
        }
        f3 wh = normalize(wo + wi);
        f3 whf = wh.z < 0.0f ? -wh : wh;
        float brdf = ggx_brdf(wo, whf, wi, ax, ay);
        Spec<N> Fr = F(fabsf(dot(wo, whf)));
        float comp = 1.0f;
        if (compensate) comp = 1.0f / lut_sample2(luts + kLutPureReflection, sqrtf(ax * ay), wo.z);
        f = Fr * kr * (brdf * comp);
        pdf = ggx_pdf_reflection(wo, wh, ax, ay);
    }
    // MicrofacetReflection::sample_wi (bxdf.cpp:72-77).
    __device__ __forceinline__ f3 sample_local(f3 wo, f2 u, bool &valid) const {
        f3 wh = ggx_sample_vndf(wo, u, ax, ay);
        f3 wi = reflect_dir(wo, wh);
        valid = wo.z * wi.z > 0.0f;
        return wi;
    }
};

// DielectricLobe (src/base/scattering/lobe.cpp:253-450).
template <int N>
struct DielLobe {
    float ax, ay;
    Spec<N> eta;  // per wavelength, already corrected for the side (Interaction::correct_eta)
    Spec<N> kt;
    bool compensate;
    // Fresnel: dielectric per wavelength (glass), or FresnelSchlick with F0
    // per channel and eta[0] (the principled transmission lobe).
    bool schlick;
    Spec<N> f0;

    __device__ __forceinline__ Spec<N> F(float c) const {
        Spec<N> r;
        if (schlick) {
            // FresnelSchlick::evaluate (fresnel.h:60-67).
            const float f_real = fresnel_dielectric(c, eta.v[0]);
            const float f0_real = schlick_F0_from_ior(eta.v[0]);
            const float t = clampf((f_real - f0_real) / (1.0f - f0_real), 0.0f, 1.0f);
#pragma unroll
            for (int i = 0; i < N; ++i) r.v[i] = f0.v[i] + t * (1.0f - f0.v[i]);
            return r;
        }
#pragma unroll
        for (int i = 0; i < N; ++i) r.v[i] = fresnel_dielectric(c, eta.v[i]);
        return r;
    }
    __device__ __forceinline__ float refl_prob(const Spec<N> &Fr) const {
        Spec<N> total;
#pragma unroll
        for (int i = 0; i < N; ++i) total.v[i] = (1.0f - Fr.v[i]) * kt.v[i] + Fr.v[i];
        return avg(Fr) / avg(total);
    }
    __device__ __forceinline__ float comp(f3 wo, const float *luts) const {
        if (!compensate) return 1.0f;
        float e = eta.v[0];
        const float *t = luts + (e > 1.0f ? kLutDielectric : kLutDielectricInv);
        float z = ((e > 1.0f ? e : 1.0f / e) - kIorLower) / (kIorUpper - kIorLower);
        float x = sqrtf(sqrtf(ax * ay));
        return 1.0f / lut_sample3(t, 2, 0, x, fabsf(wo.z), z);
    }
    __device__ __forceinline__ void eval_local(f3 wo, f3 wi, const float *luts, Spec<N> &f, float &pdf,
                                               uint32_t &flags, float &eta_out) const {
        bool reflect = wo.z * wi.z > 0.0f;
        float e0 = eta.v[0];
        float eta_p = reflect ? 1.0f : e0;
        eta_out = eta_p;
        f3 wh = normalize(wo + wi * eta_p);
        if (dot(wh, wo) < 0.0f) wh = -wh;
        Spec<N> Fr = F(fabsf(dot(wh, wo)));
        float c = comp(wo, luts);
        if (reflect) {
            f = Fr * (ggx_brdf(wo, wh, wi, ax, ay) * c);
            pdf = ggx_pdf_reflection(wo, wh, ax, ay) * refl_prob(Fr);
            flags = kFlagGlossyRefl;
        } else {
            f3 wh2 = normalize(wo + wi * e0);
            float bt = ggx_btdf(wo, wh2, wi, e0, ax, ay, true);
            Spec<N> T;
#pragma unroll
            for (int i = 0; i < N; ++i) T.v[i] = (1.0f - Fr.v[i]) * kt.v[i];
            f = T * (bt * c);
            pdf = ggx_pdf_transmission(wo, wh, wi, e0, ax, ay) * (1.0f - refl_prob(Fr));
            flags = kFlagGlossyTrans;
        }
    }
    // DielectricLobe::sample_wi_local_impl (lobe.cpp:431-449): 2D for the
    // microfacet normal, then 1D to choose reflection or refraction.
    __device__ __forceinline__ f3 sample_local(f3 wo, Sampler &smp, bool &valid) const {
        f3 wh = ggx_sample_vndf(wo, smp.next2(), ax, ay);
        float d = dot(wo, wh);
        Spec<N> Fr = F(fabsf(d));
        float uc = smp.next();
        f3 wi;
        if (uc < refl_prob(Fr)) {
            wi = reflect_dir(wo, wh);
            valid = wo.z * wi.z > 0.0f;
        } else {
            bool ok = refract_dir(wo, wh, eta.v[0], wi);
            valid = ok && !(wo.z * wi.z > 0.0f);
        }
        return wi;
    }
};

// SheenLTC (principled_bsdf.cpp:17-118, Zeltner et al. 2022): a linearly
// transformed cosine lobe whose (a, b) and albedo scale come from the fitted
// table at (cos theta of wo against the geometric normal, sheen roughness).
template <int N>
struct SheenLobe {
    float a, b;
    Spec<N> tint;  // sheen tint * weight * layer weight * the table's scale
    // eval_ltc: the cosine density of M^-1 wi times the Jacobian a^2 / |M^-1 wi|^3.
    __device__ __forceinline__ float eval_ltc(f3 wi) const {
        f3 w = make3(a * wi.x + b * wi.z, a * wi.y, wi.z);
        const float len = length(w);
        w = make3(w.x / len, w.y / len, w.z / len);
        const float jac = (a * a) / (len * len * len);
        return w.z * kInvPi * jac;
    }
    __device__ __forceinline__ void eval_local(f3 wo, f3 wi, Spec<N> &f, float &pdf) const {
        const float ltc = eval_ltc(wi);
        const bool below = wi.z < 0.0f || wo.z < 0.0f;
#pragma unroll
        for (int i = 0; i < N; ++i) f.v[i] = below ? 0.0f : (ltc * tint.v[i]) / wi.z;
        pdf = ltc;
    }
    // A cosine-hemisphere direction through M = [[1/a, 0, -b/a], [0, 1/a, 0], [0, 0, 1]].
    __device__ __forceinline__ f3 sample_local(f2 u) const {
        const f3 w = cosine_hemisphere(u);
        return normalize(make3(w.x / a - w.z * b / a, w.y / a, w.z));
    }
};

// Material types compiled into a Bsdf: bit t set for MaterialType t.  Kernels
// that shade one material class at a time instantiate only its code.
constexpr uint32_t kAllMaterials = 0x3fu;
template <uint32_t M>
__device__ __forceinline__ constexpr bool has_mat(uint32_t t) {
    return ((M >> t) & 1u) != 0u;
}

template <int N, uint32_t M = kAllMaterials>
struct Bsdf {
    uint32_t type;
    Frame frame;
    f3 ng;
    const float *luts;
    bool dispersive;
    // Diffuse colour (diffuse, principled diffuse lobe, substrate Rd).
    Spec<N> kd;
    // Substrate specular colour Rs; plastic: the lobe's Schlick Fresnel sits
    // in mf[0] (F0 = schlick_F0(ior) * Rs, eta0 = ior).
    Spec<N> ks;
    bool plastic;
    // Microfacet lobes: metal uses mf[0]; principled uses mf[0] = metallic,
    // mf[1] = specular, mf[2] = coat.
    MfLobe<N> mf[3];
    DielLobe<N> dl;
    SheenLobe<N> sh;
    // Principled lobe-set sample weights (normalised) in the reference's lobe
    // order: sheen, coat, metallic, transmission, specular, diffuse; and
    // whether the transmission lobe is present.
    float w_sheen, w_coat, w_metal, w_trans, w_spec, w_diff;
    float trans_scale;
    bool has_trans;

    // FresnelBlend (substrate.cpp:12-72) inside its MicrofacetLobe, through
    // BxDF::safe_evaluate (bxdf.cpp:30-43): Ashikhmin-Shirley glossy
    // specular over a diffuse base; the lobe picks specular with probability
    // F_dielectric(|cos wo|, 1.5) (the lobe's FresnelDielectric).
    __device__ __forceinline__ void substrate_eval(f3 wo, f3 wi, Spec<N> &f, float &pdf) const {
        if (!(wo.z * wi.z > 0.0f)) {
            f = Spec<N>::fill(0.0f);
            pdf = 0.0f;
            return;
        }
        const float ax = mf[0].ax, ay = mf[0].ay;
        const f3 wh = normalize(wi + wo);
        const float ci = fabsf(wi.z), co = fabsf(wo.z);
        const float d = ggx_D(wh, ax, ay) / (4.0f * fabsf(dot(wi, wh)) * fmaxf(ci, co));
        const float sw = pow5(clampf(1.0f - dot(wi, wh), 0.0f, 1.0f));
        const float mi = 1.0f - 0.5f * ci, mo = 1.0f - 0.5f * co;
        const float g = (28.0f / (23.0f * kPi)) * (1.0f - pow5(mi)) * (1.0f - pow5(mo));
#pragma unroll
        for (int i = 0; i < N; ++i) {
            const float spec = d * (ks.v[i] + sw * (1.0f - ks.v[i]));
            const float diff = g * kd.v[i] * (1.0f - ks.v[i]);
            f.v[i] = spec + diff;
        }
        const float fr = fresnel_dielectric(co, 1.5f);
        const float pd = ci * kInvPi;
        pdf = pd + fr * (ggx_pdf_reflection(wo, wh, ax, ay) - pd);
    }
    // PlasticLobe (plastic.cpp:27-59), evaluated without a hemisphere test
    // (evaluate_local_impl): Lambert(Rd) (1 - F) + GGX reflection with the
    // Schlick F at |wh . wo|; pdf lerp(avg F, cosine, GGX reflection).
    __device__ __forceinline__ void plastic_eval(f3 wo, f3 wi, Spec<N> &f, float &pdf) const {
        const float ax = mf[0].ax, ay = mf[0].ay;
        const f3 wh = normalize(wo + wi);
        const Spec<N> F = mf[0].F(fabsf(dot(wh, wo)));
        const float brdf = ggx_brdf(wo, wh, wi, ax, ay);
#pragma unroll
        for (int i = 0; i < N; ++i) f.v[i] = kd.v[i] * kInvPi * (1.0f - F.v[i]) + brdf * F.v[i];
        const float pd = fabsf(wi.z) * kInvPi;
        pdf = pd + avg(F) * (ggx_pdf_reflection(wo, wh, ax, ay) - pd);
    }
    // PlasticLobe::sample_wi_local_impl (plastic.cpp:61-78): a microfacet
    // normal (2D) and one number against avg F(|cos wo|) pick the mirror
    // direction (valid on wo's side) or a fresh cosine-hemisphere direction
    // (2D, upper hemisphere).
    __device__ __forceinline__ f3 plastic_sample(f3 wo, Sampler &smp, bool &valid) const {
        const f3 wh = ggx_sample_vndf(wo, smp.next2(), mf[0].ax, mf[0].ay);
        const Spec<N> F = mf[0].F(fabsf(wo.z));
        const float uc = smp.next();
        if (uc < avg(F)) {
            const f3 wi = reflect_dir(wo, wh);
            valid = wo.z * wi.z > 0.0f;
            return wi;
        }
        valid = true;
        return cosine_hemisphere(smp.next2());
    }
    __device__ __forceinline__ f3 substrate_sample(f3 wo, f2 u) const {
        const float fr = fresnel_dielectric(fabsf(wo.z), 1.5f);
        f3 wi;
        if (u.x < fr) {
            u.x = u.x / fr;
            wi = reflect_dir(wo, ggx_sample_vndf(wo, u, mf[0].ax, mf[0].ay));
        } else {
            u.x = (u.x - fr) / (1.0f - fr);
            wi = cosine_hemisphere(u);
            wi.z = wo.z < 0.0f ? -wi.z : wi.z;
        }
        return wi;
    }

    // MaterialEvaluator::albedo (material.cpp:91-98) at c = dot(shading
    // normal, wo), as each lobe defines it: Lambert kd; MicrofacetLobe
    // kr * F(c) (lobe.cpp:208-210: metal, mirror, plastic with kr = 1 and its
    // Schlick F, substrate with FresnelBlend's Rd and the dielectric F at 1.5);
    // DielectricLobe kt (1 - F) + F at |c| (lobe.cpp:308-313); the principled
    // lobe set summed with each lobe's weight (LobeSet::albedo, lobe.cpp:
    // 564-570): SheenLTC's tint, CoatLobe's and SpecularLobe's table values
    // (principled_bsdf.cpp:154-160,198-205), the F82 metallic lobe, the
    // transmission lobe; a black body reflects nothing.
    __device__ VS_OUTLINE Spec<N> albedo(float c) const {
        Spec<N> r = Spec<N>::fill(0.0f);
        if (has_mat<M>(kMatDiffuse) && type == kMatDiffuse) {
            r = kd;
        } else if (has_mat<M>(kMatMetal) && type == kMatMetal) {
            r = mf[0].kr * mf[0].F(c);
        } else if (has_mat<M>(kMatGlass) && type == kMatGlass) {
            const Spec<N> F = dl.F(fabsf(c));
#pragma unroll
            for (int i = 0; i < N; ++i) r.v[i] = dl.kt.v[i] * (1.0f - F.v[i]) + F.v[i];
        } else if (has_mat<M>(kMatSubstrate) && type == kMatSubstrate) {
            if (plastic) {
                r = mf[0].F(c);
            } else {
                const float F = fresnel_dielectric(c, 1.5f);
#pragma unroll
                for (int i = 0; i < N; ++i) r.v[i] = kd.v[i] * F;
            }
        } else if (has_mat<M>(kMatPrincipled) && type == kMatPrincipled) {
            if (w_sheen > 0.0f) r = r + sh.tint;
            if (w_coat > 0.0f) {
                const float x = sqrtf(sqrtf(mf[2].ax * mf[2].ax));
                const float z = (mf[2].eta0 - kCoatIorLower) / (kCoatIorUpper - kCoatIorLower);
                r = r + mf[2].kr * lut_sample3(luts + kLutCoat, 1, 0, x, c, z);
            }
            if (w_metal > 0.0f) r = r + mf[0].kr * mf[0].F(c);
            if (has_trans) {
                const Spec<N> F = dl.F(fabsf(c));
#pragma unroll
                for (int i = 0; i < N; ++i) r.v[i] += (dl.kt.v[i] * (1.0f - F.v[i]) + F.v[i]) * trans_scale;
            }
            if (w_spec > 0.0f) {
                const float ior = mf[1].eta0;
                const float x = sqrtf(sqrtf(mf[1].ax * mf[1].ay));
                const float z = sqrtf(fabsf((ior - 1.0f) / (ior + 1.0f)));
                const float sl = lut_sample3(luts + kLutSpecular, 1, 0, x, c, z);
#pragma unroll
                for (int i = 0; i < N; ++i) r.v[i] += (mf[1].fa.v[i] + sl * (1.0f - mf[1].fa.v[i])) * mf[1].kr.v[i];
            }
            if (w_diff > 0.0f) r = r + kd;
        }
        return r;
    }

    // Zero the pdf of a direction whose geometric side contradicts the flags
    // (MaterialEvaluator::evaluate, material.cpp:137-147).
    __device__ __forceinline__ void discard_check(f3 wo, f3 wi, BsdfEval<N> &e) const {
        bool same = dot(wo, ng) * dot(wi, ng) > 0.0f;
        bool trans = (e.flags & kFlagTransmission) != 0u;
        if (same == trans) e.pdf = 0.0f;
    }

    // The lobe set at local directions, before MaterialEvaluator's check of
    // the geometric side; a dielectric lobe sets eta.
    __device__ __forceinline__ BsdfEval<N> eval_core(f3 wo, f3 wi, float &eta) const {
        BsdfEval<N> e;
        float acos_i = fabsf(wi.z);
        if (has_mat<M>(kMatDiffuse) && type == kMatDiffuse) {
            bool s = wo.z * wi.z > 0.0f;
            e.f = s ? kd * (kInvPi * acos_i) : Spec<N>::fill(0.0f);
            e.pdf = s ? acos_i * kInvPi : 0.0f;
            e.flags = kFlagDiffRefl;
        } else if (has_mat<M>(kMatMetal) && type == kMatMetal) {
            mf[0].eval_local(wo, wi, luts, e.f, e.pdf);
            e.f = e.f * acos_i;
            e.flags = kFlagGlossyRefl;
        } else if (has_mat<M>(kMatGlass) && type == kMatGlass) {
            dl.eval_local(wo, wi, luts, e.f, e.pdf, e.flags, eta);
            e.f = e.f * acos_i;
        } else if (has_mat<M>(kMatSubstrate) && type == kMatSubstrate) {
            if (plastic) plastic_eval(wo, wi, e.f, e.pdf);
            else substrate_eval(wo, wi, e.f, e.pdf);
            e.f = e.f * acos_i;
            e.flags = kFlagReflection;
        } else if (has_mat<M>(kMatPrincipled) && type == kMatPrincipled) {
            // LobeSet::evaluate_impl (lobe.cpp:665-681): sum of the lobes, each
            // masked by its own hemisphere test, pdfs weighted by the
            // normalised sample weights.
            e.f = Spec<N>::fill(0.0f);
            e.pdf = 0.0f;
            e.flags = 0u;
            bool same = wo.z * wi.z > 0.0f;
            Spec<N> f;
            float p;
            if (w_sheen > 0.0f) {
                sh.eval_local(wo, wi, f, p);
                if (same) {
                    e.f = e.f + f * acos_i;
                    e.pdf += p * w_sheen;
                }
                e.flags |= kFlagGlossyRefl;
            }
            if (w_coat > 0.0f) {
                mf[2].eval_local(wo, wi, luts, f, p);
                if (same) {
                    e.f = e.f + f * acos_i;
                    e.pdf += p * w_coat;
                }
                e.flags |= kFlagGlossyRefl;
            }
            if (w_metal > 0.0f) {
                mf[0].eval_local(wo, wi, luts, f, p);
                if (same) {
                    e.f = e.f + f * acos_i;
                    e.pdf += p * w_metal;
                }
                e.flags |= kFlagGlossyRefl;
            }
            if (has_trans) {
                uint32_t fl;
                dl.eval_local(wo, wi, luts, f, p, fl, eta);
                // Lobe::evaluate's |cos| first, then WeightedLobe::weight (lobe.cpp:686-697).
                e.f = e.f + (f * acos_i) * trans_scale;
                e.pdf += p * w_trans;
                e.flags |= fl;
            }
            if (w_spec > 0.0f) {
                mf[1].eval_local(wo, wi, luts, f, p);
                if (same) {
                    e.f = e.f + f * acos_i;
                    e.pdf += p * w_spec;
                }
                e.flags |= kFlagGlossyRefl;
            }
            if (w_diff > 0.0f) {
                if (same) {
                    e.f = e.f + kd * (kInvPi * acos_i);
                    e.pdf += acos_i * kInvPi * w_diff;
                }
                e.flags |= kFlagDiffRefl;
            }
        } else {
            // BlackBodyLobe (black_body.cpp:32-39): no scattering.
            e.f = Spec<N>::fill(0.0f);
            e.pdf = 1.0f;
            e.flags = kFlagUnset;
        }
        return e;
    }

    __device__ VS_OUTLINE BsdfEval<N> evaluate(f3 wo_w, f3 wi_w, float *eta_out) const {
        f3 wo = frame.to_local(wo_w), wi = frame.to_local(wi_w);
        float eta = 1.0f;
        BsdfEval<N> e = eval_core(wo, wi, eta);
        if (eta_out) *eta_out = eta;
        discard_check(wo_w, wi_w, e);
        return e;
    }

    // Lobe k of the principled lobe set (sheen, coat, metallic, transmission,
    // specular, diffuse) drawing its own direction.
    __device__ __forceinline__ f3 sample_principled_lobe(int k, f3 wo, Sampler &smp, bool &valid) const {
        f3 wi;
        if (k == 0) wi = sh.sample_local(smp.next2());
        else if (k == 1) wi = mf[2].sample_local(wo, smp.next2(), valid);
        else if (k == 2) wi = mf[0].sample_local(wo, smp.next2(), valid);
        else if (k == 3) wi = dl.sample_local(wo, smp, valid);
        else if (k == 4) wi = mf[1].sample_local(wo, smp.next2(), valid);
        else {
            wi = cosine_hemisphere(smp.next2());
            wi.z = wo.z < 0.0f ? -wi.z : wi.z;
        }
        return wi;
    }

    // The direction draws of a scattering material's lobe (set).
    __device__ __forceinline__ f3 sample_dir(f3 wo, Sampler &smp, bool &valid) const {
        f3 wi = wo;
        if (has_mat<M>(kMatDiffuse) && type == kMatDiffuse) {
            wi = cosine_hemisphere(smp.next2());
            wi.z = wo.z < 0.0f ? -wi.z : wi.z;
        } else if (has_mat<M>(kMatMetal) && type == kMatMetal) {
            wi = mf[0].sample_local(wo, smp.next2(), valid);
        } else if (has_mat<M>(kMatGlass) && type == kMatGlass) {
            wi = dl.sample_local(wo, smp, valid);
        } else if (has_mat<M>(kMatSubstrate) && type == kMatSubstrate) {
            if (plastic) wi = plastic_sample(wo, smp, valid);
            else wi = substrate_sample(wo, smp.next2());
        } else if (has_mat<M>(kMatPrincipled) && type == kMatPrincipled) {
            // LobeSet::sample_wi_impl (lobe.cpp:598-627): 1D lobe choice, an
            // unused 2D draw, then the chosen lobe's own draws.
            float uc = smp.next();
            (void)smp.next2();
            int strategy = 0;
            float sum = 0.0f;
            const float ws[6] = {w_sheen, w_coat, w_metal, w_trans, w_spec, w_diff};
            const bool present[6] = {w_sheen > 0.0f, w_coat > 0.0f, w_metal > 0.0f, has_trans, w_spec > 0.0f,
                                     w_diff > 0.0f};
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                if (!present[i]) continue;
                strategy = uc > sum ? i : strategy;
                sum += ws[i];
            }
            wi = sample_principled_lobe(strategy, wo, smp, valid);
        }
        return wi;
    }

    __device__ VS_OUTLINE BsdfSample<N> sample(f3 wo_w, Sampler &smp) const {
        BsdfSample<N> bs;
        bs.eta = 1.0f;
        const bool scatters = (has_mat<M>(kMatDiffuse) && type == kMatDiffuse) ||
                              (has_mat<M>(kMatMetal) && type == kMatMetal) ||
                              (has_mat<M>(kMatGlass) && type == kMatGlass) ||
                              (has_mat<M>(kMatSubstrate) && type == kMatSubstrate) ||
                              (has_mat<M>(kMatPrincipled) && type == kMatPrincipled);
        if (!scatters) {
            bs.wi = wo_w;
            bs.eval.f = Spec<N>::fill(0.0f);
            bs.eval.pdf = 1.0f;
            bs.eval.flags = kFlagDiffRefl;
            return bs;
        }
        bool valid = true;
        const f3 wi = sample_dir(frame.to_local(wo_w), smp, valid);
        bs.wi = frame.to_world(wi);
        bs.eval = evaluate(wo_w, bs.wi, &bs.eta);
        if (!valid) bs.eval.pdf = 0.0f;
        return bs;
    }
};

// Material::create_evaluator for the in-scope plugins.  The lobe parameters
// come from the 64-byte material record written by the scene loader.
template <int N, uint32_t M = kAllMaterials>
__device__ VS_OUTLINE Bsdf<N, M> make_bsdf(const DeviceScene &s, const Material &m, const Frame &frame, f3 ng, f3 wo,
                                f2 uv, const Wavelengths<N> &wl) {
    Bsdf<N, M> b;
    b.type = m.type;
    b.frame = frame;
    b.ng = ng;
    b.luts = s.luts;
    b.dispersive = (m.flags & kMatFlagDispersive) != 0u && !is_rgb(wl);
    b.w_sheen = b.w_coat = b.w_metal = b.w_trans = b.w_spec = b.w_diff = 0.0f;
    b.plastic = false;
    b.has_trans = false;
    b.trans_scale = 0.0f;
    if (has_mat<M>(kMatDiffuse) && m.type == kMatDiffuse) {
        b.kd = colour_spectrum<N>(s, m, uv, wl);
    } else if (has_mat<M>(kMatMetal) && m.type == kMatMetal) {
        // MetalMaterial::create_lobe_set (metal.cpp:137-156).
        MfLobe<N> &l = b.mf[0];
        l.ax = m.p[0];
        l.ay = m.p[1];
        l.compensate = true;
        l.eta0 = 1.0f;
        if (m.flags & kMatFlagConstantFresnel) {
            // MirrorMaterial::create_lobe_set (mirror.cpp:59-74): FresnelConstant, kr = colour.
            l.fresnel = kFresnelConstant;
            l.kr = colour_spectrum<N>(s, m, uv, wl);
        } else if (m.flags & kMatFlagF82) {
            // MetallicMaterial::create_lobe_set (metallic.cpp:42-60): kr =
            // colour, FresnelF82Tint with F0 = colour and init_from_F82(edge
            // tint) (fresnel.h:114-120).
            l.fresnel = kFresnelF82;
            l.kr = colour_spectrum<N>(s, m, uv, wl);
            const Spec<N> edge = albedo_spectrum<N>(m.p + 2, wl);
            const float f = 6.0f / 7.0f;
            const float f5 = f * f * f * f * f;
#pragma unroll
            for (int i = 0; i < N; ++i) {
                l.fa.v[i] = l.kr.v[i];
                const float fs = l.kr.v[i] + f5 * (1.0f - l.kr.v[i]);
                l.fb.v[i] = fs * (7.0f / (f5 * f)) * (1.0f - edge.v[i]);
            }
        } else {
            l.fresnel = kFresnelConductor;
            l.kr = Spec<N>::fill(1.0f);
            const float *eta = s.spd + m.spd0;
            const float *k = s.spd + m.spd1;
#pragma unroll
            for (int i = 0; i < N; ++i) {
                l.fa.v[i] = spd_eval(eta + 1, static_cast<int>(eta[0]), fabsf(wl.lambda[i]));
                l.fb.v[i] = spd_eval(k + 1, static_cast<int>(k[0]), fabsf(wl.lambda[i]));
            }
        }
    } else if (has_mat<M>(kMatGlass) && m.type == kMatGlass) {
        // GlassMaterial::create_lobe_set (glass.cpp:240-257).
        DielLobe<N> &d = b.dl;
        d.ax = m.p[0];
        d.ay = m.p[1];
        d.kt = colour_spectrum<N>(s, m, uv, wl);
        d.compensate = true;
        d.schlick = false;
        bool front = dot(wo, ng) > 0.0f;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            // RGB transport reads the curve at the first channel's wavelength
            // for every channel (GlassMaterial::init_ior, glass.cpp:224-228).
            const float lam = is_rgb(wl) ? -wl.lambda[0] : wl.lambda[i];
            float ior = m.spd0 != kInvalid ? spd_eval(s.spd + m.spd0 + 1, static_cast<int>(s.spd[m.spd0]), lam)
                                           : m.p[2];
            d.eta.v[i] = front ? ior : 1.0f / ior;
        }
    } else if (has_mat<M>(kMatSubstrate) && m.type == kMatSubstrate) {
        // SubstrateMaterial::create_lobe_set (substrate.cpp:126-148);
        // PlasticMaterial::create_lobe_set (plastic.cpp:105-129).
        b.kd = colour_spectrum<N>(s, m, uv, wl);
        b.ks = albedo_spectrum<N>(m.p + 2, wl);
        b.mf[0].ax = m.p[0];
        b.mf[0].ay = m.p[1];
        b.plastic = (m.flags & kMatFlagPlastic) != 0u;
        if (b.plastic) {
            b.mf[0].fresnel = kFresnelSchlick;
            b.mf[0].eta0 = m.p[5];
            b.mf[0].compensate = false;
            b.mf[0].kr = Spec<N>::fill(1.0f);
            const float f0 = schlick_F0_from_ior(m.p[5]);
#pragma unroll
            for (int i = 0; i < N; ++i) b.mf[0].fa.v[i] = f0 * b.ks.v[i];
        }
    } else if (has_mat<M>(kMatPrincipled) && m.type == kMatPrincipled) {
        // PrincipledBSDF::create_lobe_set (principled_bsdf.cpp:352-461): the
        // lobes in the reference's order, each layer's albedo taking its share
        // of the weight left for the layers below (layering_weight, :209-214).
        float ax = m.p[0], ay = m.p[1];
        float metallic_param = m.p[2];
        float ior = m.p[3];
        Spec<N> color = colour_spectrum<N>(s, m, uv, wl);
        const float tint_coef[3] = {m.p[4], m.p[5], m.p[6]};
        Spec<N> tint = albedo_spectrum<N>(tint_coef, wl);
        float cos_theta = dot(wo, ng);
        float front = cos_theta > 0.0f ? 1.0f : 0.0f;
        Spec<N> weight = Spec<N>::fill(1.0f);
        float sw_sheen = 0.0f, sw_coat = 0.0f, sw_metal = 0.0f, sw_trans = 0.0f, sw_spec = 0.0f, sw_diff = 0.0f;
        // The sheen / coat / transmission parameter block (zero weights without one).
        const float *xp = m.spd0 != kInvalid ? s.spd + m.spd0 + 1 : nullptr;
        auto layer = [&](const Spec<N> &alb) {
            float mx = -3.402823466e+38f;
#pragma unroll
            for (int i = 0; i < N; ++i) mx = fmaxf(mx, safe_div(alb.v[i], weight.v[i]));
            weight = weight * clampf(1.0f - mx, 0.0f, 1.0f);
        };
        if (xp && xp[0] != 0.0f) {
            // SheenLTC (principled_bsdf.cpp:372-383).
            const float sheen_w = xp[0] * front;
            const float c0 = lut_sample2c(s.luts + kLutSheen, 4, 0, cos_theta, xp[1]);
            const float c1 = lut_sample2c(s.luts + kLutSheen, 4, 1, cos_theta, xp[1]);
            const float c2 = lut_sample2c(s.luts + kLutSheen, 4, 2, cos_theta, xp[1]);
            b.sh.a = c0;
            b.sh.b = c1;
            b.sh.tint = albedo_spectrum<N>(xp + 2, wl) * sheen_w * weight * c2;
            sw_sheen = avg(b.sh.tint);
            layer(b.sh.tint);
        }
        if (xp && xp[5] != 0.0f) {
            // CoatLobe (principled_bsdf.cpp:384-400): GGX reflection with
            // alpha = roughness^2 and a dielectric Fresnel; albedo from its table.
            MfLobe<N> &l = b.mf[2];
            const float cc_w = xp[5] * front;
            float cc_r = clampf(xp[6], 0.0001f, 1.0f);
            cc_r = cc_r * cc_r;
            l.ax = l.ay = cc_r;
            l.fresnel = kFresnelDielectric;
            l.compensate = false;
            l.eta0 = xp[7];
            l.kr = weight * cc_w * albedo_spectrum<N>(xp + 8, wl);
            const float x = sqrtf(sqrtf(cc_r * cc_r));
            const float z = (xp[7] - kCoatIorLower) / (kCoatIorUpper - kCoatIorLower);
            const float sc = lut_sample3(s.luts + kLutCoat, 1, 0, x, cos_theta, z);
            const Spec<N> alb = l.kr * sc;
            sw_coat = avg(alb);
            layer(alb);
        }
        // Metallic: F82 tint (F0 = colour, F82 = specular tint).
        float metallic = metallic_param * front;
        {
            MfLobe<N> &l = b.mf[0];
            l.ax = ax;
            l.ay = ay;
            l.fresnel = kFresnelF82;
            l.compensate = true;
            l.kr = weight * metallic;
            const float f = 6.0f / 7.0f;
            const float f5 = f * f * f * f * f;
#pragma unroll
            for (int i = 0; i < N; ++i) {
                l.fa.v[i] = color.v[i];
                float fs = color.v[i] + f5 * (1.0f - color.v[i]);
                l.fb.v[i] = fs * (7.0f / (f5 * f)) * (1.0f - tint.v[i]);
            }
            l.eta0 = 1.0f;
            sw_metal = metallic * avg(weight);
            weight = weight * (1.0f - metallic);
        }
        if (xp && xp[11] != 0.0f) {
            // Transmission (principled_bsdf.cpp:415-428): a compensated
            // DielectricLobe with FresnelSchlick (F0 = schlick_F0(eta) * tint),
            // kt = colour, weighted in f and in sampling by the mean of
            // transmission weight * layer weight.
            const float trans_w = xp[11];
            DielLobe<N> &d = b.dl;
            d.ax = ax;
            d.ay = ay;
            d.kt = color;
            d.compensate = true;
            d.schlick = true;
            const float eta = cos_theta > 0.0f ? ior : 1.0f / ior;
            d.eta = Spec<N>::fill(eta);
            d.f0 = tint * schlick_F0_from_ior(eta);
            const Spec<N> tw = weight * trans_w;
            sw_trans = avg(tw);
            b.trans_scale = sw_trans;
            b.has_trans = true;
            weight = weight * (1.0f - trans_w);
        }
        // Specular: Schlick with F0 = schlick(ior) * tint; albedo from its table.
        {
            MfLobe<N> &l = b.mf[1];
            l.ax = ax;
            l.ay = ay;
            l.fresnel = kFresnelSchlick;
            l.compensate = false;
            l.kr = weight;
            float f0 = schlick_F0_from_ior(ior);
            l.fa = tint * f0;
            l.eta0 = ior;
            float x = sqrtf(sqrtf(ax * ay));
            float z = sqrtf(fabsf((ior - 1.0f) / (ior + 1.0f)));
            float sl = lut_sample3(s.luts + kLutSpecular, 1, 0, x, cos_theta, z);
            Spec<N> alb;
#pragma unroll
            for (int i = 0; i < N; ++i) alb.v[i] = (l.fa.v[i] + sl * (1.0f - l.fa.v[i])) * weight.v[i];
            sw_spec = avg(alb);
            layer(alb);
        }
        // Diffuse.
        b.kd = color * weight * front;
        sw_diff = avg(b.kd);
        // LobeSet::normalize_sampled_weight (lobe.cpp:483-492).
        float sum = sw_sheen + sw_coat + sw_metal + sw_trans + sw_spec + sw_diff;
        b.w_sheen = sw_sheen / sum;
        b.w_coat = sw_coat / sum;
        b.w_metal = sw_metal / sum;
        b.w_trans = b.has_trans ? sw_trans / sum : 0.0f;
        b.w_spec = sw_spec / sum;
        b.w_diff = sw_diff / sum;
    }
    return b;
}

// MixMaterial / AddMaterial (mix.cpp:62-68, add.cpp:56-59): LobeSet::create_mix
// / create_add (lobe.cpp:495-521) over the two materials' lobe sets,
// flattened (LobeSet::flatten, lobe.cpp:533-560, the registry's default): a
// child that is itself a lobe set (principled) contributes its lobes with
// weights and sample weights scaled by its sample weight; a single-lobe child
// contributes its lobe with its weight and sample weight, masked by the lobe's
// hemisphere factor (valid_world_factor, lobe.cpp:35-38; 1 for a dielectric
// lobe).  mix: weights = sample weights = (1 - frac, frac); add: weights 1,
// sample weights normalised to 1/2 (LobeSet::initialize), so a principled
// child of an add counts at half weight.  LobeSet does not override
// is_dispersive, so a mix leaves the secondary wavelengths alone.
template <int N>
struct MixBsdf {
    Bsdf<N> c[2];
    float w[2], sw[2];
    bool dispersive;

    __device__ __forceinline__ static bool multi(const Bsdf<N> &b) { return b.type == kMatPrincipled; }

    __device__ VS_OUTLINE BsdfEval<N> evaluate(f3 wo_w, f3 wi_w, float *eta_out) const {
        const f3 wo = c[0].frame.to_local(wo_w), wi = c[0].frame.to_local(wi_w);
        const bool same = wo.z * wi.z > 0.0f;
        float eta = 1.0f;
        BsdfEval<N> e;
        e.f = Spec<N>::fill(0.0f);
        e.pdf = 0.0f;
        e.flags = 0u;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const BsdfEval<N> ek = c[k].eval_core(wo, wi, eta);
            const bool m = multi(c[k]);
            const float factor = (m || c[k].type == kMatGlass || same) ? 1.0f : 0.0f;
            e.f = e.f + ek.f * ((m ? sw[k] : w[k]) * factor);
            e.pdf += ek.pdf * (sw[k] * factor);
            e.flags |= ek.flags;
        }
        if (eta_out) *eta_out = eta;
        c[0].discard_check(wo_w, wi_w, e);
        return e;
    }

    // LobeSet::sample_wi_impl (lobe.cpp:598-627) over the flattened lobes.
    __device__ VS_OUTLINE BsdfSample<N> sample(f3 wo_w, Sampler &smp) const {
        const f3 wo = c[0].frame.to_local(wo_w);
        const float uc = smp.next();
        (void)smp.next2();
        int child = 0, lobe = -1;
        float sum = 0.0f;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const Bsdf<N> &b = c[k];
            if (multi(b)) {
                const float ws[6] = {b.w_sheen, b.w_coat, b.w_metal, b.w_trans, b.w_spec, b.w_diff};
                const bool present[6] = {b.w_sheen > 0.0f, b.w_coat > 0.0f, b.w_metal > 0.0f, b.has_trans,
                                         b.w_spec > 0.0f, b.w_diff > 0.0f};
#pragma unroll
                for (int i = 0; i < 6; ++i) {
                    if (!present[i]) continue;
                    if (uc > sum) {
                        child = k;
                        lobe = i;
                    }
                    sum += ws[i] * sw[k];
                }
            } else {
                if (uc > sum) {
                    child = k;
                    lobe = -1;
                }
                sum += sw[k];
            }
        }
        bool valid = true;
        const Bsdf<N> &b = c[child];
        const f3 wi = lobe < 0 ? b.sample_dir(wo, smp, valid) : b.sample_principled_lobe(lobe, wo, smp, valid);
        BsdfSample<N> bs;
        bs.eta = 1.0f;
        bs.wi = c[0].frame.to_world(wi);
        bs.eval = evaluate(wo_w, bs.wi, &bs.eta);
        if (!valid) bs.eval.pdf = 0.0f;
        return bs;
    }
};

template <int N>
__device__ VS_OUTLINE MixBsdf<N> make_mix_bsdf(const DeviceScene &s, const Material &m, const Frame &frame, f3 ng,
                                              f3 wo, f2 uv, const Wavelengths<N> &wl) {
    MixBsdf<N> r;
    r.c[0] = make_bsdf<N>(s, s.materials[m.spd0], frame, ng, wo, uv, wl);
    r.c[1] = make_bsdf<N>(s, s.materials[m.spd1], frame, ng, wo, uv, wl);
    if (m.flags & kMatFlagAdd) {
        r.w[0] = r.w[1] = 1.0f;
        r.sw[0] = r.sw[1] = 0.5f;
    } else {
        r.w[0] = r.sw[0] = 1.0f - m.p[0];
        r.w[1] = r.sw[1] = m.p[0];
    }
    r.dispersive = false;
    return r;
}

// The BSDF type path shading builds for a material mask: the mix class gets
// the composite, every other mask the one-material Bsdf.
constexpr uint32_t kMixMask = 1u << kMatMix;
template <int N, uint32_t M>
struct ShadeBsdf {
    using type = Bsdf<N, M>;
    __device__ __forceinline__ static type make(const DeviceScene &s, const Material &m, const Frame &frame, f3 ng,
                                                f3 wo, f2 uv, const Wavelengths<N> &wl) {
        return make_bsdf<N, M>(s, m, frame, ng, wo, uv, wl);
    }
};
template <int N>
struct ShadeBsdf<N, kMixMask> {
    using type = MixBsdf<N>;
    __device__ __forceinline__ static type make(const DeviceScene &s, const Material &m, const Frame &frame, f3 ng,
                                                f3 wo, f2 uv, const Wavelengths<N> &wl) {
        return make_mix_bsdf<N>(s, m, frame, ng, wo, uv, wl);
    }
};

}  // namespace vs

// BSDFs of the in-scope material plugins, evaluated and sampled in world space
// the way MaterialEvaluator does with individual shading normals
// (src/base/scattering/material.cpp:132-184): each lobe works in its local
// frame, multiplies f by |cos theta_i|, and the evaluator zeroes the pdf when
// wi and wo lie on sides of the geometric normal that contradict the lobe's
// reflection/transmission flag.
#pragma once

#include "vs_device.cuh"

namespace vs {

// BxDFFlag (src/base/sample.h:24-49).
constexpr uint32_t kFlagUnset = 1u;
constexpr uint32_t kFlagReflection = 1u << 1;
constexpr uint32_t kFlagTransmission = 1u << 2;
constexpr uint32_t kFlagDiffuse = 1u << 3;
constexpr uint32_t kFlagGlossy = 1u << 4;
constexpr uint32_t kFlagSpecular = 1u << 5;
constexpr uint32_t kFlagDiffRefl = kFlagDiffuse | kFlagReflection;

template <int N>
struct BsdfEval {
    Spec<N> f;
    float pdf[N];  // scatter pdf per wavelength; only pdf[0] is used unless dispersive
    uint32_t flags;
    __device__ __forceinline__ bool valid(bool per_lambda) const {
        if (!per_lambda) return pdf[0] > 0.0f;
        bool ok = true;
#pragma unroll
        for (int i = 0; i < N; ++i) ok = ok && (pdf[i] > 0.0f);
        return ok;
    }
    __device__ __forceinline__ Spec<N> throughput(bool per_lambda) const {
        Spec<N> r;
#pragma unroll
        for (int i = 0; i < N; ++i) r.v[i] = f.v[i] / (per_lambda ? pdf[i] : pdf[0]);
        return r;
    }
    __device__ __forceinline__ void set_pdf(float p) {
#pragma unroll
        for (int i = 0; i < N; ++i) pdf[i] = p;
    }
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
    float r = sqrtf(u.x);
    float theta = k2Pi * u.y;
    float dx = r * cosf(theta), dy = r * sinf(theta);
    float z = sqrtf(fmaxf(0.0f, 1.0f - dx * dx - dy * dy));
    return {dx, dy, z};
}

__device__ __forceinline__ bool same_hemisphere_world(f3 a, f3 b, f3 n) { return dot(a, n) * dot(b, n) > 0.0f; }

template <int N>
struct Bsdf {
    uint32_t type;
    Frame frame;
    f3 ng;
    Spec<N> kr;
    bool dispersive;

    // Zero the pdf of a sample whose geometric side contradicts its flag
    // (MaterialEvaluator::evaluate, material.cpp:137-147).
    __device__ __forceinline__ void discard_check(f3 wo, f3 wi, BsdfEval<N> &e) const {
        bool same = same_hemisphere_world(wo, wi, ng);
        bool trans = (e.flags & kFlagTransmission) != 0u;
        if (same == trans) e.set_pdf(0.0f);
    }

    __device__ __forceinline__ BsdfEval<N> evaluate(f3 wo_w, f3 wi_w, const Wavelengths<N> &) const {
        BsdfEval<N> e;
        f3 wo = frame.to_local(wo_w), wi = frame.to_local(wi_w);
        if (type == kMatDiffuse) {
            // DiffuseLobe -> LambertReflection::safe_evaluate (bxdf.cpp:30-43).
            bool s = wo.z * wi.z > 0.0f;
            float acos_i = fabsf(wi.z);
            e.f = s ? kr * (kInvPi * acos_i) : Spec<N>::fill(0.0f);
            e.set_pdf(s ? acos_i * kInvPi : 0.0f);
            e.flags = kFlagDiffRefl;
        } else {
            // BlackBodyLobe (black_body.cpp:32-39): no scattering.
            e.f = Spec<N>::fill(0.0f);
            e.set_pdf(1.0f);
            e.flags = kFlagUnset;
        }
        discard_check(wo_w, wi_w, e);
        return e;
    }

    __device__ __forceinline__ BsdfSample<N> sample(f3 wo_w, Sampler &smp, const Wavelengths<N> &wl) const {
        BsdfSample<N> bs;
        bs.eta = 1.0f;
        if (type == kMatDiffuse) {
            f2 u = smp.next2();
            f3 wo = frame.to_local(wo_w);
            f3 wi = cosine_hemisphere(u);
            wi.z = wo.z < 0.0f ? -wi.z : wi.z;
            bs.wi = frame.to_world(wi);
            bs.eval = evaluate(wo_w, bs.wi, wl);
        } else {
            bs.wi = wo_w;
            bs.eval.f = Spec<N>::fill(0.0f);
            bs.eval.set_pdf(1.0f);
            bs.eval.flags = kFlagDiffRefl;
        }
        return bs;
    }
};

template <int N>
__device__ __forceinline__ Bsdf<N> make_bsdf(const DeviceScene &s, const Material &m, const Frame &frame, f3 ng,
                                             f3 wo, const Wavelengths<N> &wl) {
    Bsdf<N> b;
    b.type = m.type;
    b.frame = frame;
    b.ng = ng;
    b.dispersive = (m.flags & kMatFlagDispersive) != 0u;
    if (m.type == kMatDiffuse) b.kr = albedo_spectrum<N>(m.coef, wl);
    else b.kr = Spec<N>::fill(0.0f);
    return b;
}

}  // namespace vs

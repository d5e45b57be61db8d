// Device-side building blocks of the spectral path tracer for sm_100a:
// samplers, hero wavelengths, compressed BVH8 traversal, surface interaction,
// area-light sampling, BSDFs and the per-path integrator loop.
//
// Each function cites the reference routine whose semantics it restates.
#pragma once

#include "vs_math.h"
#include "vs_scene.h"
#include "vs_spectral.h"
#include "vs_devscene.h"
#include <cuda_runtime.h>

// Large device functions called from several places.  They are inlined:
// on B200 that measured 10-17% faster than calls in the path-tracing
// megakernel and 4% faster in the ReSTIR kernels, whose out-of-line stack
// frames spilled through L2 to HBM.  Define VS_OUTLINE as __noinline__ to
// build them out of line.
#ifndef VS_OUTLINE
#define VS_OUTLINE __forceinline__
#endif

namespace vs {

// ---------------------------------------------------------------------------
// Constant tables: CIE X/Y/Z and D65 downsampled to every 5th nm (94 entries,
// src/base/color/spd.cpp:31-38,96-110) and the CIE Y integral (:14-23).
// ---------------------------------------------------------------------------
struct SpectralConsts {
    float cie_x[kSpd5Count];
    float cie_y[kSpd5Count];
    float cie_z[kSpd5Count];
    float d65[kSpd5Count];
    float inv_cie_y_integral;
};
// Internal linkage: every translation unit that launches kernels reading it
// fills its own copy with upload_spectral_consts_tu().
static __constant__ SpectralConsts c_spec;

static inline cudaError_t upload_spectral_consts_tu(const float *x, const float *y, const float *z, const float *d65,
                                                    float y_integral) {
    SpectralConsts c;
    for (int i = 0; i < kSpd5Count; ++i) {
        c.cie_x[i] = x[i];
        c.cie_y[i] = y[i];
        c.cie_z[i] = z[i];
        c.d65[i] = d65[i];
    }
    c.inv_cie_y_integral = 1.0f / y_integral;
    return cudaMemcpyToSymbol(c_spec, &c, sizeof(c));
}

// ---------------------------------------------------------------------------
// Samplers.  IndependentSampler (src/render_core/samplers/independent.cpp:24-42)
// seeds with tea(tea(px, py), tea(sample, dim)) (src/math/util.h:13-24, 4
// rounds) and draws with a 24-bit LCG (:27-33).  The PCG option draws from
// PCG32 (O'Neill 2014, XSH-RR output) seeded from the same TEA hash and a seed.
// ---------------------------------------------------------------------------
VS_HD uint32_t tea4(uint32_t v0, uint32_t v1) {
    uint32_t s0 = 0;
#pragma unroll
    for (int n = 0; n < 4; ++n) {
        s0 += 0x9e3779b9u;
        v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + s0) ^ ((v1 >> 5) + 0xc8013ea4u);
        v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + s0) ^ ((v0 >> 5) + 0x7e95761eu);
    }
    return v0;
}

struct Sampler {
    uint64_t state;  // LCG state (low 32 bits) or the 64-bit PCG32 state
    uint32_t kind;
    uint32_t seed;   // PCG32 stream selector: increment (seed << 1) | 1
    VS_HD void start(uint32_t px, uint32_t py, uint32_t sample, uint32_t dim, uint32_t k, uint32_t sd) {
        kind = k;
        seed = sd;
        uint32_t s = tea4(tea4(px, py), tea4(sample, dim));
        if (kind == kSamplerIndependent) {
            state = s;
        } else {
            // PCG32 seeding (pcg32_srandom_r): state 0, one step, add the
            // initial state (the TEA hash), one more step.
            const uint64_t inc = (static_cast<uint64_t>(seed) << 1u) | 1u;
            state = inc;
            state += s;
            state = state * 6364136223846793005ull + inc;
        }
    }
    VS_HD float next() {
        if (kind == kSamplerIndependent) {
            uint32_t s = static_cast<uint32_t>(state);
            s = 1664525u * s + 1013904223u;
            state = s;
            return static_cast<float>(s & 0x00ffffffu) * (1.0f / 16777216.0f);
        }
        // PCG32 step and XSH-RR output; the top 24 bits make the float.
        const uint64_t old = state;
        state = old * 6364136223846793005ull + ((static_cast<uint64_t>(seed) << 1u) | 1u);
        const uint32_t xorshifted = static_cast<uint32_t>(((old >> 18u) ^ old) >> 27u);
        const uint32_t rot = static_cast<uint32_t>(old >> 59u);
        const uint32_t r = (xorshifted >> rot) | (xorshifted << ((32u - rot) & 31u));
        return static_cast<float>(r >> 8) * (1.0f / 16777216.0f);
    }
    VS_HD f2 next2() {
        float a = next();
        float b = next();
        return {a, b};
    }
};

// ---------------------------------------------------------------------------
// Spectra: N hero wavelengths per path.
// ---------------------------------------------------------------------------
template <int N>
struct Spec {
    float v[N];
    __device__ __forceinline__ static Spec fill(float s) {
        Spec r;
#pragma unroll
        for (int i = 0; i < N; ++i) r.v[i] = s;
        return r;
    }
    __device__ __forceinline__ float max() const {
        float m = v[0];
#pragma unroll
        for (int i = 1; i < N; ++i) m = fmaxf(m, v[i]);
        return m;
    }
    __device__ __forceinline__ bool all_zero() const {
        bool z = true;
#pragma unroll
        for (int i = 0; i < N; ++i) z = z && (v[i] == 0.0f);
        return z;
    }
};
template <int N>
__device__ __forceinline__ Spec<N> operator*(const Spec<N> &a, const Spec<N> &b) {
    Spec<N> r;
#pragma unroll
    for (int i = 0; i < N; ++i) r.v[i] = a.v[i] * b.v[i];
    return r;
}
template <int N>
__device__ __forceinline__ Spec<N> operator+(const Spec<N> &a, const Spec<N> &b) {
    Spec<N> r;
#pragma unroll
    for (int i = 0; i < N; ++i) r.v[i] = a.v[i] + b.v[i];
    return r;
}
template <int N>
__device__ __forceinline__ Spec<N> operator*(const Spec<N> &a, float s) {
    Spec<N> r;
#pragma unroll
    for (int i = 0; i < N; ++i) r.v[i] = a.v[i] * s;
    return r;
}

template <int N>
struct Wavelengths {
    float lambda[N];
    float pdf[N];
};

// SRGBSpectrum (spectra/srgb.cpp:16-24): three channels at the peak
// wavelengths of the sRGB primaries (the published constant of the ocarina
// module the reference builds on, absent from its tree: unpinned), pdf 1.
// The wavelengths are stored negated: the sign marks RGB transport, so that
// colour decodes pass RGB through and spectral data (conductor and glass
// IOR curves) is read at |lambda|.
template <int N>
__device__ __forceinline__ Wavelengths<N> rgb_wavelengths() {
    Wavelengths<N> w;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        w.lambda[i] = i == 0 ? -602.785f : (i == 1 ? -539.285f : -445.772f);
        w.pdf[i] = 1.0f;
    }
    return w;
}
// RGB transport always has three channels (the loader sets the dimension),
// so the test compiles away for the other widths.
template <int N>
__device__ __forceinline__ bool is_rgb(const Wavelengths<N> &w) {
    if constexpr (N != 3) return false;
    return w.lambda[0] < 0.0f;
}

__device__ __forceinline__ float cie_spd(const float *tab, float lambda) {
    return spd_eval(tab, kSpd5Count, lambda);
}

// HeroWavelengthSpectrum::sample_wavelength (hero.cpp:286-299).
template <int N>
__device__ __forceinline__ Wavelengths<N> sample_wavelengths(float u) {
    Wavelengths<N> w;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        float offset = static_cast<float>(static_cast<uint32_t>(i) * (1.0f / N));
        float up = u + offset;
        up = up - floorf(up);
        float l = sample_visible_wavelength(up);
        w.lambda[i] = l;
        w.pdf[i] = visible_wavelength_pdf(l);
    }
    return w;
}

// HeroWavelengthSpectrum::cie_xyz + xyz_to_linear_srgb (hero.cpp:261-285).
template <int N>
__device__ VS_OUTLINE f3 linear_srgb(const Spec<N> &s, const Wavelengths<N> &w) {
    // SRGBSpectrum::linear_srgb: the channels themselves.
    if (is_rgb(w)) return make3(s.v[0], s.v[N > 1 ? 1 : 0], s.v[N > 2 ? 2 : 0]);
    f3 sum = make3(0.0f);
    int valid = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        float l = w.lambda[i];
        float p = w.pdf[i];
        valid += p > 0.0f ? 1 : 0;
        sum.x += safe_div(cie_spd(c_spec.cie_x, l) * s.v[i], p);
        sum.y += safe_div(cie_spd(c_spec.cie_y, l) * s.v[i], p);
        sum.z += safe_div(cie_spd(c_spec.cie_z, l) * s.v[i], p);
    }
    float factor = 1.0f / (static_cast<float>(valid) * (1.0f / c_spec.inv_cie_y_integral));
    return xyz_to_linear_srgb(sum * factor);
}

// Albedo spectrum of sigmoid coefficients (RGBAlbedoSpectrum, hero.cpp:177-184).
template <int N>
__device__ __forceinline__ Spec<N> albedo_spectrum(const float *c, const Wavelengths<N> &w) {
    Spec<N> r;
    if (is_rgb(w)) {
        // SRGBSpectrum::decode_to_albedo: the colour itself (c holds RGB).
#pragma unroll
        for (int i = 0; i < N; ++i) r.v[i] = c[i < 3 ? i : 2];
        return r;
    }
#pragma unroll
    for (int i = 0; i < N; ++i) r.v[i] = sigmoid_poly(c[0], c[1], c[2], w.lambda[i]);
    return r;
}

// Radiance of an area light (AreaLight::L, area.cpp:91-95; colour decode
// RGBIlluminationSpectrum, hero.cpp:204-219; blackbody emitter is new).
template <int N>
__device__ __forceinline__ Spec<N> emitter_spectrum(const AreaLight &L, const Wavelengths<N> &w) {
    Spec<N> r;
    if (is_rgb(w)) {
        // SRGBSpectrum::decode_to_illumination: the colour times the scale.
#pragma unroll
        for (int i = 0; i < N; ++i) r.v[i] = L.rgb_avg[i < 3 ? i : 2];
        return r;
    }
#pragma unroll
    for (int i = 0; i < N; ++i) {
        float l = w.lambda[i];
        float e;
        if (L.kind == kEmitRGB) {
            e = sigmoid_poly(L.coef[0], L.coef[1], L.coef[2], l) * L.coef[3] * cie_spd(c_spec.d65, l);
        } else {
            e = planck(l, L.coef[0]) * L.coef[1];
        }
        r.v[i] = e * L.scale;
    }
    return r;
}

// ---------------------------------------------------------------------------
// Ray origin offset (Waechter & Binder, "A Fast and Robust Method for Avoiding
// Self-Intersection", Ray Tracing Gems ch. 6): integer ulp nudge along the
// normal away from the origin, plain float nudge near zero.
// ---------------------------------------------------------------------------
VS_HD float offset_component(float p, float n) {
    const float kOrigin = 1.0f / 32.0f;
    const float kFloatScale = 1.0f / 65536.0f;
    const float kIntScale = 256.0f;
    int of = static_cast<int>(kIntScale * n);
    int pi = static_cast<int>(float_bits(p));
    float pn = bits_float(static_cast<uint32_t>(pi + (p < 0.0f ? -of : of)));
    return fabsf(p) < kOrigin ? p + kFloatScale * n : pn;
}
VS_HD f3 offset_ray_origin(f3 p, f3 n) {
    return {offset_component(p.x, n.x), offset_component(p.y, n.y), offset_component(p.z, n.z)};
}

// spawn_ray / spawn_ray_to (src/base/scattering/interaction.h:272-291).
struct Ray {
    f3 o;
    f3 d;
    float tmax;
};
VS_HD Ray spawn_ray(f3 pos, f3 ng, f3 dir) {
    f3 n = dot(ng, dir) > 0.0f ? ng : -ng;
    return {offset_ray_origin(pos, n), dir, 3.402823466e+38f};
}
VS_HD Ray spawn_ray_to(f3 pos, f3 ng, f3 target) {
    f3 dir = target - pos;
    f3 n = dot(ng, dir) > 0.0f ? ng : -ng;
    return {offset_ray_origin(pos, n), dir, 1.0f - kShadowEpsilon};
}

// ---------------------------------------------------------------------------
// Watertight ray/triangle test (Woop, Benthin, Wald, JCGT 2013) written with
// explicitly rounded operations so that it gives bit-identical results on the
// GPU and in the CPU oracle.  Barycentrics: u weights vertex 1, v vertex 2.
// ---------------------------------------------------------------------------
struct RayPre {
    f3 o;
    f3 d;
    f3 inv_d;
    int kx, ky, kz;
    float sx, sy, sz;
    uint32_t oct;  // bit i set when d[i] < 0
};

__device__ __forceinline__ RayPre precompute_ray(f3 o, f3 d) {
    RayPre r;
    r.o = o;
    r.d = d;
    const float tiny = 1e-30f;
    r.inv_d = {1.0f / (fabsf(d.x) > tiny ? d.x : copysignf(tiny, d.x)),
               1.0f / (fabsf(d.y) > tiny ? d.y : copysignf(tiny, d.y)),
               1.0f / (fabsf(d.z) > tiny ? d.z : copysignf(tiny, d.z))};
    float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    int kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    int kx = kz + 1 == 3 ? 0 : kz + 1;
    int ky = kx + 1 == 3 ? 0 : kx + 1;
    if (comp(d, kz) < 0.0f) {
        int t = kx; kx = ky; ky = t;
    }
    r.kx = kx; r.ky = ky; r.kz = kz;
    float dz = comp(d, kz);
    r.sx = __fdiv_rn(comp(d, kx), dz);
    r.sy = __fdiv_rn(comp(d, ky), dz);
    r.sz = __fdiv_rn(1.0f, dz);
    r.oct = (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
    return r;
}

__device__ __forceinline__ float pick(const float4 &v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

// Returns true and fills (t, u, v) when the ray hits the triangle with
// tmin < t < tmax.
__device__ __forceinline__ bool intersect_triangle(const RayPre &r, const float4 &v0, const float4 &v1,
                                                   const float4 &v2, float tmin, float tmax,
                                                   float &t_out, float &u_out, float &v_out) {
    float ax = __fsub_rn(pick(v0, r.kx), comp(r.o, r.kx));
    float ay = __fsub_rn(pick(v0, r.ky), comp(r.o, r.ky));
    float az = __fsub_rn(pick(v0, r.kz), comp(r.o, r.kz));
    float bx = __fsub_rn(pick(v1, r.kx), comp(r.o, r.kx));
    float by = __fsub_rn(pick(v1, r.ky), comp(r.o, r.ky));
    float bz = __fsub_rn(pick(v1, r.kz), comp(r.o, r.kz));
    float cx = __fsub_rn(pick(v2, r.kx), comp(r.o, r.kx));
    float cy = __fsub_rn(pick(v2, r.ky), comp(r.o, r.ky));
    float cz = __fsub_rn(pick(v2, r.kz), comp(r.o, r.kz));
    float Ax = __fsub_rn(ax, __fmul_rn(r.sx, az));
    float Ay = __fsub_rn(ay, __fmul_rn(r.sy, az));
    float Bx = __fsub_rn(bx, __fmul_rn(r.sx, bz));
    float By = __fsub_rn(by, __fmul_rn(r.sy, bz));
    float Cx = __fsub_rn(cx, __fmul_rn(r.sx, cz));
    float Cy = __fsub_rn(cy, __fmul_rn(r.sy, cz));
    float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
    float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
    float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        double CxBy = static_cast<double>(Cx) * static_cast<double>(By);
        double CyBx = static_cast<double>(Cy) * static_cast<double>(Bx);
        U = static_cast<float>(CxBy - CyBx);
        double AxCy = static_cast<double>(Ax) * static_cast<double>(Cy);
        double AyCx = static_cast<double>(Ay) * static_cast<double>(Cx);
        V = static_cast<float>(AxCy - AyCx);
        double BxAy = static_cast<double>(Bx) * static_cast<double>(Ay);
        double ByAx = static_cast<double>(By) * static_cast<double>(Ax);
        W = static_cast<float>(BxAy - ByAx);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    float det = __fadd_rn(__fadd_rn(U, V), W);
    if (det == 0.0f) return false;
    float Az = __fmul_rn(r.sz, az);
    float Bz = __fmul_rn(r.sz, bz);
    float Cz = __fmul_rn(r.sz, cz);
    float T = __fadd_rn(__fadd_rn(__fmul_rn(U, Az), __fmul_rn(V, Bz)), __fmul_rn(W, Cz));
    float t = __fdiv_rn(T, det);
    if (!(t > tmin && t < tmax)) return false;
    t_out = t;
    u_out = __fdiv_rn(V, det);
    v_out = __fdiv_rn(W, det);
    return true;
}

// ---------------------------------------------------------------------------
// Compressed BVH8 traversal (node groups / triangle groups with an ordered hit
// mask, after Ylitie, Karras, Laine, HPG 2017).  Closest hit breaks exact ties
// in t by the lower primitive index, so the result does not depend on the
// traversal order.
// ---------------------------------------------------------------------------
constexpr int kStackSize = 32;
// Relative slack applied to box distances so that box culling is conservative
// with respect to the float triangle test.
constexpr float kBoxSlack = 1.000001f;

// A bound on the float triangle test's error in t for a hit on the triangle
// (a, b, c): 2^-16 of the vertices' largest coordinate distance from the ray
// origin, in units of t (over the ray's dominant direction component).  The
// test's error is absolute, of the order of the vertices' distances, so a
// relative slack alone does not cover hits at tiny t.  Closest-hit culling
// compares boxes against best_t plus this bound, so a box entered within the
// error of the best hit (another triangle at the same t, as on an edge shared
// next to the origin) is still opened.
__device__ __forceinline__ float tri_t_error(const RayPre &r, const float4 &a, const float4 &b, const float4 &c) {
    const float m = fmaxf(fmaxf(fmaxf(fabsf(a.x - r.o.x), fabsf(a.y - r.o.y)), fmaxf(fabsf(a.z - r.o.z), fabsf(b.x - r.o.x))),
                          fmaxf(fmaxf(fabsf(b.y - r.o.y), fabsf(b.z - r.o.z)),
                                fmaxf(fmaxf(fabsf(c.x - r.o.x), fabsf(c.y - r.o.y)), fabsf(c.z - r.o.z))));
    return m * fabsf(r.sz) * (1.0f / 65536.0f);
}

struct NodeHits {
    uint32_t internal_hits;  // bits 24..31: internal children in traversal order
    uint32_t tri_hits;       // bits 0..23: triangles of the leaf children that were hit
};

__device__ __forceinline__ float ubyte(uint32_t w, int i) {
    return static_cast<float>((w >> (8 * i)) & 0xffu);
}

// Tests the 8 children of one node; returns the new node and triangle groups.
__device__ __forceinline__ void intersect_children(const uint4 *nodes, uint32_t node_index, const RayPre &r,
                                                   float tmax, uint2 &node_group, uint2 &tri_group) {
    const uint4 *np = nodes + static_cast<size_t>(node_index) * 5u;
    uint4 w0 = __ldg(np + 0);
    uint4 w1 = __ldg(np + 1);
    uint4 w2 = __ldg(np + 2);
    uint4 w3 = __ldg(np + 3);
    uint4 w4 = __ldg(np + 4);
    float px = __uint_as_float(w0.x), py = __uint_as_float(w0.y), pz = __uint_as_float(w0.z);
    float sx = __uint_as_float((w0.w & 0xffu) << 23);
    float sy = __uint_as_float(((w0.w >> 8) & 0xffu) << 23);
    float sz = __uint_as_float(((w0.w >> 16) & 0xffu) << 23);
    uint32_t imask = w0.w >> 24;
    uint32_t qlox[2] = {w2.x, w2.y}, qloy[2] = {w2.z, w2.w}, qloz[2] = {w3.x, w3.y};
    uint32_t qhix[2] = {w3.z, w3.w}, qhiy[2] = {w4.x, w4.y}, qhiz[2] = {w4.z, w4.w};
    uint32_t meta[2] = {w1.z, w1.w};
    uint32_t ihits = 0, thits = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        int h = c >> 2, b = c & 3;
        uint32_t m = (meta[h] >> (8 * b)) & 0xffu;
        bool internal = (imask >> c) & 1u;
        if (!internal && m == 0u) continue;
        float lox = __fadd_rn(px, __fmul_rn(ubyte(qlox[h], b), sx));
        float loy = __fadd_rn(py, __fmul_rn(ubyte(qloy[h], b), sy));
        float loz = __fadd_rn(pz, __fmul_rn(ubyte(qloz[h], b), sz));
        float hix = __fadd_rn(px, __fmul_rn(ubyte(qhix[h], b), sx));
        float hiy = __fadd_rn(py, __fmul_rn(ubyte(qhiy[h], b), sy));
        float hiz = __fadd_rn(pz, __fmul_rn(ubyte(qhiz[h], b), sz));
        float t0x = (lox - r.o.x) * r.inv_d.x, t1x = (hix - r.o.x) * r.inv_d.x;
        float t0y = (loy - r.o.y) * r.inv_d.y, t1y = (hiy - r.o.y) * r.inv_d.y;
        float t0z = (loz - r.o.z) * r.inv_d.z, t1z = (hiz - r.o.z) * r.inv_d.z;
        float tn = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fmaxf(fminf(t0z, t1z), 0.0f));
        float tf = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fminf(fmaxf(t0z, t1z), tmax));
        if (tn <= tf * kBoxSlack) {
            if (internal) {
                ihits |= 1u << (24u + (static_cast<uint32_t>(c) ^ r.oct));
            } else {
                uint32_t count_bits = m >> 5;
                uint32_t offset = m & 31u;
                thits |= count_bits << offset;
            }
        }
    }
    node_group = make_uint2(w1.x, ihits | imask);
    tri_group = make_uint2(w1.y, thits);
}

__device__ __forceinline__ void count_traversal(const DeviceScene &s, uint32_t nodes, uint32_t tris) {
    if (s.stats) {
        atomicAdd(&s.stats[0], 1ull);
        atomicAdd(&s.stats[1], static_cast<unsigned long long>(nodes));
        atomicAdd(&s.stats[2], static_cast<unsigned long long>(tris));
    }
}

// ---------------------------------------------------------------------------
// Two-level traversal (instancing): the top level is the same BVH8 walk over
// instance boxes; a leaf entry's instance takes the ray into object space
// (world-to-object rows, explicitly rounded so that the oracle gets the same
// bits) and walks its mesh's BVH8.  Hits report global primitive ids (the
// instance's first primitive + the triangle's index in its mesh), and exact t
// ties go to the lower global id as in the one-level walk.
// ---------------------------------------------------------------------------
__device__ __forceinline__ f3 xf_point(const float4 &r0, const float4 &r1, const float4 &r2, f3 p) {
    return {__fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(r0.x, p.x), __fmul_rn(r0.y, p.y)), __fmul_rn(r0.z, p.z)), r0.w),
            __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(r1.x, p.x), __fmul_rn(r1.y, p.y)), __fmul_rn(r1.z, p.z)), r1.w),
            __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(r2.x, p.x), __fmul_rn(r2.y, p.y)), __fmul_rn(r2.z, p.z)), r2.w)};
}
__device__ __forceinline__ f3 xf_vector(const float4 &r0, const float4 &r1, const float4 &r2, f3 v) {
    return {__fadd_rn(__fadd_rn(__fmul_rn(r0.x, v.x), __fmul_rn(r0.y, v.y)), __fmul_rn(r0.z, v.z)),
            __fadd_rn(__fadd_rn(__fmul_rn(r1.x, v.x), __fmul_rn(r1.y, v.y)), __fmul_rn(r1.z, v.z)),
            __fadd_rn(__fadd_rn(__fmul_rn(r2.x, v.x), __fmul_rn(r2.y, v.y)), __fmul_rn(r2.z, v.z))};
}

// The closest hit inside instance `inst` with t below the current best.
static __device__ __noinline__ void instance_closest(const DeviceScene &s, const RayPre &rw, uint32_t inst,
                                                      float tmax, float &best_t, float &best_err, uint32_t &best_prim,
                                                      float &best_u, float &best_v, uint32_t &visits) {
    const float4 *x = s.inst_xf + 4u * inst;
    const float4 r0 = __ldg(x), r1 = __ldg(x + 1), r2 = __ldg(x + 2), meta = __ldg(x + 3);
    const uint32_t first = __float_as_uint(meta.y);
    const RayPre r = precompute_ray(xf_point(r0, r1, r2, rw.o), xf_vector(r0, r1, r2, rw.d));
    uint2 stack[kStackSize];
    int sp = 0;
    uint2 ng = make_uint2(__float_as_uint(meta.x), (1u << (24u + (0u ^ r.oct))) | 1u);
    uint2 tg;
    while (true) {
        {
            uint32_t bit = __ffs(ng.y & 0xff000000u) - 1u;
            ng.y &= ~(1u << bit);
            uint32_t slot = (bit - 24u) ^ r.oct;
            uint32_t child = ng.x + __popc(ng.y & 0xffu & ((1u << slot) - 1u));
            if ((ng.y & 0xff000000u) != 0u && sp < kStackSize) stack[sp++] = ng;
            intersect_children(s.nodes, child, r, (best_t + best_err) * kBoxSlack, ng, tg);
            ++visits;
        }
        while (tg.y & 0x00ffffffu) {
            uint32_t bit = __ffs(tg.y & 0x00ffffffu) - 1u;
            tg.y &= ~(1u << bit);
            const float4 *tp = s.tri_v + static_cast<size_t>(tg.x + bit) * 3u;
            float4 a = __ldg(tp + 0), b = __ldg(tp + 1), c = __ldg(tp + 2);
            float t, u, v;
            float tri_tmax = best_prim == kInvalid ? tmax : best_t * kBoxSlack;
            if (intersect_triangle(r, a, b, c, 0.0f, tri_tmax, t, u, v)) {
                uint32_t prim = first + __float_as_uint(a.w);
                if (t < best_t || (t == best_t && prim < best_prim)) {
                    best_t = t; best_prim = prim; best_u = u; best_v = v;
                    best_err = tri_t_error(r, a, b, c);
                }
            }
        }
        if (ng.y <= 0x00ffffffu) {
            if (sp == 0) break;
            ng = stack[--sp];
        }
    }
}

// Whether the ray hits anything inside instance `inst` with t in (0, tmax).
static __device__ __noinline__ bool instance_any(const DeviceScene &s, const RayPre &rw, uint32_t inst, float tmax,
                                                 uint32_t &visits) {
    const float4 *x = s.inst_xf + 4u * inst;
    const float4 r0 = __ldg(x), r1 = __ldg(x + 1), r2 = __ldg(x + 2), meta = __ldg(x + 3);
    const RayPre r = precompute_ray(xf_point(r0, r1, r2, rw.o), xf_vector(r0, r1, r2, rw.d));
    uint2 stack[kStackSize];
    int sp = 0;
    uint2 ng = make_uint2(__float_as_uint(meta.x), (1u << (24u + (0u ^ r.oct))) | 1u);
    uint2 tg;
    while (true) {
        {
            uint32_t bit = __ffs(ng.y & 0xff000000u) - 1u;
            ng.y &= ~(1u << bit);
            uint32_t slot = (bit - 24u) ^ r.oct;
            uint32_t child = ng.x + __popc(ng.y & 0xffu & ((1u << slot) - 1u));
            if ((ng.y & 0xff000000u) != 0u && sp < kStackSize) stack[sp++] = ng;
            intersect_children(s.nodes, child, r, tmax * kBoxSlack, ng, tg);
            ++visits;
        }
        while (tg.y & 0x00ffffffu) {
            uint32_t bit = __ffs(tg.y & 0x00ffffffu) - 1u;
            tg.y &= ~(1u << bit);
            const float4 *tp = s.tri_v + static_cast<size_t>(tg.x + bit) * 3u;
            float4 a = __ldg(tp + 0), b = __ldg(tp + 1), c = __ldg(tp + 2);
            float t, u, v;
            if (intersect_triangle(r, a, b, c, 0.0f, tmax, t, u, v)) return true;
        }
        if (ng.y <= 0x00ffffffu) {
            if (sp == 0) return false;
            ng = stack[--sp];
        }
    }
}

// Closest hit with t in (0, tmax).  Returns false on a miss.
static __device__ __noinline__ bool trace_closest(const DeviceScene &s, const RayPre &r, float tmax, Hit &hit,
                                           float &t_hit) {
    uint2 stack[kStackSize];
    int sp = 0;
    uint32_t nodes_visited = 0, tris_tested = 0;
    float best_t = tmax, best_err = 0.0f;
    uint32_t best_prim = kInvalid;
    float best_u = 0.0f, best_v = 0.0f;
    // Root as the only internal child (slot 0) of a virtual parent at index 0.
    uint2 ng = make_uint2(0u, (1u << (24u + (0u ^ r.oct))) | 1u);
    uint2 tg;
    // Invariant at the top of the loop: ng holds at least one internal hit.
    while (true) {
        {
            uint32_t bit = __ffs(ng.y & 0xff000000u) - 1u;
            ng.y &= ~(1u << bit);
            uint32_t slot = (bit - 24u) ^ r.oct;
            uint32_t child = ng.x + __popc(ng.y & 0xffu & ((1u << slot) - 1u));
            if ((ng.y & 0xff000000u) != 0u && sp < kStackSize) stack[sp++] = ng;
            intersect_children(s.nodes, child, r, (best_t + best_err) * kBoxSlack, ng, tg);
            ++nodes_visited;
        }
        if (s.two_level) {
            while (tg.y & 0x00ffffffu) {
                uint32_t bit = __ffs(tg.y & 0x00ffffffu) - 1u;
                tg.y &= ~(1u << bit);
                instance_closest(s, r, __ldg(s.tlas_inst + tg.x + bit), tmax, best_t, best_err, best_prim, best_u,
                                 best_v, nodes_visited);
            }
        }
        while (tg.y & 0x00ffffffu) {
            uint32_t bit = __ffs(tg.y & 0x00ffffffu) - 1u;
            tg.y &= ~(1u << bit);
            uint32_t ti = tg.x + bit;
            const float4 *tp = s.tri_v + static_cast<size_t>(ti) * 3u;
            float4 a = __ldg(tp + 0), b = __ldg(tp + 1), c = __ldg(tp + 2);
            float t, u, v;
            ++tris_tested;
            float tri_tmax = best_prim == kInvalid ? tmax : best_t * kBoxSlack;
            if (intersect_triangle(r, a, b, c, 0.0f, tri_tmax, t, u, v)) {
                uint32_t prim = __float_as_uint(a.w);
                if (t < best_t || (t == best_t && prim < best_prim)) {
                    best_t = t; best_prim = prim; best_u = u; best_v = v;
                    best_err = tri_t_error(r, a, b, c);
                }
            }
        }
        if (ng.y <= 0x00ffffffu) {
            if (sp == 0) break;
            ng = stack[--sp];
        }
    }
    count_traversal(s, nodes_visited, tris_tested);
    if (best_prim == kInvalid) return false;
    hit.prim_id = best_prim;
    hit.inst_id = __ldg(&s.prims[best_prim].w);
    hit.u = best_u;
    hit.v = best_v;
    t_hit = best_t;
    return true;
}

// Any hit with t in (0, tmax).
static __device__ __noinline__ bool trace_any(const DeviceScene &s, const RayPre &r, float tmax) {
    uint2 stack[kStackSize];
    int sp = 0;
    uint32_t nodes_visited = 0, tris_tested = 0;
    uint2 ng = make_uint2(0u, (1u << (24u + (0u ^ r.oct))) | 1u);
    uint2 tg;
    // Invariant at the top of the loop: ng holds at least one internal hit.
    while (true) {
        {
            uint32_t bit = __ffs(ng.y & 0xff000000u) - 1u;
            ng.y &= ~(1u << bit);
            uint32_t slot = (bit - 24u) ^ r.oct;
            uint32_t child = ng.x + __popc(ng.y & 0xffu & ((1u << slot) - 1u));
            if ((ng.y & 0xff000000u) != 0u && sp < kStackSize) stack[sp++] = ng;
            intersect_children(s.nodes, child, r, tmax * kBoxSlack, ng, tg);
            ++nodes_visited;
        }
        if (s.two_level) {
            while (tg.y & 0x00ffffffu) {
                uint32_t bit = __ffs(tg.y & 0x00ffffffu) - 1u;
                tg.y &= ~(1u << bit);
                if (instance_any(s, r, __ldg(s.tlas_inst + tg.x + bit), tmax, nodes_visited)) {
                    count_traversal(s, nodes_visited, tris_tested);
                    return true;
                }
            }
        }
        while (tg.y & 0x00ffffffu) {
            uint32_t bit = __ffs(tg.y & 0x00ffffffu) - 1u;
            tg.y &= ~(1u << bit);
            uint32_t ti = tg.x + bit;
            const float4 *tp = s.tri_v + static_cast<size_t>(ti) * 3u;
            float4 a = __ldg(tp + 0), b = __ldg(tp + 1), c = __ldg(tp + 2);
            float t, u, v;
            ++tris_tested;
            if (intersect_triangle(r, a, b, c, 0.0f, tmax, t, u, v)) {
                count_traversal(s, nodes_visited, tris_tested);
                return true;
            }
        }
        if (ng.y <= 0x00ffffffu) {
            if (sp == 0) break;
            ng = stack[--sp];
        }
    }
    count_traversal(s, nodes_visited, tris_tested);
    return false;
}

// Resumable traversal: the node and triangle visits of trace_closest /
// trace_any, one node (with the triangles it hit) per step, so that a warp can
// give a lane whose ray has finished a new ray while the others continue (ray
// replacement).  A ray visits the same nodes and triangles in the same order,
// so it gets the same result.
struct TravState {
    uint2 ng, tg;
    int sp;
    float tmax;
    float best_t;
    float best_err;  // tri_t_error of the best hit
    uint32_t best_prim;
    float best_u, best_v;
};

__device__ __forceinline__ void trav_init(TravState &t, const RayPre &r, float tmax) {
    t.ng = make_uint2(0u, (1u << (24u + (0u ^ r.oct))) | 1u);
    t.tg = make_uint2(0u, 0u);
    t.sp = 0;
    t.tmax = tmax;
    t.best_t = tmax;
    t.best_err = 0.0f;
    t.best_prim = kInvalid;
    t.best_u = 0.0f;
    t.best_v = 0.0f;
}

// Which traversal code a kernel compiles: kLevelsFlat (one world-space BVH8
// only), kLevelsTwo (instanced scenes only) or kLevelsAny (decided per ray
// from the scene: kernels that serve several scenes at once).  Kernels of one
// scene pick their instantiation on the host, so the flat traversal keeps its
// registers.
constexpr int kLevelsFlat = 0, kLevelsTwo = 1, kLevelsAny = 2;

// One step of the closest-hit traversal; true when the traversal has ended
// (the result is in t.best_*).
template <int Levels = kLevelsFlat>
__device__ __forceinline__ bool closest_step(const DeviceScene &s, const RayPre &r, TravState &t, uint2 *stack) {
    {
        uint32_t bit = __ffs(t.ng.y & 0xff000000u) - 1u;
        t.ng.y &= ~(1u << bit);
        uint32_t slot = (bit - 24u) ^ r.oct;
        uint32_t child = t.ng.x + __popc(t.ng.y & 0xffu & ((1u << slot) - 1u));
        if ((t.ng.y & 0xff000000u) != 0u && t.sp < kStackSize) stack[t.sp++] = t.ng;
        intersect_children(s.nodes, child, r, (t.best_t + t.best_err) * kBoxSlack, t.ng, t.tg);
    }
    if (Levels == kLevelsTwo || (Levels == kLevelsAny && s.two_level)) {
        uint32_t visits = 0;
        while (t.tg.y & 0x00ffffffu) {
            uint32_t bit = __ffs(t.tg.y & 0x00ffffffu) - 1u;
            t.tg.y &= ~(1u << bit);
            instance_closest(s, r, __ldg(s.tlas_inst + t.tg.x + bit), t.tmax, t.best_t, t.best_err, t.best_prim,
                             t.best_u, t.best_v, visits);
        }
    }
    while (t.tg.y & 0x00ffffffu) {
        uint32_t bit = __ffs(t.tg.y & 0x00ffffffu) - 1u;
        t.tg.y &= ~(1u << bit);
        uint32_t ti = t.tg.x + bit;
        const float4 *tp = s.tri_v + static_cast<size_t>(ti) * 3u;
        float4 a = __ldg(tp + 0), b = __ldg(tp + 1), c = __ldg(tp + 2);
        float th, u, v;
        float tri_tmax = t.best_prim == kInvalid ? t.tmax : t.best_t * kBoxSlack;
        if (intersect_triangle(r, a, b, c, 0.0f, tri_tmax, th, u, v)) {
            uint32_t prim = __float_as_uint(a.w);
            if (th < t.best_t || (th == t.best_t && prim < t.best_prim)) {
                t.best_t = th;
                t.best_err = tri_t_error(r, a, b, c);
                t.best_prim = prim;
                t.best_u = u;
                t.best_v = v;
            }
        }
    }
    if (t.ng.y <= 0x00ffffffu) {
        if (t.sp == 0) return true;
        t.ng = stack[--t.sp];
    }
    return false;
}

// The hit of a finished closest-hit traversal (inst_id kInvalid: miss).
__device__ __forceinline__ Hit trav_hit(const DeviceScene &s, const TravState &t) {
    if (t.best_prim == kInvalid) return Hit{kInvalid, kInvalid, 0.0f, 0.0f};
    return Hit{__ldg(&s.prims[t.best_prim].w), t.best_prim, t.best_u, t.best_v};
}

// One step of the any-hit traversal; true when it has ended, with `hit` set
// when an intersection was found.
template <int Levels = kLevelsFlat>
__device__ __forceinline__ bool any_step(const DeviceScene &s, const RayPre &r, TravState &t, uint2 *stack,
                                         bool &hit) {
    {
        uint32_t bit = __ffs(t.ng.y & 0xff000000u) - 1u;
        t.ng.y &= ~(1u << bit);
        uint32_t slot = (bit - 24u) ^ r.oct;
        uint32_t child = t.ng.x + __popc(t.ng.y & 0xffu & ((1u << slot) - 1u));
        if ((t.ng.y & 0xff000000u) != 0u && t.sp < kStackSize) stack[t.sp++] = t.ng;
        intersect_children(s.nodes, child, r, t.tmax * kBoxSlack, t.ng, t.tg);
    }
    if (Levels == kLevelsTwo || (Levels == kLevelsAny && s.two_level)) {
        uint32_t visits = 0;
        while (t.tg.y & 0x00ffffffu) {
            uint32_t bit = __ffs(t.tg.y & 0x00ffffffu) - 1u;
            t.tg.y &= ~(1u << bit);
            if (instance_any(s, r, __ldg(s.tlas_inst + t.tg.x + bit), t.tmax, visits)) {
                hit = true;
                return true;
            }
        }
    }
    while (t.tg.y & 0x00ffffffu) {
        uint32_t bit = __ffs(t.tg.y & 0x00ffffffu) - 1u;
        t.tg.y &= ~(1u << bit);
        uint32_t ti = t.tg.x + bit;
        const float4 *tp = s.tri_v + static_cast<size_t>(ti) * 3u;
        float4 a = __ldg(tp + 0), b = __ldg(tp + 1), c = __ldg(tp + 2);
        float th, u, v;
        if (intersect_triangle(r, a, b, c, 0.0f, t.tmax, th, u, v)) {
            hit = true;
            return true;
        }
    }
    if (t.ng.y <= 0x00ffffffu) {
        if (t.sp == 0) {
            hit = false;
            return true;
        }
        t.ng = stack[--t.sp];
    }
    return false;
}

}  // namespace vs

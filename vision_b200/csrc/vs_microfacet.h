// GGX microfacet and Fresnel math in a local shading frame (z = normal),
// shared by the kernels and by the host-side albedo-table precompute.
// Restates src/base/scattering/microfacet.h, microfacet.cpp, fresnel.h and
// src/math/optics.h, src/math/complex.h.
#pragma once

#include "vs_math.h"

namespace vs {

VS_HD f3 reflect_dir(f3 wo, f3 n) { return -wo + n * (2.0f * dot(wo, n)); }

// square_to_disk (src/math/warp.h:20-26).
VS_HD f2 square_to_disk(f2 u) {
    float r = sqrtf(u.x);
    float theta = k2Pi * u.y;
    return {r * cosf(theta), r * sinf(theta)};
}

// GGX normal distribution (microfacet.cpp:12-33).
VS_HD float ggx_D(f3 wh, float ax, float ay) {
    f3 H = {wh.x / ax, wh.y / ay, wh.z};
    float l2 = length_sq(H);
    return kInvPi / (ax * ay * (l2 * l2));
}

// Smith lambda for GGX (microfacet.cpp:40-65).
VS_HD float ggx_lambda(f3 w, float ax, float ay) {
    if (w.z == 0.0f) return 0.0f;
    float t = (sqr(ax * w.x) + sqr(ay * w.y)) / sqr(w.z);
    return 0.5f * (sqrtf(1.0f + t) - 1.0f);
}
VS_HD float ggx_G1(f3 w, float ax, float ay) { return 1.0f / (1.0f + ggx_lambda(w, ax, ay)); }
VS_HD float ggx_G(f3 wo, f3 wi, float ax, float ay) {
    return 1.0f / (1.0f + ggx_lambda(wo, ax, ay) + ggx_lambda(wi, ax, ay));
}

// Visible-normal sampling (Heitz, JCGT 2018; microfacet.cpp:71-92,100-108).
VS_HD f3 ggx_sample_vndf(f3 wo, f2 u, float ax, float ay) {
    bool flip = wo.z < 0.0f;
    f3 Ve = flip ? -wo : wo;
    f3 Vh = normalize(make3(ax * Ve.x, ay * Ve.y, Ve.z));
    float len_sq = Vh.x * Vh.x + Vh.y * Vh.y;
    f3 T1 = len_sq > 1e-7f ? make3(-Vh.y, Vh.x, 0.0f) / sqrtf(len_sq) : make3(1.0f, 0.0f, 0.0f);
    f3 T2 = len_sq > 1e-7f ? cross(Vh, T1) : make3(0.0f, 1.0f, 0.0f);
    f2 t = square_to_disk(u);
    float s = 0.5f * (1.0f + Vh.z);
    float a = safe_sqrt(1.0f - t.x * t.x);
    t.y = a + s * (t.y - a);
    f3 Nh = T1 * t.x + T2 * t.y + Vh * safe_sqrt(1.0f - (t.x * t.x + t.y * t.y));
    f3 Ne = normalize(make3(ax * Nh.x, ay * Nh.y, fmaxf(0.0f, Nh.z)));
    return flip ? -Ne : Ne;
}

// PDF_wh with visible sampling (microfacet.cpp:146-155).
VS_HD float ggx_pdf_wh(f3 wo, f3 wh, float ax, float ay) {
    return ggx_D(wh, ax, ay) * ggx_G1(wo, ax, ay) * fabsf(dot(wo, wh)) / fabsf(wo.z);
}
// PDF_wi_reflection / PDF_wi_transmission (microfacet.h:133-165).
VS_HD float ggx_pdf_reflection(f3 wo, f3 wh, float ax, float ay) {
    return ggx_pdf_wh(wo, wh, ax, ay) / (4.0f * fabsf(dot(wo, wh)));
}
VS_HD float ggx_pdf_transmission(f3 wo, f3 wh, f3 wi, float eta, float ax, float ay) {
    float denom = sqr(dot(wi, wh) * eta + dot(wo, wh));
    return ggx_pdf_wh(wo, wh, ax, ay) * (fabsf(dot(wi, wh)) / denom);
}
// BRDF_div_fr (microfacet.h:167-175) and BTDF_div_ft (microfacet.cpp:160-174).
VS_HD float ggx_brdf(f3 wo, f3 wh, f3 wi, float ax, float ay) {
    return ggx_D(wh, ax, ay) * ggx_G(wo, wi, ax, ay) / fabsf(4.0f * wo.z * wi.z);
}
VS_HD float ggx_btdf(f3 wo, f3 wh, f3 wi, float eta, float ax, float ay, bool radiance) {
    float num = ggx_D(wh, ax, ay) * ggx_G(wo, wi, ax, ay) * fabsf(dot(wi, wh) * dot(wo, wh));
    float denom = sqr(dot(wi, wh) * eta + dot(wo, wh)) * fabsf(wi.z * wo.z);
    float ft = denom == 0.0f ? 0.0f : num / denom;
    return radiance ? ft * (1.0f / (eta * eta)) : ft;
}

// fresnel_dielectric (src/math/optics.h:70-79).
VS_HD float fresnel_dielectric(float abs_cos_i, float eta) {
    float sin2_i = 1.0f - abs_cos_i * abs_cos_i;
    float sin2_t = sin2_i / (eta * eta);
    float cos_t = safe_sqrt(1.0f - sin2_t);
    float r_parl = (eta * abs_cos_i - cos_t) / (eta * abs_cos_i + cos_t);
    float r_perp = (abs_cos_i - eta * cos_t) / (abs_cos_i + eta * cos_t);
    return sin2_t >= 1.0f ? 1.0f : (r_parl * r_parl + r_perp * r_perp) * 0.5f;
}

// fresnel_complex (src/math/optics.h:92-115) with the complex arithmetic of
// src/math/complex.h: eta_c = eta + i k.  Products are unfused (mul_rn), so
// every kernel that inlines the conductor rounds it alike (and as the host).
struct cplx {
    float re, im;
};
VS_HD cplx c_add(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
VS_HD cplx c_sub(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
VS_HD cplx c_mul(cplx a, cplx b) {
    return {mul_rn(a.re, b.re) - mul_rn(a.im, b.im), mul_rn(a.re, b.im) + mul_rn(a.im, b.re)};
}
VS_HD cplx c_div(cplx a, cplx b) {
    float s = 1.0f / (mul_rn(b.re, b.re) + mul_rn(b.im, b.im));
    return {mul_rn(s, mul_rn(a.re, b.re) + mul_rn(a.im, b.im)), mul_rn(s, mul_rn(a.im, b.re) - mul_rn(a.re, b.im))};
}
VS_HD float c_norm(cplx z) { return mul_rn(z.re, z.re) + mul_rn(z.im, z.im); }
VS_HD cplx c_sqrt(cplx z) {
    float n = sqrtf(c_norm(z));
    float t1 = sqrtf(mul_rn(0.5f, n + fabsf(z.re)));
    float t2 = mul_rn(0.5f, z.im) / t1;
    if (n == 0.0f) return {0.0f, 0.0f};
    if (z.re >= 0.0f) return {t1, t2};
    return {fabsf(t2), copysignf(t1, z.im)};
}
VS_HD float fresnel_complex(float cos_i, float eta, float k) {
    cplx e = {eta, k};
    float sin2_i = 1.0f - mul_rn(cos_i, cos_i);
    cplx sin2_t = c_div({sin2_i, 0.0f}, c_mul(e, e));
    cplx cos_t = c_sqrt(c_sub({1.0f, 0.0f}, sin2_t));
    cplx ec = {mul_rn(e.re, cos_i), mul_rn(e.im, cos_i)};
    cplx r_parl = c_div(c_sub(ec, cos_t), c_add(ec, cos_t));
    cplx ect = c_mul(e, cos_t);
    cplx r_perp = c_div(c_sub({cos_i, 0.0f}, ect), c_add({cos_i, 0.0f}, ect));
    return mul_rn(c_norm(r_parl) + c_norm(r_perp), 0.5f);
}

// refract (src/math/optics.h:27-39).
VS_HD bool refract_dir(f3 wi, f3 n, float eta, f3 &wt) {
    float cos_i = dot(n, wi);
    float sin2_i = fmaxf(0.0f, 1.0f - cos_i * cos_i);
    float sin2_t = sin2_i / (eta * eta);
    float cos_t = safe_sqrt(1.0f - sin2_t);
    wt = -wi / eta + n * (cos_i / eta - cos_t);
    return sin2_t < 1.0f;
}

VS_HD float schlick_F0_from_ior(float ior) { return sqr((ior - 1.0f) / (ior + 1.0f)); }
VS_HD float schlick_ior_from_F0(float f0) {
    float s = sqrtf(clampf(f0, 0.0f, 0.99f));
    return (1.0f + s) / (1.0f - s);
}

// Albedo lookup tables of the compensated lobes, addressed like a normalised
// texture with linear filtering and clamp-to-edge: texel i covers
// [i / res, (i + 1) / res] (MaterialLut::sample, material.h:39-41).
constexpr int kLutRes = 32;
VS_HD float lut_coord(float u, int &i0, int &i1) {
    float x = u * kLutRes - 0.5f;
    float fl = floorf(x);
    float f = x - fl;
    int i = static_cast<int>(fl);
    i0 = i < 0 ? 0 : (i > kLutRes - 1 ? kLutRes - 1 : i);
    i1 = i + 1 < 0 ? 0 : (i + 1 > kLutRes - 1 ? kLutRes - 1 : i + 1);
    return f;
}
// 2D table, 1 channel, index [y][x].
VS_HD float lut_sample2(const float *t, float u, float v) {
    int x0, x1, y0, y1;
    float fx = lut_coord(u, x0, x1), fy = lut_coord(v, y0, y1);
    float a = t[y0 * kLutRes + x0] + fx * (t[y0 * kLutRes + x1] - t[y0 * kLutRes + x0]);
    float b = t[y1 * kLutRes + x0] + fx * (t[y1 * kLutRes + x1] - t[y1 * kLutRes + x0]);
    return a + fy * (b - a);
}
// 3D table with `ch` channels per texel, index [z][y][x][c].
VS_HD float lut_sample3(const float *t, int ch, int c, float u, float v, float w) {
    int x0, x1, y0, y1, z0, z1;
    float fx = lut_coord(u, x0, x1), fy = lut_coord(v, y0, y1), fz = lut_coord(w, z0, z1);
    auto at = [&](int x, int y, int z) { return t[((z * kLutRes + y) * kLutRes + x) * ch + c]; };
    float c00 = at(x0, y0, z0) + fx * (at(x1, y0, z0) - at(x0, y0, z0));
    float c10 = at(x0, y1, z0) + fx * (at(x1, y1, z0) - at(x0, y1, z0));
    float c01 = at(x0, y0, z1) + fx * (at(x1, y0, z1) - at(x0, y0, z1));
    float c11 = at(x0, y1, z1) + fx * (at(x1, y1, z1) - at(x0, y1, z1));
    float c0 = c00 + fy * (c10 - c00);
    float c1 = c01 + fy * (c11 - c01);
    return c0 + fz * (c1 - c0);
}

// 2D table with `ch` channels per texel, index [y][x][c].
VS_HD float lut_sample2c(const float *t, int ch, int c, float u, float v) {
    int x0, x1, y0, y1;
    float fx = lut_coord(u, x0, x1), fy = lut_coord(v, y0, y1);
    auto at = [&](int x, int y) { return t[(y * kLutRes + x) * ch + c]; };
    float a = at(x0, y0) + fx * (at(x1, y0) - at(x0, y0));
    float b = at(x0, y1) + fx * (at(x1, y1) - at(x0, y1));
    return a + fy * (b - a);
}

// Offsets of the tables in the concatenated LUT buffer.
constexpr int kLutPureReflection = 0;                             // 32^2, 1 channel
constexpr int kLutDielectric = kLutPureReflection + 32 * 32;        // 32^3, 2 channels
constexpr int kLutDielectricInv = kLutDielectric + 2 * 32 * 32 * 32; // 32^3, 2 channels
constexpr int kLutSpecular = kLutDielectricInv + 2 * 32 * 32 * 32;   // 32^3, 1 channel
constexpr int kLutFloats = kLutSpecular + 32 * 32 * 32;
// The principled BSDF's tables follow the compensation tables in the device
// buffer: the CoatLobe albedo (32^3, 1 channel: roughness ratio, cos theta,
// ior ratio) and the SheenLTC fits (32^2, 4 channels (a, b, scale, 0): cos
// theta, sheen roughness).
constexpr int kLutCoat = kLutFloats;
constexpr int kLutSheen = kLutCoat + 32 * 32 * 32;
constexpr int kLutDeviceFloats = kLutSheen + 32 * 32 * 4;
// CoatLobe's ior range (principled_bsdf.cpp:124-125).
constexpr float kCoatIorLower = 1.003f;
constexpr float kCoatIorUpper = 4.0f;

// Lobe constants (src/base/scattering/lobe.h:24-25,181-185).
constexpr float kAlphaLower = 0.001f;
constexpr float kAlphaUpper = 1.0f;
constexpr float kIorLower = 1.003f;
constexpr float kIorUpper = 5.0f;

}  // namespace vs

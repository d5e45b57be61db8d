// One Monte Carlo sample of the albedo tables of the energy-compensated lobes
// (Lobe::integral_albedo, lobe.cpp:12-26, in importance transport), shared by
// the CPU generator (luts.cpp) and the GPU one (lut_gen.cu) so that both
// evaluate the same estimator:
//   PureReflectionLobe  [y][x]     x: alpha = clamp(x^2, 0.001, 1), y: cos theta_o,
//                                  Fresnel = 1 (lobe.h:346-356, lobe.cpp:189-193)
//   DielectricLobe(Inv) [z][y][x]  x: alpha, y: cos theta_o, z: ior = lerp(z, 1.003, 5)
//                                  (inverted for Inv); channels (total, reflected)
//   SpecularLobe        [z][y][x]  x: alpha, y: cos theta_o, z: ior = schlick_ior(z^4),
//                                  Schlick Fresnel with F0 = 0.04 (principled_bsdf.cpp:164-207)
// A cell's estimate stratifies the microfacet-normal sample on an S x S grid
// with one jitter per cell; sample k = i * S + j sits in stratum (i, j).
#pragma once

#include "vs_microfacet.h"

namespace vs {

enum LutTable : uint32_t { kLutTablePure = 0, kLutTableDiel = 1, kLutTableDielInv = 2, kLutTableSpec = 3 };

// Cells of the four tables in output order (kLutPureReflection ... kLutSpecular).
constexpr uint32_t kLutCells = 32u * 32u + 3u * 32u * 32u * 32u;

VS_HD float lut_hash01(uint32_t a, uint32_t b) {
    uint32_t h = a * 0x9e3779b1u ^ (b + 0x7f4a7c15u) * 0x85ebca6bu;
    h ^= h >> 15;
    h *= 0x2c1b3c6du;
    h ^= h >> 12;
    h *= 0x297a2d39u;
    h ^= h >> 15;
    return static_cast<float>(h >> 8) * (1.0f / 16777216.0f);
}

// The parameters of one table cell.
struct LutCell {
    uint32_t table;
    uint32_t seed;     // hash key of the cell
    uint32_t out;      // index of its first output float
    f3 wo;
    float alpha;
    float eta;         // dielectric: relative IOR; specular: IOR of the Schlick curve
    float f0_real;     // specular: F0 of that IOR
    float jx, jy;      // stratum jitter
};

// Cell `c` in [0, kLutCells): the 2D table first, then the three 3D tables.
VS_HD LutCell lut_cell(uint32_t c) {
    LutCell k;
    uint32_t ix, iy, iz = 0;
    if (c < 1024u) {
        k.table = kLutTablePure;
        ix = c % 32u;
        iy = c / 32u;
        k.seed = iy * 32u + ix;
        k.out = kLutPureReflection + k.seed;
    } else {
        const uint32_t r = c - 1024u;
        k.table = 1u + r / 32768u;
        const uint32_t cell = r % 32768u;
        ix = cell % 32u;
        iy = (cell / 32u) % 32u;
        iz = cell / 1024u;
        if (k.table == kLutTableDiel) {
            k.seed = cell;
            k.out = kLutDielectric + 2u * cell;
        } else if (k.table == kLutTableDielInv) {
            k.seed = cell + 40000u;
            k.out = kLutDielectricInv + 2u * cell;
        } else {
            k.seed = cell + 90000u;
            k.out = kLutSpecular + cell;
        }
    }
    const float x = static_cast<float>(ix) / 31.0f, y = static_cast<float>(iy) / 31.0f;
    const float z = static_cast<float>(iz) / 31.0f;
    k.alpha = clampf(x * x, kAlphaLower, kAlphaUpper);
    const float cw = clampf(y, 1e-4f, 1.0f);
    k.wo = {sqrtf(1.0f - cw * cw), 0.0f, cw};
    k.eta = 1.0f;
    k.f0_real = 0.0f;
    uint32_t h0 = 1u, h1 = 2u;
    if (k.table == kLutTableDiel || k.table == kLutTableDielInv) {
        const float ior = kIorLower + z * (kIorUpper - kIorLower);
        k.eta = k.table == kLutTableDielInv ? 1.0f / ior : ior;
        h0 = 3u;
        h1 = 4u;
    } else if (k.table == kLutTableSpec) {
        k.eta = schlick_ior_from_F0(z * z * z * z);
        k.f0_real = schlick_F0_from_ior(k.eta);
        h0 = 7u;
        h1 = 8u;
    }
    k.jx = lut_hash01(k.seed, h0);
    k.jy = lut_hash01(k.seed, h1);
    return k;
}

// Sample k of an S x S stratification of cell `c`: adds f cos / pdf to
// acc[0] (and the reflected part of a dielectric to acc[1]).
VS_HD void lut_sample(const LutCell &c, uint32_t strata, uint32_t k, double acc[2]) {
    const uint32_t i = k / strata, j = k % strata;
    const float inv = 1.0f / static_cast<float>(strata);
    const f2 u = {(static_cast<float>(i) + c.jx) * inv, (static_cast<float>(j) + c.jy) * inv};
    const f3 wo = c.wo;
    const float a = c.alpha;
    const f3 wh = ggx_sample_vndf(wo, u, a, a);
    if (c.table == kLutTablePure || c.table == kLutTableSpec) {
        const f3 wi = reflect_dir(wo, wh);
        if (!(wo.z * wi.z > 0.0f)) return;
        const f3 h = normalize(wo + wi);
        const f3 hf = h.z < 0.0f ? -h : h;
        float f = ggx_brdf(wo, hf, wi, a, a);
        if (c.table == kLutTableSpec) {
            const float cs = fabsf(dot(wo, hf));
            const float t = clampf((fresnel_dielectric(cs, c.eta) - c.f0_real) / (1.0f - c.f0_real), 0.0f, 1.0f);
            f *= 0.04f + t * (1.0f - 0.04f);
        }
        const float pdf = ggx_pdf_reflection(wo, h, a, a);
        if (pdf > 0.0f) acc[0] += f / pdf * fabsf(wi.z);
        return;
    }
    // Rough dielectric without compensation (DielectricPrecompute::integral_albedo):
    // one more number picks reflection or refraction.
    const float eta = c.eta;
    const float uc = lut_hash01(c.seed * (strata * strata) + k, 6u);
    const float F = fresnel_dielectric(fabsf(dot(wo, wh)), eta);
    f3 wi;
    bool valid;
    if (uc < F) {
        wi = reflect_dir(wo, wh);
        valid = wo.z * wi.z > 0.0f;
    } else {
        valid = refract_dir(wo, wh, eta, wi) && !(wo.z * wi.z > 0.0f);
    }
    if (!valid) return;
    const bool reflect = wo.z * wi.z > 0.0f;
    const float eta_p = reflect ? 1.0f : eta;
    f3 h = normalize(wo + wi * eta_p);
    if (dot(h, wo) < 0.0f) h = -h;
    const float Fe = fresnel_dielectric(fabsf(dot(h, wo)), eta);
    float f, pdf;
    if (reflect) {
        f = ggx_brdf(wo, h, wi, a, a) * Fe;
        pdf = ggx_pdf_reflection(wo, h, a, a) * Fe;
    } else {
        const f3 h2 = normalize(wo + wi * eta);
        f = ggx_btdf(wo, h2, wi, eta, a, a, false) * (1.0f - Fe);
        pdf = ggx_pdf_transmission(wo, h, wi, eta, a, a) * (1.0f - Fe);
    }
    if (!(pdf > 0.0f)) return;
    const float r = f / pdf * fabsf(wi.z);
    acc[0] += r;
    if (reflect) acc[1] += r;
}

// Writes a cell's estimate (1 or 2 floats) from its sums over n samples.
VS_HD void lut_store(const LutCell &c, const double acc[2], uint32_t n, float *out) {
    out[c.out] = static_cast<float>(acc[0] / n);
    if (c.table == kLutTableDiel || c.table == kLutTableDielInv) out[c.out + 1] = static_cast<float>(acc[1] / n);
}

}  // namespace vs

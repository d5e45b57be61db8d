// Albedo tables of the energy-compensated lobes.
//
// The reference ships these as precomputed arrays (precomputed_table.h, made
// by apps/precompute: Material::precompute_lobe, material.h:121-163, 2^21
// Monte Carlo samples per cell).  Rendering uses those values as shipped
// (data/albedo_luts.inc), so compensated lobes match the reference value for
// value.  This file also regenerates the tables from the lobes' own
// definitions with stratified visible-normal sampling, using the same cell
// parameterisation as the reference's from_ratio_* functions:
//   PureReflectionLobe  [y][x]     x: alpha = clamp(x^2, 0.001, 1), y: cos theta_o,
//                                  Fresnel = 1 (lobe.h:346-356, lobe.cpp:189-193)
//   DielectricLobe(Inv) [z][y][x]  x: alpha = clamp(x^2, 0.001, 1), y: cos theta_o,
//                                  z: ior = lerp(z, 1.003, 5) (inverted for Inv);
//                                  channels (total, reflected) (glass.cpp:14-76)
//   SpecularLobe        [z][y][x]  x: alpha, y: cos theta_o, z: ior = schlick_ior(z^4),
//                                  Schlick Fresnel with F0 = 0.04 (principled_bsdf.cpp:164-207)
// Each cell is the estimate E[f cos / pdf] of Lobe::integral_albedo
// (lobe.cpp:12-26) in importance transport.  The regenerated tables are
// cached on disk and exposed for comparison; they differ from the shipped ones
// by up to ~0.03 in cells where the reference's estimate drew its 2D samples
// from consecutive outputs of its 24-bit LCG.
#include "vs_host.h"
#include "vs_microfacet.h"

#include "data/albedo_luts.inc"

#include <atomic>
#include <fstream>
#include <mutex>
#include <thread>

namespace vs {

namespace {

constexpr int kStrata = 32;  // kStrata^2 samples per cell

float hash01(uint32_t a, uint32_t b) {
    uint32_t h = a * 0x9e3779b1u ^ (b + 0x7f4a7c15u) * 0x85ebca6bu;
    h ^= h >> 15;
    h *= 0x2c1b3c6du;
    h ^= h >> 12;
    h *= 0x297a2d39u;
    h ^= h >> 15;
    return static_cast<float>(h >> 8) * (1.0f / 16777216.0f);
}

f3 wo_from_ratio(float y) {
    float c = clampf(y, 1e-4f, 1.0f);
    return {sqrtf(1.0f - c * c), 0.0f, c};
}

// Pure reflection, Fresnel 1: f cos / pdf = G2 / G1 for valid reflections.
float pure_reflection_cell(int ix, int iy) {
    float x = ix / 31.0f, y = iy / 31.0f;
    float a = clampf(x * x, kAlphaLower, kAlphaUpper);
    f3 wo = wo_from_ratio(y);
    double acc = 0.0;
    uint32_t cell = static_cast<uint32_t>(iy * 32 + ix);
    float jx = hash01(cell, 1), jy = hash01(cell, 2);
    for (int i = 0; i < kStrata; ++i)
        for (int j = 0; j < kStrata; ++j) {
            f2 u = {(i + jx) / kStrata, (j + jy) / kStrata};
            f3 wh = ggx_sample_vndf(wo, u, a, a);
            f3 wi = reflect_dir(wo, wh);
            if (!(wo.z * wi.z > 0.0f)) continue;
            f3 h = normalize(wo + wi);
            f3 hf = h.z < 0.0f ? -h : h;
            float f = ggx_brdf(wo, hf, wi, a, a);
            float pdf = ggx_pdf_reflection(wo, h, a, a);
            if (pdf > 0.0f) acc += f / pdf * fabsf(wi.z);
        }
    return static_cast<float>(acc / (kStrata * kStrata));
}

// Rough dielectric without compensation (DielectricPrecompute::integral_albedo).
void dielectric_cell(int ix, int iy, int iz, bool inverse, float out[2]) {
    float x = ix / 31.0f, y = iy / 31.0f, z = iz / 31.0f;
    float a = clampf(x * x, kAlphaLower, kAlphaUpper);
    f3 wo = wo_from_ratio(y);
    float ior = kIorLower + z * (kIorUpper - kIorLower);
    float eta = inverse ? 1.0f / ior : ior;
    double tot = 0.0, refl = 0.0;
    uint32_t cell = static_cast<uint32_t>((iz * 32 + iy) * 32 + ix) + (inverse ? 40000u : 0u);
    float jx = hash01(cell, 3), jy = hash01(cell, 4);
    for (int i = 0; i < kStrata; ++i)
        for (int j = 0; j < kStrata; ++j) {
            f2 u = {(i + jx) / kStrata, (j + jy) / kStrata};
            float uc = hash01(cell * 1024u + static_cast<uint32_t>(i * kStrata + j), 6u);
            f3 wh = ggx_sample_vndf(wo, u, a, a);
            float F = fresnel_dielectric(fabsf(dot(wo, wh)), eta);
            f3 wi;
            bool valid;
            if (uc < F) {
                wi = reflect_dir(wo, wh);
                valid = wo.z * wi.z > 0.0f;
            } else {
                valid = refract_dir(wo, wh, eta, wi) && !(wo.z * wi.z > 0.0f);
            }
            if (!valid) continue;
            bool reflect = wo.z * wi.z > 0.0f;
            float eta_p = reflect ? 1.0f : eta;
            f3 h = normalize(wo + wi * eta_p);
            if (dot(h, wo) < 0.0f) h = -h;
            float Fe = fresnel_dielectric(fabsf(dot(h, wo)), eta);
            float f, pdf;
            if (reflect) {
                f = ggx_brdf(wo, h, wi, a, a) * Fe;
                pdf = ggx_pdf_reflection(wo, h, a, a) * Fe;
            } else {
                f3 h2 = normalize(wo + wi * eta);
                f = ggx_btdf(wo, h2, wi, eta, a, a, false) * (1.0f - Fe);
                pdf = ggx_pdf_transmission(wo, h, wi, eta, a, a) * (1.0f - Fe);
            }
            if (!(pdf > 0.0f)) continue;
            float r = f / pdf * fabsf(wi.z);
            tot += r;
            if (reflect) refl += r;
        }
    out[0] = static_cast<float>(tot / (kStrata * kStrata));
    out[1] = static_cast<float>(refl / (kStrata * kStrata));
}

// Schlick-Fresnel specular lobe (SpecularLobe::create_for_precompute).
float specular_cell(int ix, int iy, int iz) {
    float x = ix / 31.0f, y = iy / 31.0f, z = iz / 31.0f;
    float a = clampf(x * x, kAlphaLower, kAlphaUpper);
    f3 wo = wo_from_ratio(y);
    float ior = schlick_ior_from_F0(z * z * z * z);
    double acc = 0.0;
    uint32_t cell = static_cast<uint32_t>((iz * 32 + iy) * 32 + ix) + 90000u;
    float jx = hash01(cell, 7), jy = hash01(cell, 8);
    float f0_real = schlick_F0_from_ior(ior);
    for (int i = 0; i < kStrata; ++i)
        for (int j = 0; j < kStrata; ++j) {
            f2 u = {(i + jx) / kStrata, (j + jy) / kStrata};
            f3 wh = ggx_sample_vndf(wo, u, a, a);
            f3 wi = reflect_dir(wo, wh);
            if (!(wo.z * wi.z > 0.0f)) continue;
            f3 h = normalize(wo + wi);
            f3 hf = h.z < 0.0f ? -h : h;
            float c = fabsf(dot(wo, hf));
            float t = clampf((fresnel_dielectric(c, ior) - f0_real) / (1.0f - f0_real), 0.0f, 1.0f);
            float F = 0.04f + t * (1.0f - 0.04f);
            float f = ggx_brdf(wo, hf, wi, a, a) * F;
            float pdf = ggx_pdf_reflection(wo, h, a, a);
            if (pdf > 0.0f) acc += f / pdf * fabsf(wi.z);
        }
    return static_cast<float>(acc / (kStrata * kStrata));
}

std::vector<float> build() {
    std::vector<float> t(kLutFloats, 0.0f);
    // Jobs: 32 rows of the 2D table, then one row (32 cells) per (table, z, y).
    std::atomic<int> next{0};
    auto worker = [&]() {
        while (true) {
            int j = next.fetch_add(1);
            if (j >= 32 + 3 * 32 * 32) break;
            if (j < 32) {
                for (int ix = 0; ix < 32; ++ix) t[kLutPureReflection + j * 32 + ix] = pure_reflection_cell(ix, j);
                continue;
            }
            int k = j - 32;
            int table = k / 1024, iz = (k / 32) % 32, iy = k % 32;
            for (int ix = 0; ix < 32; ++ix) {
                int cell = (iz * 32 + iy) * 32 + ix;
                if (table == 0 || table == 1) {
                    float o[2];
                    dielectric_cell(ix, iy, iz, table == 1, o);
                    int base = table == 0 ? kLutDielectric : kLutDielectricInv;
                    t[base + 2 * cell] = o[0];
                    t[base + 2 * cell + 1] = o[1];
                } else {
                    t[kLutSpecular + cell] = specular_cell(ix, iy, iz);
                }
            }
        }
    };
    unsigned nt = std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::thread> th;
    for (unsigned i = 0; i < nt; ++i) th.emplace_back(worker);
    for (auto &x : th) x.join();
    return t;
}

std::mutex g_mutex;
std::vector<float> g_luts;

}  // namespace

const float *microfacet_luts() { return VS_ALBEDO_LUTS; }

const float *regenerate_microfacet_luts(const std::string &cache_path) {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_luts.empty()) return g_luts.data();
    if (!cache_path.empty()) {
        std::ifstream in(cache_path, std::ios::binary);
        if (in) {
            std::vector<float> t(kLutFloats);
            in.read(reinterpret_cast<char *>(t.data()), static_cast<std::streamsize>(t.size() * sizeof(float)));
            if (in.gcount() == static_cast<std::streamsize>(t.size() * sizeof(float))) {
                g_luts = std::move(t);
                return g_luts.data();
            }
        }
    }
    g_luts = build();
    if (!cache_path.empty()) {
        std::string tmp = cache_path + ".tmp";
        std::ofstream out(tmp, std::ios::binary);
        if (out) {
            out.write(reinterpret_cast<const char *>(g_luts.data()), static_cast<std::streamsize>(g_luts.size() * sizeof(float)));
            out.close();
            std::rename(tmp.c_str(), cache_path.c_str());
        }
    }
    return g_luts.data();
}

}  // namespace vs

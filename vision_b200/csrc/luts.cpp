// Albedo tables of the energy-compensated lobes.
//
// The reference ships these as precomputed arrays (precomputed_table.h, made
// by apps/precompute: Material::precompute_lobe, material.h:121-163, 2^21
// Monte Carlo samples per cell).  Rendering uses those values as shipped
// (data/albedo_luts.inc), so compensated lobes match the reference value for
// value.  This file also regenerates the tables from the lobes' own
// definitions with stratified visible-normal sampling, using the same cell
// parameterisation as the reference's from_ratio_* functions (the cells and
// the per-sample estimator are in vs_lut_samples.h, shared with the GPU
// generator in lut_gen.cu).  The regenerated tables are
// cached on disk and exposed for comparison; they differ from the shipped ones
// by up to ~0.03 in cells where the reference's estimate drew its 2D samples
// from consecutive outputs of its 24-bit LCG.
#include "vs_host.h"
#include "vs_microfacet.h"
#include "vs_lut_samples.h"

#include "data/albedo_luts.inc"
#include "data/principled_luts.inc"

#include <atomic>
#include <fstream>
#include <mutex>
#include <thread>

namespace vs {

namespace {

constexpr uint32_t kStrata = 32;  // kStrata^2 samples per cell

std::vector<float> build() {
    std::vector<float> t(kLutFloats, 0.0f);
    // Jobs of 32 cells each, in output order.
    std::atomic<uint32_t> next{0};
    auto worker = [&]() {
        while (true) {
            const uint32_t job = next.fetch_add(1);
            if (job * 32u >= kLutCells) break;
            for (uint32_t c = job * 32u; c < job * 32u + 32u; ++c) {
                const LutCell cell = lut_cell(c);
                double acc[2] = {0.0, 0.0};
                for (uint32_t k = 0; k < kStrata * kStrata; ++k) lut_sample(cell, kStrata, k, acc);
                lut_store(cell, acc, kStrata * kStrata, t.data());
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
const float *coat_lut() { return VS_COAT_LUT; }
const float *sheen_ltc_lut() { return VS_SHEEN_LTC; }

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

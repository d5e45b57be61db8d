// RGB -> spectrum uplift table.
//
// The reference reads a precomputed 3 x 64^3 table of sigmoid-polynomial
// coefficients (srgb2spec.h, used by RGBToSpectrumTable in
// src/render_core/spectra/hero.cpp:51-175).  That table is not part of the
// reference tree, so this file regenerates it with the published method of
// Jakob and Hanika, "A Low-Dimensional Function Space for Efficient Spectral
// Upsampling" (Eurographics 2019): for every table cell the three coefficients
// of s(c0 l^2 + c1 l + c2) are fitted by Gauss-Newton so that the reflectance
// seen under D65 reproduces the cell's linear-sRGB colour in CIELAB, sweeping
// each (x, y) column outward from a middle brightness and warm-starting every
// solve from its neighbour.  The table layout and the host-side trilinear
// decode follow hero.cpp:92-175.
#include "vs_host.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <thread>

#include "data/spectral_tables.inc"

namespace vs {

namespace {

constexpr int kRes = 64;
constexpr int kStepNm = 1;

struct Cmf {
    // Integration weights for X, Y, Z under D65, normalised so that a perfect
    // white reflector has Y = 1.
    std::vector<double> lambda, wx, wy, wz;
    double white[3];
};

const Cmf &cmf() {
    static Cmf c = [] {
        Cmf m;
        double ny = 0.0;
        for (int i = 0; i < kCieSamples; i += kStepNm) ny += VS_CIE_D65[i] * VS_CIE_Y[i];
        for (int i = 0; i < kCieSamples; i += kStepNm) {
            double w = VS_CIE_D65[i] / ny;
            m.lambda.push_back(360.0 + i);
            m.wx.push_back(w * VS_CIE_X[i]);
            m.wy.push_back(w * VS_CIE_Y[i]);
            m.wz.push_back(w * VS_CIE_Z[i]);
        }
        m.white[0] = m.white[1] = m.white[2] = 0.0;
        for (size_t i = 0; i < m.lambda.size(); ++i) {
            m.white[0] += m.wx[i];
            m.white[1] += m.wy[i];
            m.white[2] += m.wz[i];
        }
        return m;
    }();
    return c;
}

double lab_f(double t) {
    const double d = 6.0 / 29.0;
    return t > d * d * d ? std::cbrt(t) : t / (3.0 * d * d) + 4.0 / 29.0;
}

void xyz_to_lab(const double xyz[3], double lab[3]) {
    const Cmf &m = cmf();
    double fx = lab_f(xyz[0] / m.white[0]);
    double fy = lab_f(xyz[1] / m.white[1]);
    double fz = lab_f(xyz[2] / m.white[2]);
    lab[0] = 116.0 * fy - 16.0;
    lab[1] = 500.0 * (fx - fy);
    lab[2] = 200.0 * (fy - fz);
}

// Linear sRGB -> XYZ (matrix of src/base/color/cie.h:423-429).
void rgb_to_xyz(const double rgb[3], double xyz[3]) {
    xyz[0] = 0.412453 * rgb[0] + 0.357580 * rgb[1] + 0.180423 * rgb[2];
    xyz[1] = 0.212671 * rgb[0] + 0.715160 * rgb[1] + 0.072169 * rgb[2];
    xyz[2] = 0.019334 * rgb[0] + 0.119193 * rgb[1] + 0.950227 * rgb[2];
}

double sigmoid(double x) { return 0.5 * x / std::sqrt(1.0 + x * x) + 0.5; }

// Lab of the reflectance s(c0 t^2 + c1 t + c2), t = normalised wavelength.
void model_lab(const double c[3], double lab[3]) {
    const Cmf &m = cmf();
    double xyz[3] = {0, 0, 0};
    for (size_t i = 0; i < m.lambda.size(); ++i) {
        double t = (m.lambda[i] - 360.0) / 470.0;
        double s = sigmoid((c[0] * t + c[1]) * t + c[2]);
        xyz[0] += s * m.wx[i];
        xyz[1] += s * m.wy[i];
        xyz[2] += s * m.wz[i];
    }
    xyz_to_lab(xyz, lab);
}

bool solve3(double a[3][3], double b[3], double x[3]) {
    // Gaussian elimination with partial pivoting.
    int p[3] = {0, 1, 2};
    for (int c = 0; c < 3; ++c) {
        int best = c;
        for (int r = c + 1; r < 3; ++r)
            if (std::fabs(a[p[r]][c]) > std::fabs(a[p[best]][c])) best = r;
        std::swap(p[c], p[best]);
        if (std::fabs(a[p[c]][c]) < 1e-15) return false;
        for (int r = c + 1; r < 3; ++r) {
            double f = a[p[r]][c] / a[p[c]][c];
            for (int k = c; k < 3; ++k) a[p[r]][k] -= f * a[p[c]][k];
            b[p[r]] -= f * b[p[c]];
        }
    }
    for (int c = 2; c >= 0; --c) {
        double s = b[p[c]];
        for (int k = c + 1; k < 3; ++k) s -= a[p[c]][k] * x[k];
        x[c] = s / a[p[c]][c];
    }
    return true;
}

// Gauss-Newton fit of the normalised-wavelength coefficients to an RGB.
void fit(const double rgb[3], double c[3]) {
    double xyz[3], target[3];
    rgb_to_xyz(rgb, xyz);
    xyz_to_lab(xyz, target);
    for (int it = 0; it < 40; ++it) {
        double lab[3], r[3];
        model_lab(c, lab);
        for (int k = 0; k < 3; ++k) r[k] = lab[k] - target[k];
        double err = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        if (err < 1e-8) break;
        double J[3][3];
        const double h = 1e-4;
        for (int k = 0; k < 3; ++k) {
            double cp[3] = {c[0], c[1], c[2]}, cm[3] = {c[0], c[1], c[2]};
            cp[k] += h;
            cm[k] -= h;
            double lp[3], lm[3];
            model_lab(cp, lp);
            model_lab(cm, lm);
            for (int j = 0; j < 3; ++j) J[j][k] = (lp[j] - lm[j]) / (2.0 * h);
        }
        double dx[3];
        if (!solve3(J, r, dx)) break;
        double mx = std::max(std::fabs(dx[0]), std::max(std::fabs(dx[1]), std::fabs(dx[2])));
        double scale = mx > 200.0 ? 200.0 / mx : 1.0;
        for (int k = 0; k < 3; ++k) c[k] -= scale * dx[k];
        double mc = std::max(std::fabs(c[0]), std::max(std::fabs(c[1]), std::fabs(c[2])));
        if (mc > 1e4) {  // keep the sigmoid argument bounded near saturated colours
            for (int k = 0; k < 3; ++k) c[k] *= 1e4 / mc;
        }
    }
}

// Normalised-wavelength coefficients -> coefficients in nm.
void to_nm(const double c[3], float out[3]) {
    const double lo = 360.0, range = 470.0;
    double A = c[0] / (range * range);
    double B = c[1] / range - 2.0 * c[0] * lo / (range * range);
    double C = c[0] * lo * lo / (range * range) - c[1] * lo / range + c[2];
    out[0] = static_cast<float>(A);
    out[1] = static_cast<float>(B);
    out[2] = static_cast<float>(C);
}

double smoothstep(double x) { return x * x * (3.0 - 2.0 * x); }

std::vector<float> build_table() {
    std::vector<float> table(static_cast<size_t>(3) * kRes * kRes * kRes * 4, 0.0f);
    std::vector<double> zs(kRes);
    for (int k = 0; k < kRes; ++k) zs[k] = smoothstep(smoothstep(k / double(kRes - 1)));
    const int k0 = kRes / 5;
    std::atomic<int> next{0};
    auto worker = [&]() {
        while (true) {
            int job = next.fetch_add(1);
            if (job >= 3 * kRes * kRes) break;
            int l = job / (kRes * kRes);
            int j = (job / kRes) % kRes;
            int i = job % kRes;
            double x = i / double(kRes - 1), y = j / double(kRes - 1);
            auto run = [&](int k, double c[3]) {
                double z = zs[k];
                double rgb[3];
                rgb[l] = z;
                rgb[(l + 1) % 3] = x * z;
                rgb[(l + 2) % 3] = y * z;
                fit(rgb, c);
                float co[3];
                to_nm(c, co);
                size_t idx = ((((static_cast<size_t>(l) * kRes + k) * kRes + j) * kRes + i) * 4);
                table[idx + 0] = co[0];
                table[idx + 1] = co[1];
                table[idx + 2] = co[2];
                table[idx + 3] = 0.0f;
            };
            double c[3] = {0.0, 0.0, 0.0};
            for (int k = k0; k < kRes; ++k) run(k, c);
            c[0] = c[1] = c[2] = 0.0;
            for (int k = k0; k >= 0; --k) run(k, c);
        }
    };
    unsigned nt = std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t) th.emplace_back(worker);
    for (auto &t : th) t.join();
    return table;
}

std::mutex g_table_mutex;
std::vector<float> g_table;

}  // namespace

const float *rgb2spec_table(const std::string &cache_path) {
    std::lock_guard<std::mutex> lock(g_table_mutex);
    if (!g_table.empty()) return g_table.data();
    const size_t n = static_cast<size_t>(3) * kRes * kRes * kRes * 4;
    if (!cache_path.empty()) {
        std::ifstream in(cache_path, std::ios::binary);
        if (in) {
            std::vector<float> t(n);
            in.read(reinterpret_cast<char *>(t.data()), static_cast<std::streamsize>(n * sizeof(float)));
            if (in.gcount() == static_cast<std::streamsize>(n * sizeof(float))) {
                g_table = std::move(t);
                return g_table.data();
            }
        }
    }
    g_table = build_table();
    if (!cache_path.empty()) {
        std::string tmp = cache_path + ".tmp";
        std::ofstream out(tmp, std::ios::binary);
        if (out) {
            out.write(reinterpret_cast<const char *>(g_table.data()), static_cast<std::streamsize>(n * sizeof(float)));
            out.close();
            std::rename(tmp.c_str(), cache_path.c_str());
        }
    }
    return g_table.data();
}

// RGBToSpectrumTable::decode_albedo, host path (hero.cpp:92-133).
void rgb2spec_decode_albedo(const float *table, const float rgb_in[3], float out[4]) {
    float rgb[3];
    for (int k = 0; k < 3; ++k) rgb[k] = std::min(std::max(rgb_in[k], 0.0f), 1.0f);
    float y = 0.212671f * rgb[0] + 0.715160f * rgb[1] + 0.072169f * rgb[2];
    if (rgb[0] == rgb[1] && rgb[1] == rgb[2]) {
        float s = (rgb[0] - 0.5f) / std::sqrt(rgb[0] * (1.0f - rgb[0]));
        out[0] = 0.0f; out[1] = 0.0f; out[2] = s; out[3] = y;
        return;
    }
    uint32_t maxc = (rgb[0] > rgb[1]) ? ((rgb[0] > rgb[2]) ? 0u : 2u) : ((rgb[1] > rgb[2]) ? 1u : 2u);
    float z = rgb[maxc];
    float x = rgb[(maxc + 1u) % 3u] * (kRes - 1u) / z;
    float yy = rgb[(maxc + 2u) % 3u] * (kRes - 1u) / z;
    auto inv_ss = [](float v) { return 0.5f - std::sin(std::asin(1.0f - 2.0f * v) * (1.0f / 3.0f)); };
    float zz = inv_ss(inv_ss(z)) * (kRes - 1u);
    uint32_t xi = std::min(static_cast<uint32_t>(x), static_cast<uint32_t>(kRes - 2));
    uint32_t yi = std::min(static_cast<uint32_t>(yy), static_cast<uint32_t>(kRes - 2));
    uint32_t zi = std::min(static_cast<uint32_t>(zz), static_cast<uint32_t>(kRes - 2));
    float dx = x - static_cast<float>(xi), dy = yy - static_cast<float>(yi), dz = zz - static_cast<float>(zi);
    auto lerp = [](float t, float a, float b) { return a + t * (b - a); };
    for (int i = 0; i < 3; ++i) {
        auto co = [&](int ox, int oy, int oz) {
            size_t idx = ((((static_cast<size_t>(maxc) * kRes + (zi + oz)) * kRes + (yi + oy)) * kRes + (xi + ox)) * 4) + i;
            return table[idx];
        };
        out[i] = lerp(dz, lerp(dy, lerp(dx, co(0, 0, 0), co(1, 0, 0)), lerp(dx, co(0, 1, 0), co(1, 1, 0))),
                      lerp(dy, lerp(dx, co(0, 0, 1), co(1, 0, 1)), lerp(dx, co(0, 1, 1), co(1, 1, 1))));
    }
    out[3] = y;
}

// RGBToSpectrumTable::decode_unbound (hero.cpp:135-141): coefficients of rgb/(2 max)
// and the scale 2 max in out[3].
void rgb2spec_decode_unbound(const float *table, const float rgb_in[3], float out[4]) {
    float rgb[3] = {std::max(rgb_in[0], 0.0f), std::max(rgb_in[1], 0.0f), std::max(rgb_in[2], 0.0f)};
    float m = std::max(rgb[0], std::max(rgb[1], rgb[2]));
    float scale = 2.0f * m;
    float q[3];
    for (int k = 0; k < 3; ++k) q[k] = scale == 0.0f ? 0.0f : rgb[k] / scale;
    float c[4];
    rgb2spec_decode_albedo(table, q, c);
    out[0] = c[0]; out[1] = c[1]; out[2] = c[2]; out[3] = scale;
}

}  // namespace vs

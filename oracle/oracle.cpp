// ORACLE — test infrastructure only.  A scalar CPU restatement of the
// reference's spectral path tracer (FaithZL/Vision), used by tests/, by
// __graft_entry__.smoke() and by bench.py's cpu_baseline leg as the checker.
// It is never part of the rendering product.
//
// Parity pinning: the reference cannot be built or run (its ocarina submodule
// holds the DSL/OptiX backend and is empty; its host code is Windows-only), so
// this oracle is pinned against the reference's own data tables (CIE/D65
// spectra, metal IOR), against the golden vectors committed under
// tests/golden/ (TEA/LCG streams, alias tables, wavelength samples derived
// from the reference formulas) and, function by function, against the
// reference source lines cited below.  Path-level image parity against a
// reference binary is unpinned.
//
// The oracle reads the flattened scene exported by libvision_b200
// (vs_scene_export) so that it traces exactly the same triangles, materials
// and emitters; everything from the sampler to the film is computed here,
// independently of the CUDA code, in FP32 like the reference, with an FP64
// film option.  Compile with -ffp-contract=off: the watertight triangle test
// must round exactly like the GPU's explicitly rounded version.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "../vision_b200/csrc/data/spectral_tables.inc"

namespace oracle {

struct V3 {
    float x, y, z;
};
static inline V3 v3(float x, float y, float z) { return {x, y, z}; }
static inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline V3 mul(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
static inline V3 neg(V3 a) { return {-a.x, -a.y, -a.z}; }
static inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
static inline float len(V3 a) { return std::sqrt(dot(a, a)); }
static inline V3 normalize(V3 a) { return mul(a, 1.0f / std::sqrt(dot(a, a))); }
static inline float at(V3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
static inline uint32_t fbits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
static inline float bitsf(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

// ----- exported scene layout (include/vision_b200.h, VS_EXPORT_*) -----------
struct Material {
    uint32_t type, flags, spd0, spd1;
    float coef[4];
    float p[8];
};
struct AreaLight {
    uint32_t inst, first_prim, prim_count, alias_offset, two_sided, kind;
    float scale, lum_power;
    float coef[4];
    float rgb_avg[4];
    uint32_t shape;  // 0 area, 1 point, 2 spot
    float cos_angle, cos_start;
    uint32_t pad;
    float pos[4], dir[4];
};
static_assert(sizeof(AreaLight) == 112, "light record layout");
struct Instance {
    uint32_t mat_id, light_id, first_prim, prim_count;
};
struct Alias {
    float prob;
    uint32_t alias;
};
struct Camera {
    float c2w[4][4];
    float tan_half_fov, screen_lo_x, screen_hi_y, screen_span_x, screen_span_y, filter_rx, filter_ry;
    uint32_t width, height;
    float exposure;
    uint32_t filter;     // 0 box, 1 triangle, 2 gaussian, 3 mitchell, 4 sinc
    uint32_t thin_lens;  // 1: ThinLensCamera
    float lens_radius, focal_distance, filter_p0, filter_p1;
};
static_assert(sizeof(Camera) == 128, "Camera layout");
struct EnvLight {
    float w2o[4][4];
    float o2w[4][4];
    uint32_t width, height;
    float scale, integral, world_diameter, lum_power;
    uint32_t pad0, pad1;
};
struct Integrator {
    uint32_t max_depth, min_depth;
    float rr_threshold;
    uint32_t mis_mode, spectrum_dim, scatter_pdf_dim, sampler, seed, light_sampler, light_count, srgb, pad1;
};

}  // namespace oracle

extern "C" {
// Pointers into the exported arrays; counts in elements.
struct oracle_scene {
    const float *pos;
    const float *nrm;
    const float *uv;
    const uint32_t *idx;
    const uint32_t *prim_inst;
    uint32_t vertex_count;
    uint32_t prim_count;
    const void *instances;
    uint32_t instance_count;
    const void *materials;
    uint32_t material_count;
    const void *lights;
    uint32_t light_count;
    const void *prim_alias;
    const float *prim_pmf;
    const void *light_alias;
    const float *light_pmf;
    const void *camera;
    const void *integrator;
    const float *spd;
    // Environment light (env == nullptr: none).
    const void *env;
    const float *env_tex;
    const void *env_marginal;
    const float *env_marginal_func;
    const void *env_cond;
    const float *env_cond_func;
    const float *rgb2spec;
    // Instancing (two_level = 1): the distinct object-space meshes (6 uint32
    // per mesh: first vertex, vertex count, first triangle, triangle count,
    // hash), each instance's mesh and column-major world-to-object transform.
    // Rays are traced in each instance's object space, as the library's
    // two-level BVH does.
    uint32_t two_level;
    uint32_t mesh_count;
    const float *mesh_pos;
    const uint32_t *mesh_idx;
    const uint32_t *meshes;
    const uint32_t *inst_mesh;
    const float *inst_w2o;
    // Textures of `image` shader nodes: linear RGB texels (4 floats each) and
    // per texture its texel offset, width, height and 0.
    const float *tex_texels;
    const uint32_t *textures;
    uint32_t texture_count;
};
}

namespace oracle {

constexpr uint32_t kInvalid = 0xffffffffu;
constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.31830988618379067154f;
constexpr float kOneMinusEps = 0x1.fffffep-1f;
constexpr float kShadowEps = 0.0001f;

// ----- spectral tables -------------------------------------------------------
// SPD::create_cie_* downsample every 5th 1-nm sample: 94 entries, 360..825 nm
// (src/base/color/spd.cpp:31-38,96-110); cie_y_integral sums 94 trapezoids of
// 5 nm up to 830 nm (:14-23).
struct Tables {
    float x[94], y[94], z[94], d65[94];
    float y_integral;
    Tables() {
        for (int i = 0; i < 94; ++i) {
            x[i] = VS_CIE_X[5 * i];
            y[i] = VS_CIE_Y[5 * i];
            z[i] = VS_CIE_Z[5 * i];
            d65[i] = VS_CIE_D65[5 * i];
        }
        float sum = 0.0f;
        for (int i = 0; i < 94; ++i) sum += 0.5f * (VS_CIE_Y[5 * i] + VS_CIE_Y[5 * (i + 1)]);
        y_integral = sum * 5.0f;
    }
};
static const Tables &tables() {
    static Tables t;
    return t;
}

// SPD::eval (spd.cpp:67-76): spacing 471 / n, index clamped to n - 2.
static float spd_eval(const float *f, int n, float lambda) {
    float interval = 471.0f / static_cast<float>(n);
    float t = (std::min(std::max(lambda, 360.0f), 830.0f) - 360.0f) / interval;
    float sample_count = static_cast<float>(static_cast<uint32_t>((830.0f - 360.0f) / interval) + 1u);
    uint32_t i = static_cast<uint32_t>(std::min(t, sample_count - 2.0f));
    float fr = t - std::floor(t);
    return f[i] + fr * (f[i + 1] - f[i]);
}

// RGBSigmoidPolynomial (hero.cpp:27-49).
static float sigmoid_poly(const float *c, float l) {
    float x = std::fma(std::fma(c[0], l, c[1]), l, c[2]);
    if (std::isinf(x)) return x > 0.0f ? 1.0f : 0.0f;
    return 0.5f * std::fma(x, 1.0f / std::sqrt(std::fma(x, x, 1.0f)), 1.0f);
}

static float planck(float lambda_nm, float T) {
    const float c = 299792458.0f, h = 6.62606957e-34f, kb = 1.3806488e-23f;
    float l = lambda_nm * 1e-9f;
    float l2 = l * l;
    float l5 = l2 * l2 * l;
    return (2.0f * h * c * c) / (l5 * (std::exp((h * c) / (l * kb * T)) - 1.0f));
}

// ----- sampler (independent.cpp:24-42, util.h:13-33) --------------------------
static uint32_t tea(uint32_t v0, uint32_t v1) {
    uint32_t s0 = 0;
    for (int n = 0; n < 4; ++n) {
        s0 += 0x9e3779b9u;
        v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + s0) ^ ((v1 >> 5) + 0xc8013ea4u);
        v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + s0) ^ ((v0 >> 5) + 0x7e95761eu);
    }
    return v0;
}

struct Sampler {
    uint32_t kind = 0;
    uint32_t lcg = 0;
    uint64_t pcg_state = 0, pcg_inc = 1;
    void start(uint32_t px, uint32_t py, uint32_t sample, uint32_t dim, uint32_t k, uint32_t seed) {
        kind = k;
        uint32_t s = tea(tea(px, py), tea(sample, dim));
        if (kind == 0) {
            lcg = s;
        } else {
            // PCG32 (O'Neill 2014) seeding as pcg32_srandom_r: state 0, one
            // step, add the TEA hash, one more step; stream = seed.
            pcg_inc = (static_cast<uint64_t>(seed) << 1u) | 1u;
            uint64_t st = 0u;
            st = st * 6364136223846793005ull + pcg_inc;
            st += s;
            st = st * 6364136223846793005ull + pcg_inc;
            pcg_state = st;
        }
    }
    float next() {
        if (kind == 0) {
            lcg = 1664525u * lcg + 1013904223u;
            return static_cast<float>(lcg & 0x00ffffffu) * (1.0f / 16777216.0f);
        }
        // 64-bit LCG step, XSH-RR output (pcg32_random_r), top 24 bits.
        uint64_t old = pcg_state;
        pcg_state = old * 6364136223846793005ull + pcg_inc;
        uint32_t xs = static_cast<uint32_t>(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = static_cast<uint32_t>(old >> 59u);
        uint32_t r = (xs >> rot) | (xs << ((32u - rot) & 31u));
        return static_cast<float>(r >> 8) * (1.0f / 16777216.0f);
    }
};

// ----- wavelengths (hero.cpp:15-25,286-299) ----------------------------------
struct Swl {
    int n;
    float lambda[8];
    float pdf[8];
};
// SRGBSpectrum (srgb.cpp:16-24): three channels at the sRGB primaries' peak
// wavelengths, stored negated to mark RGB transport (colour decodes pass RGB
// through; spectral curves are read at |lambda|).
static Swl rgb_wavelengths(int n) {
    const float peak[3] = {602.785f, 539.285f, 445.772f};
    Swl w;
    w.n = n;
    for (int i = 0; i < n; ++i) {
        w.lambda[i] = -peak[i < 3 ? i : 2];
        w.pdf[i] = 1.0f;
    }
    return w;
}
static bool is_rgb(const Swl &w) { return w.lambda[0] < 0.0f; }
// A colour slot's value on channel i: the colour itself under RGB transport,
// else the sigmoid spectrum at the channel's wavelength.
static float sigmoid_poly(const float *c, float l);
static float alb(const float *c, const Swl &w, int i) {
    return is_rgb(w) ? c[i < 3 ? i : 2] : sigmoid_poly(c, w.lambda[i]);
}

static Swl sample_wavelengths(int n, float u) {
    Swl w;
    w.n = n;
    for (int i = 0; i < n; ++i) {
        float offset = static_cast<float>(static_cast<uint32_t>(i) * (1.0f / n));
        float up = u + offset;
        up = up - std::floor(up);
        float l = 538.0f - 138.888889f * std::atanh(0.85691062f - 1.82750197f * up);
        w.lambda[i] = l;
        float c = std::cosh(0.0072f * (l - 538.0f));
        w.pdf[i] = 0.0039398042f / (c * c);
    }
    return w;
}

// HeroWavelengthSpectrum::cie_xyz / linear_srgb (hero.cpp:261-285; cie.h:414-421).
static V3 linear_srgb(const float *s, const Swl &w) {
    if (is_rgb(w)) return {s[0], s[w.n > 1 ? 1 : 0], s[w.n > 2 ? 2 : 0]};
    const Tables &T = tables();
    double dummy = 0;
    (void)dummy;
    float X = 0, Y = 0, Z = 0;
    int valid = 0;
    for (int i = 0; i < w.n; ++i) {
        float p = w.pdf[i];
        valid += p > 0.0f;
        auto sd = [&](float a) { return p == 0.0f ? 0.0f : a / p; };
        X += sd(spd_eval(T.x, 94, w.lambda[i]) * s[i]);
        Y += sd(spd_eval(T.y, 94, w.lambda[i]) * s[i]);
        Z += sd(spd_eval(T.z, 94, w.lambda[i]) * s[i]);
    }
    float factor = 1.0f / (static_cast<float>(valid) * T.y_integral);
    X *= factor; Y *= factor; Z *= factor;
    return {3.240479f * X - 1.537150f * Y - 0.498535f * Z, -0.969256f * X + 1.875991f * Y + 0.041556f * Z,
            0.055648f * X - 0.204043f * Y + 1.057311f * Z};
}

// ----- ray offset (Waechter & Binder, Ray Tracing Gems ch. 6) -----------------
static float offset1(float p, float n) {
    int of = static_cast<int>(256.0f * n);
    int pi = static_cast<int>(fbits(p));
    float pn = bitsf(static_cast<uint32_t>(pi + (p < 0.0f ? -of : of)));
    return std::fabs(p) < 1.0f / 32.0f ? p + (1.0f / 65536.0f) * n : pn;
}
static V3 offset_ray_origin(V3 p, V3 n) { return {offset1(p.x, n.x), offset1(p.y, n.y), offset1(p.z, n.z)}; }

// ----- geometry --------------------------------------------------------------
struct Scene {
    const oracle_scene *s;
    const Instance *inst;
    const Material *mat;
    const AreaLight *lights;
    const Alias *prim_alias;
    const Alias *light_alias;
    Camera cam;
    Integrator ip;
    EnvLight env;
    bool has_env = false;
    // Binary BVH over primitives (median split), for scenes too large to brute force.
    struct Node {
        float lo[3], hi[3];
        uint32_t left, right, first, count;
    };
    std::vector<Node> nodes;
    std::vector<uint32_t> order;
    // FilterSampler tables (fitted_curve.h:36-58) of the tabulated filters.
    static constexpr uint32_t kFilterN = 20;
    std::vector<float> f_lut, f_marginal_func, f_cond_func;
    std::vector<Alias> f_marginal, f_cond;
    float f_integral = 0.0f;

    V3 P(uint32_t v) const { return {s->pos[3 * v], s->pos[3 * v + 1], s->pos[3 * v + 2]}; }
    V3 N(uint32_t v) const { return {s->nrm[3 * v], s->nrm[3 * v + 1], s->nrm[3 * v + 2]}; }

    uint32_t build(uint32_t first, uint32_t count) {
        uint32_t id = static_cast<uint32_t>(nodes.size());
        nodes.push_back({});
        float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        float clo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, chi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (uint32_t i = first; i < first + count; ++i) {
            uint32_t p = order[i];
            for (int k = 0; k < 3; ++k) {
                V3 v = P(s->idx[3 * p + k]);
                for (int a = 0; a < 3; ++a) {
                    lo[a] = std::min(lo[a], at(v, a));
                    hi[a] = std::max(hi[a], at(v, a));
                }
            }
            for (int a = 0; a < 3; ++a) {
                float c = 0.0f;
                for (int k = 0; k < 3; ++k) c += at(P(s->idx[3 * p + k]), a);
                clo[a] = std::min(clo[a], c);
                chi[a] = std::max(chi[a], c);
            }
        }
        std::memcpy(nodes[id].lo, lo, sizeof(lo));
        std::memcpy(nodes[id].hi, hi, sizeof(hi));
        if (count <= 4) {
            nodes[id].first = first;
            nodes[id].count = count;
            nodes[id].left = nodes[id].right = 0;
            return id;
        }
        int axis = 0;
        for (int a = 1; a < 3; ++a)
            if (chi[a] - clo[a] > chi[axis] - clo[axis]) axis = a;
        uint32_t mid = first + count / 2;
        std::nth_element(order.begin() + first, order.begin() + mid, order.begin() + first + count,
                         [&](uint32_t a, uint32_t b) {
                             float ca = 0.0f, cb = 0.0f;
                             for (int k = 0; k < 3; ++k) {
                                 ca += at(P(s->idx[3 * a + k]), axis);
                                 cb += at(P(s->idx[3 * b + k]), axis);
                             }
                             return ca < cb || (ca == cb && a < b);
                         });
        uint32_t l = build(first, mid - first);
        uint32_t r = build(mid, first + count - mid);
        nodes[id].left = l;
        nodes[id].right = r;
        nodes[id].count = 0;
        return id;
    }

    // AliasTable::build (warpers/alias.h:86-118): probabilities scaled by
    // n / sum (sum in double), over-full slots fill under-full ones from the
    // back of both lists; the row integral is sum / n.
    static float alias_build(const float *w, uint32_t n, Alias *out) {
        double total = 0.0;
        for (uint32_t i = 0; i < n; ++i) total += w[i];
        const double scale = static_cast<double>(n) / total;
        std::vector<uint32_t> big, small;
        for (uint32_t i = 0; i < n; ++i) {
            out[i].prob = static_cast<float>(w[i] * scale);
            out[i].alias = i;
            if (out[i].prob > 1.0f) big.push_back(i);
            else small.push_back(i);
        }
        while (!big.empty() && !small.empty()) {
            const uint32_t b = big.back(), l = small.back();
            big.pop_back();
            small.pop_back();
            out[b].prob -= 1.0f - out[l].prob;
            out[l].alias = b;
            if (out[b].prob > 1.0f) big.push_back(b);
            else if (out[b].prob < 1.0f) small.push_back(b);
        }
        for (uint32_t i : big) out[i] = {1.0f, i};
        for (uint32_t i : small) out[i] = {1.0f, i};
        return static_cast<float>(total / static_cast<double>(n));
    }

    // GaussianFilter / MitchellFilter / LanczosSincFilter ::evaluate
    // (filters/gaussian.cpp:36-40, mitchell.cpp, sinc.cpp) at p in [0, r]^2.
    float filter_eval(float x, float y) const {
        const float pi = 3.14159265358979323846f;
        if (cam.filter == 2u) {
            const float sg = cam.filter_p0;
            auto gauss = [&](float v) { return 1.0f / std::sqrt(2.0f * pi * sg * sg) * std::exp(-(v * v) / (2.0f * sg * sg)); };
            return std::max(0.0f, gauss(x) - gauss(cam.filter_rx)) * std::max(0.0f, gauss(y) - gauss(cam.filter_ry));
        }
        if (cam.filter == 3u) {
            const float B = cam.filter_p0, C = cam.filter_p1;
            auto mitchell = [&](float v) {
                v = std::fabs(v);
                float r = 0.0f;
                if (v <= 1.0f)
                    r = (12.0f - 9.0f * B - 6.0f * C) * v * v * v + (-18.0f + 12.0f * B + 6.0f * C) * v * v +
                        (6.0f - 2.0f * B);
                else if (v <= 2.0f)
                    r = (-B - 6.0f * C) * v * v * v + (6.0f * B + 30.0f * C) * v * v + (-12.0f * B - 48.0f * C) * v +
                        (8.0f * B + 24.0f * C);
                return r * (1.0f / 6.0f);
            };
            return mitchell(2.0f * x / cam.filter_rx) * mitchell(2.0f * y / cam.filter_ry);
        }
        const float tau = cam.filter_p0;
        auto sinc = [&](float v) {
            const float a = pi * v;
            return 1.0f + a * a == 1.0f ? 1.0f : std::sin(a) / a;
        };
        auto windowed = [&](float v, float r) { return std::fabs(v) > r ? 0.0f : sinc(v) * sinc(v / tau); };
        return windowed(x, cam.filter_rx) * windowed(y, cam.filter_ry) * 4.0f;
    }

    // FilterSampler::build (fitted_curve.h:36-58) + AliasTable2D::build
    // (warpers/alias2d.cpp:32-67): the filter at cell centres of [0, r]^2,
    // normalised by its average; rows and marginal over |filter|.
    void build_filter() {
        const uint32_t n = kFilterN;
        f_lut.assign(n * n, 0.0f);
        f_cond_func.assign(n * n, 0.0f);
        for (uint32_t y = 0; y < n; ++y)
            for (uint32_t x = 0; x < n; ++x) {
                const float v = filter_eval((static_cast<float>(x) + 0.5f) / static_cast<float>(n) * cam.filter_rx,
                                            (static_cast<float>(y) + 0.5f) / static_cast<float>(n) * cam.filter_ry);
                f_lut[y * n + x] = v;
                f_cond_func[y * n + x] = std::fabs(v);
            }
        float total = 0.0f;
        for (float v : f_lut) total += v;
        const float mean = total / static_cast<float>(n * n);
        for (float &v : f_lut) v = v / mean;
        f_cond.resize(n * n);
        f_marginal_func.resize(n);
        for (uint32_t y = 0; y < n; ++y)
            f_marginal_func[y] = alias_build(f_cond_func.data() + y * n, n, f_cond.data() + y * n);
        f_marginal.resize(n);
        f_integral = alias_build(f_marginal_func.data(), n, f_marginal.data());
    }

    explicit Scene(const oracle_scene *sc) : s(sc) {
        inst = static_cast<const Instance *>(sc->instances);
        mat = static_cast<const Material *>(sc->materials);
        lights = static_cast<const AreaLight *>(sc->lights);
        prim_alias = static_cast<const Alias *>(sc->prim_alias);
        light_alias = static_cast<const Alias *>(sc->light_alias);
        std::memcpy(&cam, sc->camera, sizeof(Camera));
        std::memcpy(&ip, sc->integrator, sizeof(Integrator));
        if (sc->env) {
            std::memcpy(&env, sc->env, sizeof(EnvLight));
            has_env = true;
        }
        if (cam.filter >= 2u) build_filter();
        if (sc->two_level) {
            build_instances();
            return;
        }
        order.resize(sc->prim_count);
        for (uint32_t i = 0; i < sc->prim_count; ++i) order[i] = i;
        nodes.reserve(sc->prim_count / 2 + 8);
        build(0, sc->prim_count);
    }

    // Two-level scenes: a median-split BVH per mesh over its object-space
    // triangles, each instance's world box (from its world-space vertices)
    // and world-to-object rows.
    struct MeshBvh {
        const float *pos;
        const uint32_t *idx;
        std::vector<Node> nodes;
        std::vector<uint32_t> order;
        V3 Pm(uint32_t v) const { return {pos[3 * v], pos[3 * v + 1], pos[3 * v + 2]}; }
        uint32_t build(uint32_t first, uint32_t count) {
            uint32_t id = static_cast<uint32_t>(nodes.size());
            nodes.push_back({});
            float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
            for (uint32_t i = first; i < first + count; ++i)
                for (int k = 0; k < 3; ++k) {
                    V3 v = Pm(idx[3 * order[i] + k]);
                    for (int a = 0; a < 3; ++a) {
                        lo[a] = std::min(lo[a], at(v, a));
                        hi[a] = std::max(hi[a], at(v, a));
                    }
                }
            std::memcpy(nodes[id].lo, lo, sizeof(lo));
            std::memcpy(nodes[id].hi, hi, sizeof(hi));
            if (count <= 4) {
                nodes[id].first = first;
                nodes[id].count = count;
                return id;
            }
            int axis = 0;
            for (int a = 1; a < 3; ++a)
                if (hi[a] - lo[a] > hi[axis] - lo[axis]) axis = a;
            uint32_t mid = first + count / 2;
            auto key = [&](uint32_t t) {
                float c = 0.0f;
                for (int k = 0; k < 3; ++k) c += at(Pm(idx[3 * t + k]), axis);
                return c;
            };
            std::nth_element(order.begin() + first, order.begin() + mid, order.begin() + first + count,
                             [&](uint32_t a, uint32_t b) { return key(a) < key(b) || (key(a) == key(b) && a < b); });
            uint32_t l = build(first, mid - first);
            uint32_t r = build(mid, first + count - mid);
            nodes[id].left = l;
            nodes[id].right = r;
            nodes[id].count = 0;
            return id;
        }
    };
    std::vector<MeshBvh> mesh_bvh;
    std::vector<float> inst_lo, inst_hi, inst_rows;  // 3, 3 and 12 floats per instance

    void build_instances() {
        mesh_bvh.resize(s->mesh_count);
        for (uint32_t m = 0; m < s->mesh_count; ++m) {
            const uint32_t *r = s->meshes + 6 * m;
            MeshBvh &b = mesh_bvh[m];
            b.pos = s->mesh_pos + 3 * static_cast<size_t>(r[0]);
            b.idx = s->mesh_idx + 3 * static_cast<size_t>(r[2]);
            b.order.resize(r[3]);
            for (uint32_t i = 0; i < r[3]; ++i) b.order[i] = i;
            b.build(0, r[3]);
        }
        inst_lo.assign(3 * s->instance_count, FLT_MAX);
        inst_hi.assign(3 * s->instance_count, -FLT_MAX);
        inst_rows.resize(12 * s->instance_count);
        for (uint32_t i = 0; i < s->instance_count; ++i) {
            const Instance &in = inst[i];
            for (uint32_t p = in.first_prim; p < in.first_prim + in.prim_count; ++p)
                for (int k = 0; k < 3; ++k) {
                    V3 v = P(s->idx[3 * p + k]);
                    for (int a = 0; a < 3; ++a) {
                        inst_lo[3 * i + a] = std::min(inst_lo[3 * i + a], at(v, a));
                        inst_hi[3 * i + a] = std::max(inst_hi[3 * i + a], at(v, a));
                    }
                }
            // Pad the box a little: it only culls instances, and a hit found in
            // object space may lie a rounding step outside the world box.
            for (int a = 0; a < 3; ++a) {
                const float pad = 1e-5f * std::max(std::fabs(inst_lo[3 * i + a]), std::fabs(inst_hi[3 * i + a])) + 1e-6f;
                inst_lo[3 * i + a] -= pad;
                inst_hi[3 * i + a] += pad;
            }
            const float *m = s->inst_w2o + 16 * static_cast<size_t>(i);  // m[4 c + r]
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 4; ++c) inst_rows[12 * i + 4 * r + c] = m[4 * c + r];
        }
    }
};

// Watertight ray/triangle test (Woop, Benthin, Wald, JCGT 2013), same operation
// order and rounding as the GPU version.
struct RayPre {
    V3 o, d, inv;
    int kx, ky, kz;
    float sx, sy, sz;
};
static RayPre precompute(V3 o, V3 d) {
    RayPre r;
    r.o = o;
    r.d = d;
    const float tiny = 1e-30f;
    auto inv1 = [&](float x) { return 1.0f / (std::fabs(x) > tiny ? x : std::copysign(tiny, x)); };
    r.inv = {inv1(d.x), inv1(d.y), inv1(d.z)};
    float ax = std::fabs(d.x), ay = std::fabs(d.y), az = std::fabs(d.z);
    int kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    int kx = kz + 1 == 3 ? 0 : kz + 1;
    int ky = kx + 1 == 3 ? 0 : kx + 1;
    if (at(d, kz) < 0.0f) std::swap(kx, ky);
    r.kx = kx; r.ky = ky; r.kz = kz;
    float dz = at(d, kz);
    r.sx = at(d, kx) / dz;
    r.sy = at(d, ky) / dz;
    r.sz = 1.0f / dz;
    return r;
}
static bool tri_hit(const RayPre &r, V3 v0, V3 v1, V3 v2, float tmin, float tmax, float &t_out, float &u_out,
                    float &v_out) {
    float ax = at(v0, r.kx) - at(r.o, r.kx), ay = at(v0, r.ky) - at(r.o, r.ky), az = at(v0, r.kz) - at(r.o, r.kz);
    float bx = at(v1, r.kx) - at(r.o, r.kx), by = at(v1, r.ky) - at(r.o, r.ky), bz = at(v1, r.kz) - at(r.o, r.kz);
    float cx = at(v2, r.kx) - at(r.o, r.kx), cy = at(v2, r.ky) - at(r.o, r.ky), cz = at(v2, r.kz) - at(r.o, r.kz);
    float Ax = ax - r.sx * az, Ay = ay - r.sy * az;
    float Bx = bx - r.sx * bz, By = by - r.sy * bz;
    float Cx = cx - r.sx * cz, Cy = cy - r.sy * cz;
    float U = Cx * By - Cy * Bx;
    float V = Ax * Cy - Ay * Cx;
    float W = Bx * Ay - By * Ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = static_cast<float>(static_cast<double>(Cx) * By - static_cast<double>(Cy) * Bx);
        V = static_cast<float>(static_cast<double>(Ax) * Cy - static_cast<double>(Ay) * Cx);
        W = static_cast<float>(static_cast<double>(Bx) * Ay - static_cast<double>(By) * Ax);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    float det = (U + V) + W;
    if (det == 0.0f) return false;
    float Az = r.sz * az, Bz = r.sz * bz, Cz = r.sz * cz;
    float T = (U * Az + V * Bz) + W * Cz;
    float t = T / det;
    if (!(t > tmin && t < tmax)) return false;
    t_out = t;
    u_out = V / det;
    v_out = W / det;
    return true;
}

static bool box_hit(const RayPre &r, const float *lo, const float *hi, float tmax) {
    float tn = 0.0f, tf = tmax;
    for (int a = 0; a < 3; ++a) {
        float t0 = (lo[a] - at(r.o, a)) * at(r.inv, a), t1 = (hi[a] - at(r.o, a)) * at(r.inv, a);
        tn = std::max(tn, std::min(t0, t1));
        tf = std::min(tf, std::max(t0, t1));
    }
    return tn <= tf * 1.000001f;
}

struct HitRec {
    uint32_t prim = kInvalid;
    float t = 0, u = 0, v = 0;
};

// The ray in an instance's object space: rows r[0..11] of the world-to-object
// transform, products and sums in the GPU's order (no contraction).
static RayPre instance_ray(const float *w, const RayPre &r) {
    V3 o = {((w[0] * r.o.x + w[1] * r.o.y) + w[2] * r.o.z) + w[3], ((w[4] * r.o.x + w[5] * r.o.y) + w[6] * r.o.z) + w[7],
            ((w[8] * r.o.x + w[9] * r.o.y) + w[10] * r.o.z) + w[11]};
    V3 d = {(w[0] * r.d.x + w[1] * r.d.y) + w[2] * r.d.z, (w[4] * r.d.x + w[5] * r.d.y) + w[6] * r.d.z,
            (w[8] * r.d.x + w[9] * r.d.y) + w[10] * r.d.z};
    return precompute(o, d);
}

// Two-level closest hit: every instance whose world box the ray meets, its
// mesh's triangles in object space; global ids first_prim + triangle index,
// exact ties in t to the lower global id.
static HitRec closest_instanced(const Scene &sc, const RayPre &rw, float tmax) {
    HitRec best;
    best.t = tmax;
    for (uint32_t i = 0; i < sc.s->instance_count; ++i) {
        if (!box_hit(rw, &sc.inst_lo[3 * i], &sc.inst_hi[3 * i], best.t * 1.000001f)) continue;
        const RayPre r = instance_ray(&sc.inst_rows[12 * i], rw);
        const Scene::MeshBvh &b = sc.mesh_bvh[sc.s->inst_mesh[i]];
        const uint32_t first = sc.inst[i].first_prim;
        uint32_t stack[128];
        int sp = 0;
        stack[sp++] = 0;
        while (sp) {
            const Scene::Node &n = b.nodes[stack[--sp]];
            if (!box_hit(r, n.lo, n.hi, best.t * 1.000001f)) continue;
            if (n.count) {
                for (uint32_t k = n.first; k < n.first + n.count; ++k) {
                    uint32_t t3 = b.order[k];
                    float t, u, v;
                    float lim = best.prim == kInvalid ? tmax : best.t * 1.000001f;
                    if (tri_hit(r, b.Pm(b.idx[3 * t3]), b.Pm(b.idx[3 * t3 + 1]), b.Pm(b.idx[3 * t3 + 2]), 0.0f, lim, t, u,
                                v)) {
                        uint32_t p = first + t3;
                        if (t < best.t || (t == best.t && p < best.prim)) {
                            best.prim = p; best.t = t; best.u = u; best.v = v;
                        }
                    }
                }
            } else {
                stack[sp++] = n.left;
                stack[sp++] = n.right;
            }
        }
    }
    return best;
}

static bool any_instanced(const Scene &sc, const RayPre &rw, float tmax) {
    for (uint32_t i = 0; i < sc.s->instance_count; ++i) {
        if (!box_hit(rw, &sc.inst_lo[3 * i], &sc.inst_hi[3 * i], tmax * 1.000001f)) continue;
        const RayPre r = instance_ray(&sc.inst_rows[12 * i], rw);
        const Scene::MeshBvh &b = sc.mesh_bvh[sc.s->inst_mesh[i]];
        uint32_t stack[128];
        int sp = 0;
        stack[sp++] = 0;
        while (sp) {
            const Scene::Node &n = b.nodes[stack[--sp]];
            if (!box_hit(r, n.lo, n.hi, tmax * 1.000001f)) continue;
            if (n.count) {
                for (uint32_t k = n.first; k < n.first + n.count; ++k) {
                    uint32_t t3 = b.order[k];
                    float t, u, v;
                    if (tri_hit(r, b.Pm(b.idx[3 * t3]), b.Pm(b.idx[3 * t3 + 1]), b.Pm(b.idx[3 * t3 + 2]), 0.0f, tmax, t,
                                u, v))
                        return true;
                }
            } else {
                stack[sp++] = n.left;
                stack[sp++] = n.right;
            }
        }
    }
    return false;
}

// Closest hit over t in (0, tmax); exact ties in t go to the lower primitive id.
static HitRec closest(const Scene &sc, const RayPre &r, float tmax) {
    if (sc.s->two_level) return closest_instanced(sc, r, tmax);
    HitRec best;
    best.t = tmax;
    uint32_t stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
        const Scene::Node &n = sc.nodes[stack[--sp]];
        if (!box_hit(r, n.lo, n.hi, best.t * 1.000001f)) continue;
        if (n.count) {
            for (uint32_t i = n.first; i < n.first + n.count; ++i) {
                uint32_t p = sc.order[i];
                float t, u, v;
                float lim = best.prim == kInvalid ? tmax : best.t * 1.000001f;
                if (tri_hit(r, sc.P(sc.s->idx[3 * p]), sc.P(sc.s->idx[3 * p + 1]), sc.P(sc.s->idx[3 * p + 2]), 0.0f, lim,
                            t, u, v)) {
                    if (t < best.t || (t == best.t && p < best.prim)) {
                        best.prim = p; best.t = t; best.u = u; best.v = v;
                    }
                }
            }
        } else {
            stack[sp++] = n.left;
            stack[sp++] = n.right;
        }
    }
    return best;
}

static bool any_hit(const Scene &sc, const RayPre &r, float tmax) {
    if (sc.s->two_level) return any_instanced(sc, r, tmax);
    uint32_t stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
        const Scene::Node &n = sc.nodes[stack[--sp]];
        if (!box_hit(r, n.lo, n.hi, tmax * 1.000001f)) continue;
        if (n.count) {
            for (uint32_t i = n.first; i < n.first + n.count; ++i) {
                uint32_t p = sc.order[i];
                float t, u, v;
                if (tri_hit(r, sc.P(sc.s->idx[3 * p]), sc.P(sc.s->idx[3 * p + 1]), sc.P(sc.s->idx[3 * p + 2]), 0.0f, tmax,
                            t, u, v))
                    return true;
            }
        } else {
            stack[sp++] = n.left;
            stack[sp++] = n.right;
        }
    }
    return false;
}

// ----- surface interaction (geometry.cpp:78-165, interaction.h:87-110) --------
struct Frame {
    V3 x, y, z;
    V3 to_local(V3 v) const { return {dot(v, x), dot(v, y), dot(v, z)}; }
    V3 to_world(V3 v) const { return add(add(mul(x, v.x), mul(y, v.y)), mul(z, v.z)); }
};
struct It {
    V3 pos, ng, wo;
    Frame sh;
    float tu, tv;  // interpolated texture coordinates
    float area;
    uint32_t prim, mat, light;
};
static It interaction(const Scene &sc, uint32_t prim, float u, float v, V3 ray_dir) {
    It it;
    const uint32_t *ix = sc.s->idx + 3 * prim;
    V3 p0 = sc.P(ix[0]), p1 = sc.P(ix[1]), p2 = sc.P(ix[2]);
    float w = 1.0f - u - v;
    it.pos = add(add(mul(p0, w), mul(p1, u)), mul(p2, v));
    V3 dp02 = sub(p0, p2), dp12 = sub(p1, p2);
    V3 ng_un = cross(dp02, dp12);
    it.area = 0.5f * len(ng_un);
    it.ng = normalize(ng_un);
    const float *uv = sc.s->uv;
    float u0 = uv[2 * ix[0]], v0 = uv[2 * ix[0] + 1], u1 = uv[2 * ix[1]], v1 = uv[2 * ix[1] + 1], u2 = uv[2 * ix[2]],
          v2 = uv[2 * ix[2] + 1];
    it.tu = u0 * w + u1 * u + u2 * v;
    it.tv = v0 * w + v1 * u + v2 * v;
    float du02 = u0 - u2, dv02 = v0 - v2, du12 = u1 - u2, dv12 = v1 - v2;
    float det = du02 * dv12 - dv02 * du12;
    V3 dp_dv = std::fabs(det) < 1e-8f ? normalize(sub(p2, p0)) : mul(sub(mul(dp12, du02), mul(dp02, du12)), 1.0f / det);
    V3 n = add(add(mul(sc.N(ix[0]), w), mul(sc.N(ix[1]), u)), mul(sc.N(ix[2]), v));
    V3 ns = (n.x == 0.0f && n.y == 0.0f && n.z == 0.0f) ? it.ng : normalize(n);
    V3 x = normalize(cross(ns, dp_dv));
    V3 y = normalize(cross(ns, x));
    it.sh = {x, y, ns};
    it.wo = normalize(neg(ray_dir));
    it.prim = prim;
    const Instance &in = sc.inst[sc.s->prim_inst[prim]];
    it.mat = in.mat_id;
    it.light = in.light_id;
    return it;
}

// ----- emitters (area.cpp:91-149, light.cpp, lightsampler.cpp:159-267) --------
static void emitter(const AreaLight &L, const Swl &w, float *out) {
    const Tables &T = tables();
    if (is_rgb(w)) {
        for (int i = 0; i < w.n; ++i) out[i] = L.rgb_avg[i < 3 ? i : 2];
        return;
    }
    for (int i = 0; i < w.n; ++i) {
        float l = w.lambda[i];
        float e = L.kind == 0 ? sigmoid_poly(L.coef, l) * L.coef[3] * spd_eval(T.d65, 94, l) : planck(l, L.coef[0]) * L.coef[1];
        out[i] = e * L.scale;
    }
}

static uint32_t alias_sample(const Alias *tab, uint32_t size, float u, float *u_remap) {
    u = u * static_cast<float>(size);
    uint32_t idx = std::min(static_cast<uint32_t>(u), size - 1u);
    u = std::min(u - static_cast<float>(idx), kOneMinusEps);
    const Alias &e = tab[idx];
    bool keep = u < e.prob;
    if (u_remap) *u_remap = keep ? std::min(u / e.prob, kOneMinusEps) : std::min((1.0f - u) / (1.0f - e.prob), kOneMinusEps);
    return keep ? idx : e.alias;
}

static float pdf_wi(float pdf_pos, V3 ng, V3 w) {
    float c = std::fabs(dot(ng, normalize(w)));
    float r = pdf_pos * dot(w, w) / c;
    return (std::isinf(r) || std::isnan(r)) ? 0.0f : r;
}

static float light_pmf(const Scene &sc, uint32_t li) {
    return sc.ip.light_sampler == 1 ? sc.s->light_pmf[li] : 1.0f / static_cast<float>(sc.ip.light_count);
}

// ----- spherical environment (spherical.cpp, alias2d.cpp, hero.cpp:92-141) ----
static V3 mat_vec(const float (*m)[4], V3 v) {
    return {m[0][0] * v.x + m[1][0] * v.y + m[2][0] * v.z, m[0][1] * v.x + m[1][1] * v.y + m[2][1] * v.z,
            m[0][2] * v.x + m[1][2] * v.y + m[2][2] * v.z};
}

// RGBToSpectrumTable::decode_albedo (hero.cpp:92-133): sigmoid coefficients
// of the colour clamped to [0, 1], by the table's trilinear lookup.
static void decode_albedo(const float *table, const float rgb[3], float c[3]) {
    float q[3];
    for (int k = 0; k < 3; ++k) q[k] = std::min(std::max(rgb[k], 0.0f), 1.0f);
    if (q[0] == q[1] && q[1] == q[2]) {
        c[0] = c[1] = 0.0f;
        c[2] = (q[0] - 0.5f) / std::sqrt(q[0] * (1.0f - q[0]));
        return;
    }
    const uint32_t res = 64;
    uint32_t mc = (q[0] > q[1]) ? ((q[0] > q[2]) ? 0u : 2u) : ((q[1] > q[2]) ? 1u : 2u);
    float z = q[mc];
    float x = q[(mc + 1) % 3] * (res - 1u) / z;
    float y = q[(mc + 2) % 3] * (res - 1u) / z;
    auto iss = [](float v) { return 0.5f - std::sin(std::asin(1.0f - 2.0f * v) * (1.0f / 3.0f)); };
    float zz = iss(iss(z)) * (res - 1u);
    uint32_t xi = std::min(static_cast<uint32_t>(x), res - 2), yi = std::min(static_cast<uint32_t>(y), res - 2),
             zi = std::min(static_cast<uint32_t>(zz), res - 2);
    float dx = x - xi, dy = y - yi, dz = zz - zi;
    auto L = [](float t, float a, float bb) { return a + t * (bb - a); };
    for (int i = 0; i < 3; ++i) {
        auto co = [&](int ox, int oy, int oz) {
            return table[((((size_t)mc * res + (zi + oz)) * res + (yi + oy)) * res + (xi + ox)) * 4 + i];
        };
        c[i] = L(dz, L(dy, L(dx, co(0, 0, 0), co(1, 0, 0)), L(dx, co(0, 1, 0), co(1, 1, 0))),
                 L(dy, L(dx, co(0, 0, 1), co(1, 0, 1)), L(dx, co(0, 1, 1), co(1, 1, 1))));
    }
}

// RGBToSpectrumTable::decode_unbound (hero.cpp:135-141): the coefficients of
// rgb / (2 max) and the scale 2 max in c[3].
static void decode_unbound(const float *table, float r, float g, float b, float c[4]) {
    float rgb[3] = {std::max(r, 0.0f), std::max(g, 0.0f), std::max(b, 0.0f)};
    float m = std::max(rgb[0], std::max(rgb[1], rgb[2]));
    float sc = 2.0f * m;
    float q[3];
    for (int k = 0; k < 3; ++k) q[k] = sc == 0.0f ? 0.0f : rgb[k] / sc;
    c[3] = sc;
    decode_albedo(table, q, c);
}

// The `image` shader node's lookup (shadernodes/image.cpp:80-88): bilinear
// between the four nearest texel centres ((i + 0.5) / size), both axes
// repeating, row 0 of the file at v = 0.
static void texture_rgb(const Scene &sc, uint32_t id, float u, float v, float rgb[3]) {
    const uint32_t *r = sc.s->textures + 4 * id;
    const int W = static_cast<int>(r[1]), H = static_cast<int>(r[2]);
    const float *t = sc.s->tex_texels + 4 * static_cast<size_t>(r[0]);
    float x = (u - std::floor(u)) * W - 0.5f, y = (v - std::floor(v)) * H - 0.5f;
    float fx = std::floor(x), fy = std::floor(y);
    float tx = x - fx, ty = y - fy;
    int x0 = static_cast<int>(fx), y0 = static_cast<int>(fy);
    int x1 = x0 + 1, y1 = y0 + 1;
    auto wrap = [](int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); };
    x0 = wrap(x0, W);
    x1 = wrap(x1, W);
    y0 = wrap(y0, H);
    y1 = wrap(y1, H);
    for (int c = 0; c < 3; ++c) {
        float a = t[(y0 * W + x0) * 4 + c], b = t[(y0 * W + x1) * 4 + c];
        float cc = t[(y1 * W + x0) * 4 + c], d = t[(y1 * W + x1) * 4 + c];
        float top = a + tx * (b - a), bot = cc + tx * (d - cc);
        rgb[c] = top + ty * (bot - top);
    }
}

static void env_L(const Scene &sc, float u, float v, const Swl &w, float *out) {
    const int W = static_cast<int>(sc.env.width), H = static_cast<int>(sc.env.height);
    float x = u * W - 0.5f, y = v * H - 0.5f;
    float fx = std::floor(x), fy = std::floor(y);
    float tx = x - fx, ty = y - fy;
    int x0 = static_cast<int>(fx), y0 = static_cast<int>(fy);
    int x1 = ((x0 + 1) % W + W) % W;
    x0 = (x0 % W + W) % W;
    int y1 = std::min(std::max(y0 + 1, 0), H - 1);
    y0 = std::min(std::max(y0, 0), H - 1);
    const float *t = sc.s->env_tex;
    float rgb[3];
    for (int c = 0; c < 3; ++c) {
        float a = t[(y0 * W + x0) * 4 + c], b = t[(y0 * W + x1) * 4 + c];
        float cc = t[(y1 * W + x0) * 4 + c], d = t[(y1 * W + x1) * 4 + c];
        float top = a + tx * (b - a), bot = cc + tx * (d - cc);
        rgb[c] = top + ty * (bot - top);
    }
    if (is_rgb(w)) {
        for (int i = 0; i < w.n; ++i) out[i] = rgb[i < 3 ? i : 2] * sc.env.scale;
        return;
    }
    float co[4];
    decode_unbound(sc.s->rgb2spec, rgb[0], rgb[1], rgb[2], co);
    for (int i = 0; i < w.n; ++i)
        out[i] = sigmoid_poly(co, w.lambda[i]) * co[3] * spd_eval(tables().d65, 94, w.lambda[i]) * sc.env.scale;
}

static float env_pdf_map(const Scene &sc, float u, float v) {
    uint32_t W = sc.env.width, H = sc.env.height;
    uint32_t iu = std::min(static_cast<uint32_t>(std::max(u * W, 0.0f)), W - 1);
    uint32_t iv = std::min(static_cast<uint32_t>(std::max(v * H, 0.0f)), H - 1);
    return sc.env.integral > 0.0f ? sc.s->env_cond_func[iv * W + iu] / sc.env.integral : 0.0f;
}

// SphericalMap::evaluate_wi for an escaped ray direction.
static void env_eval(const Scene &sc, V3 dir, const Swl &w, float *L, float &pdf) {
    V3 local = mat_vec(sc.env.w2o, dir);
    float theta = std::acos(std::min(std::max(local.z, -1.0f), 1.0f));
    float phi = std::atan2(local.y, local.x);
    if (phi < 0.0f) phi += 2.0f * kPi;
    float u = phi * (1.0f / (2.0f * kPi)), v = theta * kInvPi;
    float st = std::sin(theta);
    env_L(sc, u, v, w, L);
    float p = env_pdf_map(sc, u, v) / (2.0f * kPi * kPi * st);
    pdf = st == 0.0f ? 0.0f : p;
}

// Projector::Le (projector.cpp:112-125): the reference point in the
// light's frame (the 3 x 4 world-to-light rows of its SPD-table block), its
// squared distance there and the colour slot at the projected uv inside the
// frustum: a texture decoded as an illumination, or the constant emitter.
static void projector_L(const Scene &sc, const AreaLight &L, V3 p_ref, const Swl &w, float *out) {
    const float *b = sc.s->spd + L.alias_offset;
    V3 p = {b[0] * p_ref.x + b[1] * p_ref.y + b[2] * p_ref.z + b[3],
            b[4] * p_ref.x + b[5] * p_ref.y + b[6] * p_ref.z + b[7],
            b[8] * p_ref.x + b[9] * p_ref.y + b[10] * p_ref.z + b[11]};
    float d2 = dot(p, p);
    float u = (p.x / p.z + b[12]) / (2.0f * b[12]);
    float v = (p.y / p.z + b[13]) / (2.0f * b[13]);
    for (int i = 0; i < w.n; ++i) out[i] = 0.0f;
    if (!(p.z > 0.0f && u >= 0.0f && u <= 1.0f && v >= 0.0f && v <= 1.0f)) return;
    uint32_t tex;
    std::memcpy(&tex, &b[14], 4);
    if (tex == kInvalid) {
        emitter(L, w, out);
        for (int i = 0; i < w.n; ++i) out[i] *= 1.0f / d2;
        return;
    }
    float rgb[3];
    texture_rgb(sc, tex, u, v, rgb);
    for (int c = 0; c < 3; ++c) rgb[c] *= L.coef[c];
    if (is_rgb(w)) {
        for (int i = 0; i < w.n; ++i) out[i] = rgb[i < 3 ? i : 2] * L.scale / d2;
        return;
    }
    float co[4];
    decode_unbound(sc.s->rgb2spec, rgb[0], rgb[1], rgb[2], co);
    for (int i = 0; i < w.n; ++i)
        out[i] = sigmoid_poly(co, w.lambda[i]) * co[3] * spd_eval(tables().d65, 94, w.lambda[i]) * L.scale / d2;
}

// Delta-position light radiance at p_ref (point.cpp:36-41, spot.cpp:47-67,
// projector.cpp:112-125): colour * scale / d^2, times the spot falloff.
static void delta_L(const Scene &sc, const AreaLight &L, V3 p_ref, const Swl &w, float *out) {
    if (L.shape == 3) {
        projector_L(sc, L, p_ref, w, out);
        return;
    }
    V3 lp = {L.pos[0], L.pos[1], L.pos[2]};
    V3 wu = sub(p_ref, lp);
    float g = 1.0f / dot(wu, wu);
    if (L.shape == 2) {
        float ct = dot(V3{L.dir[0], L.dir[1], L.dir[2]}, normalize(wu));
        float c = std::min(std::max(ct, L.cos_angle), L.cos_start);
        float range = L.cos_start - L.cos_angle;
        float f = range > 0.0f ? (c - L.cos_angle) / range : (ct >= L.cos_start ? 1.0f : 0.0f);
        float f2 = f * f;
        g *= f2 * f2;
    }
    emitter(L, w, out);
    for (int i = 0; i < w.n; ++i) out[i] *= g;
}

static float alias_cont(const Alias *tab, uint32_t size, float u, uint32_t &ofs) {
    u = u * static_cast<float>(size);
    uint32_t idx = std::min(static_cast<uint32_t>(u), size - 1u);
    u = std::min(u - static_cast<float>(idx), kOneMinusEps);
    bool keep = u < tab[idx].prob;
    float ur = keep ? std::min(u / tab[idx].prob, kOneMinusEps) : std::min((1.0f - u) / (1.0f - tab[idx].prob), kOneMinusEps);
    ofs = keep ? idx : tab[idx].alias;
    return (static_cast<float>(ofs) + ur) / static_cast<float>(size);
}

// SphericalMap::sample_only (spherical.cpp:127-132): map coordinates only.
static void env_sample_uv(const Scene &sc, float ux, float uy, float &fu, float &fv) {
    uint32_t iv, iu;
    fv = alias_cont(static_cast<const Alias *>(sc.s->env_marginal), sc.env.height, uy, iv);
    fu = alias_cont(static_cast<const Alias *>(sc.s->env_cond) + (size_t)iv * sc.env.width, sc.env.width, ux, iu);
}

// SphericalMap::evaluate_point -> evaluate (spherical.cpp:105-125,134-141):
// radiance, solid-angle pdf from the map's PDF(uv), world direction.
static void env_eval_uv(const Scene &sc, float u, float v, const Swl &w, float *L, float &pdf, V3 &wd) {
    float theta = v * kPi, phi = u * 2.0f * kPi;
    float st = std::sin(theta), ct = std::cos(theta);
    V3 local = {st * std::cos(phi), st * std::sin(phi), ct};
    wd = normalize(mat_vec(sc.env.o2w, local));
    float p = env_pdf_map(sc, u, v) / (2.0f * kPi * kPi * st);
    pdf = std::isinf(p) ? 0.0f : p;
    env_L(sc, u, v, w, L);
}

// Environment::convert_to_bary (spherical.cpp:70-73).
static void env_dir_uv(const Scene &sc, V3 dir, float &u, float &v) {
    V3 local = normalize(mat_vec(sc.env.w2o, dir));
    float theta = std::acos(std::min(std::max(local.z, -1.0f), 1.0f));
    float phi = std::atan2(local.y, local.x);
    if (phi < 0.0f) phi += 2.0f * kPi;
    u = phi * (1.0f / (2.0f * kPi));
    v = theta * kInvPi;
}

struct LS {
    float L[8];
    float pdf;
    V3 p;
};
static LS sample_light(const Scene &sc, const It &it, float ul, float ux, float uy, const Swl &w) {
    LS ls;
    uint32_t n = sc.ip.light_count;
    uint32_t li;
    float pmf_l;
    if (sc.ip.light_sampler == 1) {
        li = alias_sample(sc.light_alias, n, ul, nullptr);
        pmf_l = sc.s->light_pmf[li];
    } else {
        li = static_cast<uint32_t>(std::min(ul * static_cast<float>(n), static_cast<float>(n) - 1.0f));
        pmf_l = 1.0f / static_cast<float>(n);
    }
    if (sc.has_env && li == sc.ip.light_count - 1) {
        // SphericalMap::sample_wi + AliasTable2D::sample_continuous.
        uint32_t W = sc.env.width, H = sc.env.height;
        const Alias *marg = static_cast<const Alias *>(sc.s->env_marginal);
        const Alias *cond = static_cast<const Alias *>(sc.s->env_cond);
        uint32_t iv, iu;
        float fv = alias_cont(marg, H, uy, iv);
        float pdf_v = sc.env.integral > 0.0f ? sc.s->env_marginal_func[iv] / sc.env.integral : 0.0f;
        float fu = alias_cont(cond + (size_t)iv * W, W, ux, iu);
        float iu_int = sc.s->env_marginal_func[iv];
        float pdf_u = iu_int > 0.0f ? sc.s->env_cond_func[(size_t)iv * W + iu] / iu_int : 0.0f;
        float theta = fv * kPi, phi = fu * 2.0f * kPi;
        float st = std::sin(theta), ct = std::cos(theta);
        V3 local = {st * std::cos(phi), st * std::sin(phi), ct};
        V3 wd = normalize(mat_vec(sc.env.o2w, local));
        float p = pdf_u * pdf_v / (2.0f * kPi * kPi * st);
        ls.pdf = (std::isinf(p) ? 0.0f : p) * pmf_l;
        env_L(sc, fu, fv, w, ls.L);
        ls.p = add(it.pos, mul(wd, sc.env.world_diameter));
        return ls;
    }
    const AreaLight &L = sc.lights[li];
    if (L.shape != 0) {
        // Point / spot light (point.cpp:36-41, spot.cpp:47-67): colour * scale
        // / d^2 (times the spot falloff); pdf -pmf marks the delta light.
        delta_L(sc, L, it.pos, w, ls.L);
        ls.pdf = -pmf_l;
        ls.p = V3{L.pos[0], L.pos[1], L.pos[2]};
        return ls;
    }
    float ur = ux;
    uint32_t local = alias_sample(sc.prim_alias + L.alias_offset, L.prim_count, ux, &ur);
    float pmf_p = sc.s->prim_pmf[L.alias_offset + local];
    float su0 = std::sqrt(ur);
    float bu = 1.0f - su0, bv = uy * su0;
    uint32_t prim = L.first_prim + local;
    const uint32_t *ix = sc.s->idx + 3 * prim;
    V3 p0 = sc.P(ix[0]), p1 = sc.P(ix[1]), p2 = sc.P(ix[2]);
    float bw = 1.0f - bu - bv;
    V3 pos = add(add(mul(p0, bw), mul(p1, bu)), mul(p2, bv));
    V3 ng_un = cross(sub(p0, p2), sub(p1, p2));
    float area = 0.5f * len(ng_un);
    V3 ng = normalize(ng_un);
    float pdf_pos = (1.0f / area) * pmf_p;
    V3 wr = sub(it.pos, pos);
    bool front = dot(wr, ng) > 0.0f || L.two_sided;
    if (front) emitter(L, w, ls.L);
    else for (int i = 0; i < w.n; ++i) ls.L[i] = 0.0f;
    ls.pdf = pdf_wi(pdf_pos, ng, wr) * pmf_l;
    ls.p = offset_ray_origin(pos, dot(ng, wr) > 0.0f ? ng : neg(ng));
    return ls;
}

// ----- BSDFs ------------------------------------------------------------------
// Materials: diffuse (diffuse.cpp), black_body (black_body.cpp), metal
// (metal.cpp + ConductorLobe/PureReflectionLobe, lobe.cpp:716-735), glass
// (glass.cpp + DielectricLobe, lobe.cpp:253-450), principled_bsdf
// (principled_bsdf.cpp:352-461: sheen LTC, coat, metallic F82, transmission,
// Schlick specular, diffuse).
// Everything is evaluated in world space through per-lobe local frames the way
// MaterialEvaluator::evaluate/sample do with individual shading normals
// (material.cpp:132-184).
constexpr uint32_t kRefl = 2, kTrans = 4, kDiffRefl = 8 | 2, kGlossyRefl = 16 | 2, kGlossyTrans = 16 | 4, kUnset = 1;

namespace mf {
// microfacet.cpp / microfacet.h, GGX with visible-normal sampling.
static float D(V3 h, float ax, float ay) {
    float x = h.x / ax, y = h.y / ay, z = h.z;
    float l2 = x * x + y * y + z * z;
    return kInvPi / (ax * ay * (l2 * l2));
}
static float lambda(V3 w, float ax, float ay) {
    if (w.z == 0.0f) return 0.0f;
    float t = ((ax * w.x) * (ax * w.x) + (ay * w.y) * (ay * w.y)) / (w.z * w.z);
    return 0.5f * (std::sqrt(1.0f + t) - 1.0f);
}
static float G1(V3 w, float ax, float ay) { return 1.0f / (1.0f + lambda(w, ax, ay)); }
static float G(V3 a, V3 b, float ax, float ay) { return 1.0f / (1.0f + lambda(a, ax, ay) + lambda(b, ax, ay)); }
static V3 sample_wh(V3 wo, float u0, float u1, float ax, float ay) {
    bool flip = wo.z < 0.0f;
    V3 ve = flip ? neg(wo) : wo;
    V3 vh = normalize(v3(ax * ve.x, ay * ve.y, ve.z));
    float ls = vh.x * vh.x + vh.y * vh.y;
    V3 t1 = ls > 1e-7f ? mul(v3(-vh.y, vh.x, 0.0f), 1.0f / std::sqrt(ls)) : v3(1, 0, 0);
    V3 t2 = ls > 1e-7f ? cross(vh, t1) : v3(0, 1, 0);
    float r = std::sqrt(u0), th = 2.0f * kPi * u1;
    float tx = r * std::cos(th), ty = r * std::sin(th);
    float sw = 0.5f * (1.0f + vh.z);
    float a = std::sqrt(std::max(0.0f, 1.0f - tx * tx));
    ty = a + sw * (ty - a);
    V3 nh = add(add(mul(t1, tx), mul(t2, ty)), mul(vh, std::sqrt(std::max(0.0f, 1.0f - (tx * tx + ty * ty)))));
    V3 ne = normalize(v3(ax * nh.x, ay * nh.y, std::max(0.0f, nh.z)));
    return flip ? neg(ne) : ne;
}
static float pdf_wh(V3 wo, V3 h, float ax, float ay) {
    return D(h, ax, ay) * G1(wo, ax, ay) * std::fabs(dot(wo, h)) / std::fabs(wo.z);
}
static float pdf_refl(V3 wo, V3 h, float ax, float ay) { return pdf_wh(wo, h, ax, ay) / (4.0f * std::fabs(dot(wo, h))); }
static float pdf_trans(V3 wo, V3 h, V3 wi, float eta, float ax, float ay) {
    float d = dot(wi, h) * eta + dot(wo, h);
    return pdf_wh(wo, h, ax, ay) * (std::fabs(dot(wi, h)) / (d * d));
}
static float brdf(V3 wo, V3 h, V3 wi, float ax, float ay) {
    return D(h, ax, ay) * G(wo, wi, ax, ay) / std::fabs(4.0f * wo.z * wi.z);
}
static float btdf(V3 wo, V3 h, V3 wi, float eta, float ax, float ay) {
    float num = D(h, ax, ay) * G(wo, wi, ax, ay) * std::fabs(dot(wi, h) * dot(wo, h));
    float d = dot(wi, h) * eta + dot(wo, h);
    float den = d * d * std::fabs(wi.z * wo.z);
    float ft = den == 0.0f ? 0.0f : num / den;
    return ft * (1.0f / (eta * eta));  // radiance transport
}
static V3 reflect(V3 wo, V3 n) { return add(neg(wo), mul(n, 2.0f * dot(wo, n))); }
static bool refract(V3 wi, V3 n, float eta, V3 &wt) {
    float ci = dot(n, wi);
    float s2i = std::max(0.0f, 1.0f - ci * ci);
    float s2t = s2i / (eta * eta);
    float ct = std::sqrt(std::max(0.0f, 1.0f - s2t));
    wt = add(mul(wi, -1.0f / eta), mul(n, ci / eta - ct));
    return s2t < 1.0f;
}
static float fr_dielectric(float c, float eta) {
    float s2i = 1.0f - c * c;
    float s2t = s2i / (eta * eta);
    float ct = std::sqrt(std::max(0.0f, 1.0f - s2t));
    float rp = (eta * c - ct) / (eta * c + ct);
    float rs = (c - eta * ct) / (c + eta * ct);
    return s2t >= 1.0f ? 1.0f : (rp * rp + rs * rs) * 0.5f;
}
// fresnel_complex with Complex<> of src/math/complex.h.
static float fr_conductor(float c, float eta, float k) {
    auto mulc = [](float ar, float ai, float br, float bi, float &r, float &i) { r = ar * br - ai * bi; i = ar * bi + ai * br; };
    auto divc = [](float ar, float ai, float br, float bi, float &r, float &i) {
        float s = 1.0f / (br * br + bi * bi);
        r = s * (ar * br + ai * bi);
        i = s * (ai * br - ar * bi);
    };
    float e2r, e2i;
    mulc(eta, k, eta, k, e2r, e2i);
    float s2r, s2i;
    divc(1.0f - c * c, 0.0f, e2r, e2i, s2r, s2i);
    float zr = 1.0f - s2r, zi = -s2i;
    float n = std::sqrt(zr * zr + zi * zi);
    float t1 = std::sqrt(0.5f * (n + std::fabs(zr)));
    float t2 = 0.5f * zi / t1;
    float ctr = n == 0.0f ? 0.0f : (zr >= 0.0f ? t1 : std::fabs(t2));
    float cti = n == 0.0f ? 0.0f : (zr >= 0.0f ? t2 : std::copysign(t1, zi));
    float ecr = eta * c, eci = k * c;
    float pr, pi;
    divc(ecr - ctr, eci - cti, ecr + ctr, eci + cti, pr, pi);
    float ectr, ecti;
    mulc(eta, k, ctr, cti, ectr, ecti);
    float sr, si;
    divc(c - ectr, -ecti, c + ectr, ecti, sr, si);
    return ((pr * pr + pi * pi) + (sr * sr + si * si)) * 0.5f;
}
}  // namespace mf

#include "../vision_b200/csrc/data/albedo_luts.inc"
#include "../vision_b200/csrc/data/principled_luts.inc"

// MaterialLut::sample: normalised coordinates, linear filter, clamp to edge.
static float lut_axis(float u, int &i0, int &i1) {
    float x = u * 32.0f - 0.5f;
    float fl = std::floor(x);
    int i = static_cast<int>(fl);
    i0 = std::min(std::max(i, 0), 31);
    i1 = std::min(std::max(i + 1, 0), 31);
    return x - fl;
}
static float lut2(const float *t, float u, float v) {
    int x0, x1, y0, y1;
    float fx = lut_axis(u, x0, x1), fy = lut_axis(v, y0, y1);
    float a = t[y0 * 32 + x0] + fx * (t[y0 * 32 + x1] - t[y0 * 32 + x0]);
    float b = t[y1 * 32 + x0] + fx * (t[y1 * 32 + x1] - t[y1 * 32 + x0]);
    return a + fy * (b - a);
}
static float lut3(const float *t, int ch, float u, float v, float w) {
    int x0, x1, y0, y1, z0, z1;
    float fx = lut_axis(u, x0, x1), fy = lut_axis(v, y0, y1), fz = lut_axis(w, z0, z1);
    auto at = [&](int x, int y, int z) { return t[((z * 32 + y) * 32 + x) * ch]; };
    float c00 = at(x0, y0, z0) + fx * (at(x1, y0, z0) - at(x0, y0, z0));
    float c10 = at(x0, y1, z0) + fx * (at(x1, y1, z0) - at(x0, y1, z0));
    float c01 = at(x0, y0, z1) + fx * (at(x1, y0, z1) - at(x0, y0, z1));
    float c11 = at(x0, y1, z1) + fx * (at(x1, y1, z1) - at(x0, y1, z1));
    float c0 = c00 + fy * (c10 - c00), c1 = c01 + fy * (c11 - c01);
    return c0 + fz * (c1 - c0);
}
// 2D table with `ch` channels per texel, index [y][x][c].
static float lut2c(const float *t, int ch, int c, float u, float v) {
    int x0, x1, y0, y1;
    float fx = lut_axis(u, x0, x1), fy = lut_axis(v, y0, y1);
    auto at = [&](int x, int y) { return t[(y * 32 + x) * ch + c]; };
    float a = at(x0, y0) + fx * (at(x1, y0) - at(x0, y0));
    float b = at(x0, y1) + fx * (at(x1, y1) - at(x0, y1));
    return a + fy * (b - a);
}
static const float *kLutPure = VS_ALBEDO_LUTS;
static const float *kLutDiel = VS_ALBEDO_LUTS + 1024;
static const float *kLutDielInv = VS_ALBEDO_LUTS + 1024 + 65536;
static const float *kLutSpec = VS_ALBEDO_LUTS + 1024 + 131072;
static const float *kLutCoat = VS_COAT_LUT;     // CoatLobe albedo (precomputed_table.h)
static const float *kLutSheen = VS_SHEEN_LTC;   // SheenLTC Approximate fits (ltc_sheen_table.h)

struct Eval {
    float f[8];
    float pdf;
    uint32_t flags;
};

// A lobe of the material's lobe set.
struct Lobe {
    enum Kind { Lambert, MicrofacetRefl, Dielectric, NoScatter, Substrate, Plastic, Sheen } kind;
    // Fresnel of a microfacet lobe; a Dielectric lobe uses Schlick (F0 in fa,
    // eta[0]) or, by default, the dielectric Fresnel at each eta[i].
    enum Fr { Conductor, Schlick, F82, One, DielectricFr } fresnel = One;
    float ax = 1, ay = 1;
    bool compensate = false;
    float kr[8], fa[8], fb[8];
    float eta0 = 1.0f;
    float eta[8];
    float sample_weight = 1.0f;
    float weight = 1.0f;               // WeightedLobe::weight: scales f in the lobe set
    float ltc_a = 1.0f, ltc_b = 0.0f;  // Sheen: the LTC matrix entries
};

struct Bsdf {
    int n = 1;
    Frame fr;
    V3 ng;
    Lobe lobes[12];  // a mix of two principled materials holds two lobe sets
    int count = 0;
    bool lobe_set = false;  // LobeSet: world-space hemisphere factors and a 1D lobe choice
    bool dispersive = false;
};

static void fresnel_eval(const Lobe &l, int n, float c, float *F) {
    for (int i = 0; i < n; ++i) {
        if (l.fresnel == Lobe::Conductor) F[i] = mf::fr_conductor(c, l.fa[i], l.fb[i]);
        else if (l.fresnel == Lobe::Schlick) {
            float fr = mf::fr_dielectric(c, l.eta0);
            float f0 = ((l.eta0 - 1.0f) / (l.eta0 + 1.0f)) * ((l.eta0 - 1.0f) / (l.eta0 + 1.0f));
            float t = std::min(std::max((fr - f0) / (1.0f - f0), 0.0f), 1.0f);
            F[i] = l.fa[i] + t * (1.0f - l.fa[i]);
        } else if (l.fresnel == Lobe::F82) {
            float mu = std::min(std::max(1.0f - c, 0.0f), 1.0f);
            float mu5 = mu * mu * mu * mu * mu;
            float fs = l.fa[i] + mu5 * (1.0f - l.fa[i]);
            F[i] = std::min(std::max(fs - l.fb[i] * c * mu5 * mu, 0.0f), 1.0f);
        } else if (l.fresnel == Lobe::DielectricFr) {
            F[i] = mf::fr_dielectric(c, l.eta0);  // FresnelDielectric (fresnel.h:74-90)
        } else {
            F[i] = 1.0f;
        }
    }
}

// Fresnel of a dielectric lobe: per-wavelength dielectric (glass), or
// FresnelSchlick (fresnel.h:60-67) with F0 = fa and eta[0] (the principled
// transmission lobe).
static void diel_fresnel(const Lobe &l, int n, float c, float *F) {
    if (l.fresnel == Lobe::Schlick) {
        float fr = mf::fr_dielectric(c, l.eta[0]);
        float f0 = ((l.eta[0] - 1.0f) / (l.eta[0] + 1.0f)) * ((l.eta[0] - 1.0f) / (l.eta[0] + 1.0f));
        float t = std::min(std::max((fr - f0) / (1.0f - f0), 0.0f), 1.0f);
        for (int i = 0; i < n; ++i) F[i] = l.fa[i] + t * (1.0f - l.fa[i]);
        return;
    }
    for (int i = 0; i < n; ++i) F[i] = mf::fr_dielectric(c, l.eta[i]);
}

// Local evaluation of one lobe: f (without the cosine), pdf, flags.
static void lobe_eval(const Lobe &l, int n, V3 wo, V3 wi, float *f, float &pdf, uint32_t &flags, float &eta_out) {
    eta_out = 1.0f;
    if (l.kind == Lobe::Lambert) {
        bool s = wo.z * wi.z > 0.0f;
        for (int i = 0; i < n; ++i) f[i] = s ? l.kr[i] * kInvPi : 0.0f;
        pdf = s ? std::fabs(wi.z) * kInvPi : 0.0f;
        flags = kDiffRefl;
    } else if (l.kind == Lobe::MicrofacetRefl) {
        flags = kGlossyRefl;
        if (!(wo.z * wi.z > 0.0f)) {
            for (int i = 0; i < n; ++i) f[i] = 0.0f;
            pdf = 0.0f;
            return;
        }
        V3 h = normalize(add(wo, wi));
        V3 hf = h.z < 0.0f ? neg(h) : h;
        float F[8];
        fresnel_eval(l, n, std::fabs(dot(wo, hf)), F);
        float b = mf::brdf(wo, hf, wi, l.ax, l.ay);
        float comp = l.compensate ? 1.0f / lut2(kLutPure, std::sqrt(l.ax * l.ay), wo.z) : 1.0f;
        for (int i = 0; i < n; ++i) f[i] = b * F[i] * l.kr[i] * comp;
        pdf = mf::pdf_refl(wo, h, l.ax, l.ay);
    } else if (l.kind == Lobe::Plastic) {
        // PlasticLobe::evaluate_local_impl (plastic.cpp:27-46): no hemisphere
        // test; kr = Rd, Schlick F (fa = F0(ior) * Rs, eta0 = ior) at |wh . wo|.
        flags = kRefl;
        V3 h = normalize(add(wo, wi));
        float F[8];
        fresnel_eval(l, n, std::fabs(dot(h, wo)), F);
        float b = mf::brdf(wo, h, wi, l.ax, l.ay);
        float fs = 0.0f;
        for (int i = 0; i < n; ++i) {
            f[i] = l.kr[i] * kInvPi * (1.0f - F[i]) + b * F[i];
            fs += F[i];
        }
        float fa = fs * (1.0f / n);
        float pd = std::fabs(wi.z) * kInvPi;
        pdf = pd + fa * (mf::pdf_refl(wo, h, l.ax, l.ay) - pd);
    } else if (l.kind == Lobe::Substrate) {
        // FresnelBlend (substrate.cpp:12-72) through BxDF::safe_evaluate:
        // kr = Rd, fa = Rs; specular picked with F_dielectric(|cos wo|, 1.5).
        flags = kRefl;
        if (!(wo.z * wi.z > 0.0f)) {
            for (int i = 0; i < n; ++i) f[i] = 0.0f;
            pdf = 0.0f;
            return;
        }
        V3 h = normalize(add(wi, wo));
        float ci = std::fabs(wi.z), co = std::fabs(wo.z);
        float d = mf::D(h, l.ax, l.ay) / (4.0f * std::fabs(dot(wi, h)) * std::max(ci, co));
        auto p5 = [](float x) { float x2 = x * x; return x2 * x2 * x; };
        float w = p5(std::min(std::max(1.0f - dot(wi, h), 0.0f), 1.0f));
        float g = (28.0f / (23.0f * kPi)) * (1.0f - p5(1.0f - 0.5f * ci)) * (1.0f - p5(1.0f - 0.5f * co));
        for (int i = 0; i < n; ++i) f[i] = d * (l.fa[i] + w * (1.0f - l.fa[i])) + g * l.kr[i] * (1.0f - l.fa[i]);
        float fr = mf::fr_dielectric(co, 1.5f);
        float pd = ci * kInvPi;
        pdf = pd + fr * (mf::pdf_refl(wo, h, l.ax, l.ay) - pd);
    } else if (l.kind == Lobe::Sheen) {
        // SheenLTC::evaluate_local_impl (principled_bsdf.cpp:61-75):
        // eval_ltc(wi) = cosine pdf of M^-1 wi / |M^-1 wi| times a^2 / |M^-1 wi|^3.
        flags = kGlossyRefl;
        V3 w = {l.ltc_a * wi.x + l.ltc_b * wi.z, l.ltc_a * wi.y, wi.z};
        float L = len(w);
        w = {w.x / L, w.y / L, w.z / L};
        float jac = (l.ltc_a * l.ltc_a) / (L * L * L);
        float ltc = w.z * kInvPi * jac;
        bool below = wi.z < 0.0f || wo.z < 0.0f;
        for (int i = 0; i < n; ++i) f[i] = below ? 0.0f : (ltc * l.kr[i]) / wi.z;
        pdf = ltc;
    } else if (l.kind == Lobe::Dielectric) {
        bool refl = wo.z * wi.z > 0.0f;
        float e0 = l.eta[0];
        float ep = refl ? 1.0f : e0;
        eta_out = ep;
        V3 h = normalize(add(wo, mul(wi, ep)));
        if (dot(h, wo) < 0.0f) h = neg(h);
        float F[8], T[8];
        diel_fresnel(l, n, std::fabs(dot(h, wo)), F);
        float sf = 0, st = 0;
        for (int i = 0; i < n; ++i) {
            sf += F[i];
            st += (1.0f - F[i]) * l.kr[i] + F[i];
        }
        float pr = (sf / n) / (st / n);
        float e = e0 > 1.0f ? e0 : 1.0f / e0;
        float comp = 1.0f / lut3(e0 > 1.0f ? kLutDiel : kLutDielInv, 2, std::sqrt(std::sqrt(l.ax * l.ay)),
                                 std::fabs(wo.z), (e - 1.003f) / (5.0f - 1.003f));
        if (refl) {
            float b = mf::brdf(wo, h, wi, l.ax, l.ay);
            for (int i = 0; i < n; ++i) f[i] = F[i] * b * comp;
            pdf = mf::pdf_refl(wo, h, l.ax, l.ay) * pr;
            flags = kGlossyRefl;
        } else {
            V3 h2 = normalize(add(wo, mul(wi, e0)));
            float bt = mf::btdf(wo, h2, wi, e0, l.ax, l.ay);
            for (int i = 0; i < n; ++i) {
                T[i] = (1.0f - F[i]) * l.kr[i];
                f[i] = T[i] * bt * comp;
            }
            pdf = mf::pdf_trans(wo, h, wi, e0, l.ax, l.ay) * (1.0f - pr);
            flags = kGlossyTrans;
        }
    } else {
        for (int i = 0; i < n; ++i) f[i] = 0.0f;
        pdf = 1.0f;
        flags = kUnset;
    }
}

// MaterialEvaluator::evaluate with individual shading normals.
static Eval bsdf_eval(const Bsdf &b, V3 wo_w, V3 wi_w, float *eta_out) {
    Eval e;
    V3 wo = b.fr.to_local(wo_w), wi = b.fr.to_local(wi_w);
    float ac = std::fabs(wi.z);
    float eta = 1.0f;
    if (!b.lobe_set) {
        lobe_eval(b.lobes[0], b.n, wo, wi, e.f, e.pdf, e.flags, eta);
        for (int i = 0; i < b.n; ++i) e.f[i] *= ac;
    } else {
        for (int i = 0; i < b.n; ++i) e.f[i] = 0.0f;
        e.pdf = 0.0f;
        e.flags = 0;
        bool same = wo.z * wi.z > 0.0f;
        for (int k = 0; k < b.count; ++k) {
            const Lobe &l = b.lobes[k];
            float f[8], p;
            uint32_t fl;
            float et;
            lobe_eval(l, b.n, wo, wi, f, p, fl, et);
            float factor = (l.kind == Lobe::Dielectric || same) ? 1.0f : 0.0f;
            for (int i = 0; i < b.n; ++i) e.f[i] += (f[i] * ac) * (l.weight * factor);
            e.pdf += p * l.sample_weight * factor;
            e.flags |= fl;
            if (l.kind == Lobe::Dielectric) eta = et;
        }
    }
    if (eta_out) *eta_out = eta;
    bool same_g = dot(wo_w, b.ng) * dot(wi_w, b.ng) > 0.0f;
    if (same_g == ((e.flags & kTrans) != 0)) e.pdf = 0.0f;
    return e;
}

static V3 lobe_sample(const Lobe &l, int n, V3 wo, Sampler &smp, bool &valid) {
    valid = true;
    if (l.kind == Lobe::Lambert) {
        float u0 = smp.next(), u1 = smp.next();
        float r = std::sqrt(u0), th = 2.0f * kPi * u1;
        float dx = r * std::cos(th), dy = r * std::sin(th);
        float z = std::sqrt(std::max(0.0f, 1.0f - dx * dx - dy * dy));
        return {dx, dy, wo.z < 0.0f ? -z : z};
    }
    if (l.kind == Lobe::MicrofacetRefl) {
        float u0 = smp.next(), u1 = smp.next();
        V3 h = mf::sample_wh(wo, u0, u1, l.ax, l.ay);
        V3 wi = mf::reflect(wo, h);
        valid = wo.z * wi.z > 0.0f;
        return wi;
    }
    if (l.kind == Lobe::Plastic) {
        // PlasticLobe::sample_wi_local_impl (plastic.cpp:61-78).
        float u0 = smp.next(), u1 = smp.next();
        V3 h = mf::sample_wh(wo, u0, u1, l.ax, l.ay);
        float F[8], fs = 0.0f;
        fresnel_eval(l, n, std::fabs(wo.z), F);
        for (int i = 0; i < n; ++i) fs += F[i];
        float uc = smp.next();
        if (uc < fs * (1.0f / n)) {
            V3 wi = mf::reflect(wo, h);
            valid = wo.z * wi.z > 0.0f;
            return wi;
        }
        float v0 = smp.next(), v1 = smp.next();
        float r = std::sqrt(v0), th = 2.0f * kPi * v1;
        float dx = r * std::cos(th), dy = r * std::sin(th);
        return {dx, dy, std::sqrt(std::max(0.0f, 1.0f - dx * dx - dy * dy))};
    }
    if (l.kind == Lobe::Substrate) {
        // FresnelBlend::sample_wi (substrate.cpp:55-71): remapped u.x picks
        // the microfacet or the cosine-hemisphere direction; always valid.
        float u0 = smp.next(), u1 = smp.next();
        float fr = mf::fr_dielectric(std::fabs(wo.z), 1.5f);
        if (u0 < fr) {
            u0 = u0 / fr;
            return mf::reflect(wo, mf::sample_wh(wo, u0, u1, l.ax, l.ay));
        }
        u0 = (u0 - fr) / (1.0f - fr);
        float r = std::sqrt(u0), th = 2.0f * kPi * u1;
        float dx = r * std::cos(th), dy = r * std::sin(th);
        float z = std::sqrt(std::max(0.0f, 1.0f - dx * dx - dy * dy));
        return {dx, dy, wo.z < 0.0f ? -z : z};
    }
    if (l.kind == Lobe::Sheen) {
        // SheenLTC::sample_wi_local_impl (principled_bsdf.cpp:101-110): a
        // cosine-hemisphere direction through M, normalised.
        float u0 = smp.next(), u1 = smp.next();
        float r = std::sqrt(u0), th = 2.0f * kPi * u1;
        float dx = r * std::cos(th), dy = r * std::sin(th);
        float z = std::sqrt(std::max(0.0f, 1.0f - dx * dx - dy * dy));
        return normalize({dx / l.ltc_a - z * l.ltc_b / l.ltc_a, dy / l.ltc_a, z});
    }
    // Dielectric: microfacet normal (2D), then reflect/refract choice (1D).
    float u0 = smp.next(), u1 = smp.next();
    V3 h = mf::sample_wh(wo, u0, u1, l.ax, l.ay);
    float F[8], sf = 0, st = 0;
    diel_fresnel(l, n, std::fabs(dot(wo, h)), F);
    for (int i = 0; i < n; ++i) {
        sf += F[i];
        st += (1.0f - F[i]) * l.kr[i] + F[i];
    }
    float uc = smp.next();
    V3 wi;
    if (uc < (sf / n) / (st / n)) {
        wi = mf::reflect(wo, h);
        valid = wo.z * wi.z > 0.0f;
    } else {
        bool ok = mf::refract(wo, h, l.eta[0], wi);
        valid = ok && !(wo.z * wi.z > 0.0f);
    }
    return wi;
}

// Lobe::sample / LobeSet::sample_wi_impl + MaterialEvaluator::sample.
static Eval bsdf_sample(const Bsdf &b, V3 wo_w, Sampler &smp, V3 &wi_w, float &eta, bool no_scatter) {
    Eval e;
    if (no_scatter) {
        wi_w = wo_w;
        for (int i = 0; i < b.n; ++i) e.f[i] = 0.0f;
        e.pdf = 1.0f;
        e.flags = kDiffRefl;
        eta = 1.0f;
        return e;
    }
    V3 wo = b.fr.to_local(wo_w);
    bool valid;
    V3 wi;
    if (!b.lobe_set) {
        wi = lobe_sample(b.lobes[0], b.n, wo, smp, valid);
    } else {
        float uc = smp.next();
        smp.next();
        smp.next();
        int strategy = 0;
        float sum = 0.0f;
        for (int k = 0; k < b.count; ++k) {
            if (uc > sum) strategy = k;
            sum += b.lobes[k].sample_weight;
        }
        wi = lobe_sample(b.lobes[strategy], b.n, wo, smp, valid);
    }
    wi_w = b.fr.to_world(wi);
    e = bsdf_eval(b, wo_w, wi_w, &eta);
    if (!valid) e.pdf = 0.0f;
    return e;
}

static float spd_of(const float *spd, uint32_t off, float lambda) {
    return spd_eval(spd + off + 1, static_cast<int>(spd[off]), lambda);
}

// A material's colour slot (ShaderNodeSlot::eval_albedo_spectrum,
// shader_node.cpp:299-303): the record's constant, or (flag 32) the texture
// lookup at the hit's uv times the constant factor held in coef as RGB,
// decoded as an albedo (the RGB spectrum keeps the colour itself).
static void colour(const Scene &sc, const Material &m, const It &it, const Swl &w, float *out) {
    if (!(m.flags & 32u)) {
        for (int i = 0; i < w.n; ++i) out[i] = alb(m.coef, w, i);
        return;
    }
    uint32_t id;
    std::memcpy(&id, &m.p[7], 4);
    float rgb[3];
    texture_rgb(sc, id, it.tu, it.tv, rgb);
    for (int c = 0; c < 3; ++c) rgb[c] *= m.coef[c];
    if (is_rgb(w)) {
        for (int i = 0; i < w.n; ++i) out[i] = rgb[i < 3 ? i : 2];
        return;
    }
    float c[3];
    decode_albedo(sc.s->rgb2spec, rgb, c);
    for (int i = 0; i < w.n; ++i) out[i] = sigmoid_poly(c, w.lambda[i]);
}

// Material::create_evaluator for the supported plugins.
static Bsdf make_bsdf(const Scene &sc, const Material &m, const It &it, const Swl &w) {
    Bsdf b;
    float col[8];
    colour(sc, m, it, w, col);
    b.n = w.n;
    b.fr = it.sh;
    b.ng = it.ng;
    b.dispersive = (m.flags & 1u) != 0 && !is_rgb(w);
    Lobe &l0 = b.lobes[0];
    b.count = 1;
    if (m.type == 0) {
        l0.kind = Lobe::Lambert;
        for (int i = 0; i < w.n; ++i) l0.kr[i] = col[i];
    } else if (m.type == 2 && (m.flags & 64u)) {
        // metallic: MetallicLobe (metallic.cpp:42-60), kr = colour, F82 tint
        // with F0 = colour and the edge tint (fresnel.h:114-120).
        l0.kind = Lobe::MicrofacetRefl;
        l0.fresnel = Lobe::F82;
        l0.compensate = true;
        l0.ax = m.p[0];
        l0.ay = m.p[1];
        const float f = 6.0f / 7.0f, f5 = f * f * f * f * f;
        for (int i = 0; i < w.n; ++i) {
            l0.kr[i] = col[i];
            l0.fa[i] = col[i];
            float fs = col[i] + f5 * (1.0f - col[i]);
            l0.fb[i] = fs * (7.0f / (f5 * f)) * (1.0f - alb(m.p + 2, w, i));
        }
    } else if (m.type == 2) {  // metal: ConductorLobe; mirror: MirrorLobe (FresnelConstant, kr = colour)
        l0.kind = Lobe::MicrofacetRefl;
        const bool mirror = (m.flags & 4u) != 0;
        l0.fresnel = mirror ? Lobe::One : Lobe::Conductor;
        l0.compensate = true;
        l0.ax = m.p[0];
        l0.ay = m.p[1];
        for (int i = 0; i < w.n; ++i) {
            if (mirror) {
                l0.kr[i] = col[i];
            } else {
                l0.kr[i] = 1.0f;
                l0.fa[i] = spd_of(sc.s->spd, m.spd0, std::fabs(w.lambda[i]));
                l0.fb[i] = spd_of(sc.s->spd, m.spd1, std::fabs(w.lambda[i]));
            }
        }
    } else if (m.type == 5 && (m.flags & 8u)) {  // plastic: PlasticLobe
        l0.kind = Lobe::Plastic;
        l0.ax = m.p[0];
        l0.ay = m.p[1];
        l0.fresnel = Lobe::Schlick;
        l0.eta0 = m.p[5];
        float f0 = ((m.p[5] - 1.0f) / (m.p[5] + 1.0f)) * ((m.p[5] - 1.0f) / (m.p[5] + 1.0f));
        for (int i = 0; i < w.n; ++i) {
            l0.kr[i] = col[i];
            l0.fa[i] = f0 * alb(m.p + 2, w, i);
        }
    } else if (m.type == 5) {  // substrate: SubstrateLobe over FresnelBlend
        l0.kind = Lobe::Substrate;
        l0.ax = m.p[0];
        l0.ay = m.p[1];
        for (int i = 0; i < w.n; ++i) {
            l0.kr[i] = col[i];
            l0.fa[i] = alb(m.p + 2, w, i);
        }
    } else if (m.type == 3) {  // glass: DielectricLobe
        l0.kind = Lobe::Dielectric;
        l0.ax = m.p[0];
        l0.ay = m.p[1];
        bool front = dot(it.wo, it.ng) > 0.0f;  // Interaction::correct_eta
        for (int i = 0; i < w.n; ++i) {
            l0.kr[i] = col[i];
            float ior = m.spd0 != kInvalid ? spd_of(sc.s->spd, m.spd0, is_rgb(w) ? -w.lambda[0] : w.lambda[i]) : m.p[2];
            l0.eta[i] = front ? ior : 1.0f / ior;
        }
    } else if (m.type == 4) {
        // PrincipledBSDF::create_lobe_set (principled_bsdf.cpp:352-461): sheen,
        // coat, metallic, transmission, specular, diffuse, each layer's albedo
        // taking its share of the remaining weight (layering_weight, :209-214).
        b.lobe_set = true;
        int n = w.n;
        float ax = m.p[0], ay = m.p[1], metallic = m.p[2], ior = m.p[3];
        float color[8], tint[8], weight[8];
        const float tc[3] = {m.p[4], m.p[5], m.p[6]};
        for (int i = 0; i < n; ++i) {
            color[i] = col[i];
            tint[i] = alb(tc, w, i);
            weight[i] = 1.0f;
        }
        float cos_theta = dot(it.wo, it.ng);
        float front = cos_theta > 0.0f ? 1.0f : 0.0f;
        auto mean = [&](const float *v) {
            float a = 0;
            for (int i = 0; i < n; ++i) a += v[i];
            return a * (1.0f / n);
        };
        auto layering = [&](const float *albedo) {
            float mx = -FLT_MAX;
            for (int i = 0; i < n; ++i) mx = std::max(mx, weight[i] == 0.0f ? 0.0f : albedo[i] / weight[i]);
            float lw = std::min(std::max(1.0f - mx, 0.0f), 1.0f);
            for (int i = 0; i < n; ++i) weight[i] = weight[i] * lw;
        };
        // Sheen / coat / transmission parameters: a 12-float SPD-table block.
        const float *xp = m.spd0 != kInvalid ? sc.s->spd + m.spd0 + 1 : nullptr;
        Lobe sheen, coat, trans;
        sheen.kind = Lobe::Sheen;
        sheen.sample_weight = 0.0f;
        coat.kind = Lobe::MicrofacetRefl;
        coat.sample_weight = 0.0f;
        trans.kind = Lobe::Dielectric;
        trans.sample_weight = 0.0f;
        if (xp && xp[0] != 0.0f) {
            // SheenLTC with the Approximate fits at (cos theta, roughness).
            float sw = xp[0] * front;
            float c0 = lut2c(kLutSheen, 4, 0, cos_theta, xp[1]);
            float c1 = lut2c(kLutSheen, 4, 1, cos_theta, xp[1]);
            float c2 = lut2c(kLutSheen, 4, 2, cos_theta, xp[1]);
            sheen.ltc_a = c0;
            sheen.ltc_b = c1;
            for (int i = 0; i < n; ++i) sheen.kr[i] = alb(xp + 2, w, i) * sw * weight[i] * c2;
            sheen.sample_weight = mean(sheen.kr);
            layering(sheen.kr);
        }
        if (xp && xp[5] != 0.0f) {
            // CoatLobe: dielectric Fresnel (coat ior), alpha = roughness^2,
            // albedo = CoatLobe table (sqrt(alpha), cos theta, ior ratio) * kr.
            float cw = xp[5] * front;
            float cr = std::min(std::max(xp[6], 0.0001f), 1.0f);
            cr = cr * cr;
            coat.fresnel = Lobe::DielectricFr;
            coat.ax = coat.ay = cr;
            coat.eta0 = xp[7];
            float s3 = lut3(kLutCoat, 1, std::sqrt(std::sqrt(cr * cr)), cos_theta, (xp[7] - 1.003f) / (4.0f - 1.003f));
            float ca[8];
            for (int i = 0; i < n; ++i) {
                coat.kr[i] = cw * weight[i] * alb(xp + 8, w, i);
                ca[i] = s3 * coat.kr[i];
            }
            coat.sample_weight = mean(ca);
            layering(ca);
        }
        Lobe met;
        met.kind = Lobe::MicrofacetRefl;
        met.fresnel = Lobe::F82;
        met.compensate = true;
        met.ax = ax;
        met.ay = ay;
        float mm = metallic * front;
        const float f = 6.0f / 7.0f, f5 = f * f * f * f * f;
        for (int i = 0; i < n; ++i) {
            met.kr[i] = weight[i] * mm;
            met.fa[i] = color[i];
            float fs = color[i] + f5 * (1.0f - color[i]);
            met.fb[i] = fs * (7.0f / (f5 * f)) * (1.0f - tint[i]);
        }
        met.sample_weight = mm * mean(weight);
        for (int i = 0; i < n; ++i) weight[i] *= (1.0f - mm);
        if (xp && xp[11] != 0.0f) {
            // Transmission: compensated DielectricLobe with FresnelSchlick
            // (F0 = schlick_F0(eta) * tint, eta = correct_eta(ior)), kt =
            // colour; f and sampling weighted by mean(transmission * weight).
            float tw = xp[11];
            float eta = cos_theta > 0.0f ? ior : 1.0f / ior;
            float f0 = ((eta - 1.0f) / (eta + 1.0f)) * ((eta - 1.0f) / (eta + 1.0f));
            trans.fresnel = Lobe::Schlick;
            trans.ax = ax;
            trans.ay = ay;
            float t_w[8];
            for (int i = 0; i < n; ++i) {
                trans.kr[i] = color[i];
                trans.eta[i] = eta;
                trans.fa[i] = tint[i] * f0;
                t_w[i] = weight[i] * tw;
            }
            trans.sample_weight = mean(t_w);
            trans.weight = trans.sample_weight;
            for (int i = 0; i < n; ++i) weight[i] *= (1.0f - tw);
        }
        Lobe spec;
        spec.kind = Lobe::MicrofacetRefl;
        spec.fresnel = Lobe::Schlick;
        spec.ax = ax;
        spec.ay = ay;
        spec.eta0 = ior;
        float f0s = ((ior - 1.0f) / (ior + 1.0f)) * ((ior - 1.0f) / (ior + 1.0f));
        float sl = lut3(kLutSpec, 1, std::sqrt(std::sqrt(ax * ay)), cos_theta, std::sqrt(std::fabs((ior - 1.0f) / (ior + 1.0f))));
        float alb_s[8];
        for (int i = 0; i < n; ++i) {
            spec.kr[i] = weight[i];
            spec.fa[i] = f0s * tint[i];
            alb_s[i] = (spec.fa[i] + sl * (1.0f - spec.fa[i])) * weight[i];
        }
        spec.sample_weight = mean(alb_s);
        layering(alb_s);
        Lobe dif;
        dif.kind = Lobe::Lambert;
        for (int i = 0; i < n; ++i) dif.kr[i] = color[i] * weight[i] * front;
        dif.sample_weight = mean(dif.kr);
        float sum = sheen.sample_weight + coat.sample_weight + met.sample_weight + trans.sample_weight +
                    spec.sample_weight + dif.sample_weight;
        b.count = 0;
        for (Lobe *l : {&sheen, &coat, &met, &trans, &spec, &dif}) {
            if (!(l->sample_weight > 0.0f)) continue;
            l->sample_weight /= sum;
            b.lobes[b.count++] = *l;
        }
    } else if (m.type == 6) {
        // MixMaterial / AddMaterial (mix.cpp:62-68, add.cpp:56-59):
        // LobeSet::create_mix / create_add (lobe.cpp:495-521), flattened
        // (LobeSet::flatten, lobe.cpp:533-560): a principled child's lobes
        // with weight and sample weight scaled by its sample weight, a
        // single-lobe child's lobe with its weight and sample weight.  mix:
        // (1 - frac, frac) for both; add: weights 1, sample weights 1/2.  The
        // lobe set is not dispersive (LobeSet keeps Lobe::is_dispersive).
        const bool add = (m.flags & 16u) != 0;
        const float wt[2] = {add ? 1.0f : 1.0f - m.p[0], add ? 1.0f : m.p[0]};
        const float swt[2] = {add ? 0.5f : 1.0f - m.p[0], add ? 0.5f : m.p[0]};
        const Bsdf c[2] = {make_bsdf(sc, sc.mat[m.spd0], it, w), make_bsdf(sc, sc.mat[m.spd1], it, w)};
        b.count = 0;
        b.lobe_set = true;
        b.dispersive = false;
        for (int k = 0; k < 2; ++k) {
            for (int j = 0; j < c[k].count; ++j) {
                Lobe l = c[k].lobes[j];
                if (c[k].lobe_set) {
                    l.weight *= swt[k];
                    l.sample_weight *= swt[k];
                } else {
                    l.weight = wt[k];
                    l.sample_weight = swt[k];
                }
                b.lobes[b.count++] = l;
            }
        }
    } else {
        l0.kind = Lobe::NoScatter;
    }
    return b;
}

// MaterialEvaluator::albedo (material.cpp:91-98) at c = dot(shading normal,
// wo): each lobe's albedo times its WeightedLobe weight (LobeSet::albedo,
// lobe.cpp:564-570).  Lambert kr; microfacet kr * F(c) (lobe.cpp:208-210),
// the coat and specular lobes with their table values
// (principled_bsdf.cpp:154-160,198-205); dielectric kt (1 - F) + F at |c|
// (lobe.cpp:308-313); FresnelBlend Rd * F_dielectric(c, 1.5); plastic its
// Schlick F (MicrofacetReflection of one); sheen its tint; a black body
// nothing.
static void bsdf_albedo(const Bsdf &b, float c, float *out) {
    const int n = b.n;
    for (int i = 0; i < n; ++i) out[i] = 0.0f;
    for (int k = 0; k < b.count; ++k) {
        const Lobe &l = b.lobes[k];
        float a[8] = {0, 0, 0, 0, 0, 0, 0, 0}, F[8];
        if (l.kind == Lobe::Lambert || l.kind == Lobe::Sheen) {
            for (int i = 0; i < n; ++i) a[i] = l.kr[i];
        } else if (l.kind == Lobe::MicrofacetRefl && l.fresnel == Lobe::DielectricFr) {
            float sc = lut3(kLutCoat, 1, std::sqrt(std::sqrt(l.ax * l.ax)), c, (l.eta0 - 1.003f) / (4.0f - 1.003f));
            for (int i = 0; i < n; ++i) a[i] = l.kr[i] * sc;
        } else if (l.kind == Lobe::MicrofacetRefl && l.fresnel == Lobe::Schlick) {
            float sl = lut3(kLutSpec, 1, std::sqrt(std::sqrt(l.ax * l.ay)), c,
                            std::sqrt(std::fabs((l.eta0 - 1.0f) / (l.eta0 + 1.0f))));
            for (int i = 0; i < n; ++i) a[i] = (l.fa[i] + sl * (1.0f - l.fa[i])) * l.kr[i];
        } else if (l.kind == Lobe::MicrofacetRefl) {
            fresnel_eval(l, n, c, F);
            for (int i = 0; i < n; ++i) a[i] = l.kr[i] * F[i];
        } else if (l.kind == Lobe::Dielectric) {
            diel_fresnel(l, n, std::fabs(c), F);
            for (int i = 0; i < n; ++i) a[i] = l.kr[i] * (1.0f - F[i]) + F[i];
        } else if (l.kind == Lobe::Substrate) {
            float f = mf::fr_dielectric(c, 1.5f);
            for (int i = 0; i < n; ++i) a[i] = l.kr[i] * f;
        } else if (l.kind == Lobe::Plastic) {
            fresnel_eval(l, n, c, F);
            for (int i = 0; i < n; ++i) a[i] = F[i];
        }
        for (int i = 0; i < n; ++i) out[i] += a[i] * l.weight;
    }
}

// ----- the path (pt.cpp:53-72; integrator.cpp:134-283) ------------------------
static void check_dispersive(const Bsdf &bsdf, Swl &w) {
    if (bsdf.dispersive && w.n > 1) {  // SampledWavelengths::check_dispersive
        bool all = true;
        for (int i = 1; i < w.n; ++i) all = all && w.pdf[i] != 0.0f;
        if (all)
            for (int i = 1; i < w.n; ++i) w.pdf[i] = 0.0f;
    }
}

// math/warp.h:132-145 sample_linear / sample_tent (the tent filter).
static float sample_linear_o(float u, float a, float b) {
    float x = u * (a + b) / (a + std::sqrt(a * a + u * (b * b - a * a)));
    x = std::min(x, kOneMinusEps);
    return (u == 0.0f && a == 0.0f) ? 0.0f : x;
}
static float sample_tent_o(float u, float r) {
    return u < 0.5f ? -r * sample_linear_o((0.5f - u) * 2.0f, 1.0f, 0.0f)
                    : r * sample_linear_o((u - 0.5f) * 2.0f, 1.0f, 0.0f);
}
static float sign_o(float v) { return v > 0.0f ? 1.0f : (v < 0.0f ? -1.0f : 0.0f); }

// FilterSampler::sample (fitted_curve.h:72-80) over the scene's filter table.
static void fitted_sample(const Scene &sc, float ux, float uy, float &fx, float &fy, float &weight) {
    const uint32_t n = Scene::kFilterN;
    ux = ux * 2.0f - 1.0f;
    uy = uy * 2.0f - 1.0f;
    uint32_t iv, iu;
    float fv = alias_cont(sc.f_marginal.data(), n, std::fabs(uy), iv);
    float pdf_v = sc.f_integral > 0.0f ? sc.f_marginal_func[iv] / sc.f_integral : 0.0f;
    float fu = alias_cont(sc.f_cond.data() + iv * n, n, std::fabs(ux), iu);
    float integral_u = sc.f_marginal_func[iv];
    float pdf_u = integral_u > 0.0f ? sc.f_cond_func[iv * n + iu] / integral_u : 0.0f;
    weight = sc.f_lut[iv * n + iu] / (pdf_u * pdf_v);
    fx = fu * sign_o(ux);
    fy = fv * sign_o(uy);
}

// Sampler::sensor_sample + the scene's filter + Sensor::generate_ray, with
// ThinLensCamera's lens (thin_lens.cpp:36-43) (5 draws); returns the filter
// weight.
static float camera_ray(const Scene &sc, const Camera &cam, Sampler &smp, uint32_t px, uint32_t py, float &film_x,
                        float &film_y, V3 &ro, V3 &rd) {
    float fu = smp.next(), fv = smp.next();
    float fx, fy, weight = 1.0f;
    if (cam.filter == 0u) {
        fx = -cam.filter_rx + fu * (cam.filter_rx - -cam.filter_rx);
        fy = -cam.filter_ry + fv * (cam.filter_ry - -cam.filter_ry);
    } else if (cam.filter == 1u) {
        fx = sample_tent_o(fu, cam.filter_rx);
        fy = sample_tent_o(fv, cam.filter_ry);
    } else {
        fitted_sample(sc, fu, fv, fx, fy, weight);
        fx *= cam.filter_rx;
        fy *= cam.filter_ry;
    }
    float lu = smp.next(), lv = smp.next();
    smp.next();
    film_x = static_cast<float>(px) + 0.5f + fx;
    film_y = static_cast<float>(py) + 0.5f + fy;
    float sx = cam.screen_lo_x + film_x / static_cast<float>(cam.width) * cam.screen_span_x;
    float sy = cam.screen_hi_y - film_y / static_cast<float>(cam.height) * cam.screen_span_y;
    V3 dc = normalize(v3(sx * cam.tan_half_fov, sy * cam.tan_half_fov, 1.0f));
    const float(*m)[4] = cam.c2w;
    V3 o_local = {0.0f, 0.0f, 0.0f};
    if (cam.thin_lens) {
        // square_to_disk (warp.h:24-28): r = sqrt(u.x), theta = 2 pi u.y.
        float r = std::sqrt(lu), th = 2.0f * kPi * lv;
        o_local = {r * std::cos(th) * cam.lens_radius, r * std::sin(th) * cam.lens_radius, 0.0f};
        float ft = cam.focal_distance / dc.z;
        V3 pf = {dc.x * ft, dc.y * ft, dc.z * ft};
        dc = normalize(v3(pf.x - o_local.x, pf.y - o_local.y, pf.z - o_local.z));
        ro = {m[0][0] * o_local.x + m[1][0] * o_local.y + m[2][0] * o_local.z + m[3][0],
              m[0][1] * o_local.x + m[1][1] * o_local.y + m[2][1] * o_local.z + m[3][1],
              m[0][2] * o_local.x + m[1][2] * o_local.y + m[2][2] * o_local.z + m[3][2]};
    } else {
        ro = {m[3][0], m[3][1], m[3][2]};
    }
    rd = normalize(v3(m[0][0] * dc.x + m[1][0] * dc.y + m[2][0] * dc.z, m[0][1] * dc.x + m[1][1] * dc.y + m[2][1] * dc.z,
                      m[0][2] * dc.x + m[1][2] * dc.y + m[2][2] * dc.z));
    return weight;
}

// IlluminationIntegrator::Li from ray (ro, rd) with a starting scatter pdf and
// throughput; `first` receives the first surface hit (HitContext).
static V3 path_li(const Scene &sc, Sampler &smp, Swl &w, V3 ro, V3 rd, float scatter_pdf, const float *thr0,
                  uint32_t max_depth, It *first, bool *first_hit) {
    const Integrator &ip = sc.ip;
    int n = w.n;
    float thr[8];
    for (int i = 0; i < n; ++i) thr[i] = thr0[i];
    V3 ret = {0, 0, 0};
    float eta_scale = 1.0f;
    for (uint32_t b = 0; b < max_depth; ++b) {
        RayPre rp = precompute(ro, rd);
        HitRec h = closest(sc, rp, FLT_MAX);
        if (h.prim == kInvalid) {
            // IlluminationIntegrator::evaluate_miss (integrator.cpp:111-132).
            if (sc.has_env) {
                float Le[8], lpdf;
                env_eval(sc, normalize(sub(add(ro, rd), ro)), w, Le, lpdf);
                lpdf *= light_pmf(sc, sc.ip.light_count - 1);
                float weight = scatter_pdf / (scatter_pdf + lpdf);
                if (ip.mis_mode == 2) weight = 1.0f;
                else if (ip.mis_mode == 1) weight = b == 0 ? weight : 0.0f;
                float d[8];
                for (int i = 0; i < n; ++i) d[i] = Le[i] * thr[i] * weight;
                ret = add(ret, linear_srgb(d, w));
            }
            break;
        }
        It it = interaction(sc, h.prim, h.u, h.v, rd);
        if (first && b == 0) {
            *first = it;
            if (first_hit) *first_hit = true;
        }
        if (it.light != kInvalid) {
            const AreaLight &L = sc.lights[it.light];
            float pmf_p = sc.s->prim_pmf[L.alias_offset + (it.prim - L.first_prim)];
            float pdf_pos = (1.0f / it.area) * pmf_p;
            V3 wv = sub(ro, it.pos);
            bool front = dot(wv, it.ng) > 0.0f || L.two_sided;
            float Le[8];
            if (front) emitter(L, w, Le);
            else for (int i = 0; i < n; ++i) Le[i] = 0.0f;
            float lpdf = pdf_wi(pdf_pos, it.ng, wv) * light_pmf(sc, it.light);
            float weight = scatter_pdf / (scatter_pdf + lpdf);
            if (ip.mis_mode == 2) weight = 1.0f;
            else if (ip.mis_mode == 1) weight = b == 0 ? weight : 0.0f;
            float d[8];
            for (int i = 0; i < n; ++i) d[i] = Le[i] * thr[i] * weight;
            V3 c = linear_srgb(d, w);
            ret = add(ret, c);
        }
        float ul = smp.next();
        float ux = smp.next(), uy = smp.next();
        LS ls = sample_light(sc, it, ul, ux, uy, w);
        V3 dir = sub(ls.p, it.pos);
        V3 nn = dot(it.ng, dir) > 0.0f ? it.ng : neg(it.ng);
        bool occ = any_hit(sc, precompute(offset_ray_origin(it.pos, nn), dir), 1.0f - kShadowEps);
        const Material &mt = sc.mat[it.mat];
        Bsdf bsdf = make_bsdf(sc, mt, it, w);
        check_dispersive(bsdf, w);
        V3 wl = normalize(sub(ls.p, it.pos));
        Eval se = bsdf_eval(bsdf, it.wo, wl, nullptr);
        V3 wi_s;
        float bs_eta = 1.0f;
        Eval be = bsdf_sample(bsdf, it.wo, smp, wi_s, bs_eta, mt.type == 1);
        // direct_lighting (integrator.cpp:29-31): a delta light (pdf < 0)
        // weighs 1 and divides by its pmf.
        bool delta = ls.pdf < 0.0f;
        float lpdf = delta ? -ls.pdf : ls.pdf;
        float wmis = delta ? 1.0f : ls.pdf / (ls.pdf + se.pdf);
        if (ip.mis_mode == 1) wmis = 1.0f;
        if (!occ && se.pdf > 0.0f && lpdf > 0.0f && ip.mis_mode != 2) {
            float d[8];
            for (int i = 0; i < n; ++i) d[i] = thr[i] * (ls.L[i] * se.f[i] * (wmis / lpdf));
            ret = add(ret, linear_srgb(d, w));
        }
        eta_scale *= bs_eta * bs_eta;
        float lum = thr[0];
        for (int i = 1; i < n; ++i) lum = std::max(lum, thr[i]);
        if (!(be.pdf > 0.0f) || lum == 0.0f) break;
        for (int i = 0; i < n; ++i) thr[i] = thr[i] * (be.f[i] / be.pdf);
        if (eta_scale * lum < ip.rr_threshold && b >= ip.min_depth) {
            float q = std::min(0.95f, lum);
            float rr = smp.next();
            if (q < rr) break;
            for (int i = 0; i < n; ++i) thr[i] = thr[i] * (1.0f / q);
        }
        bool zero = true;
        for (int i = 0; i < n; ++i) zero = zero && thr[i] == 0.0f;
        if (zero) break;
        scatter_pdf = be.pdf;
        V3 nb = dot(it.ng, wi_s) > 0.0f ? it.ng : neg(it.ng);
        ro = offset_ray_origin(it.pos, nb);
        rd = wi_s;
    }
    return ret;
}

static V3 trace_path(const Scene &sc, uint32_t px, uint32_t py, uint32_t frame) {
    const Integrator &ip = sc.ip;
    int n = static_cast<int>(ip.spectrum_dim);
    Sampler smp;
    smp.start(px, py, frame, 0xffffffffu, ip.sampler, ip.seed);
    Swl w = ip.srgb ? rgb_wavelengths(n) : sample_wavelengths(n, smp.next());
    smp.start(px, py, frame, 0u, ip.sampler, ip.seed);
    float film_x, film_y;
    V3 ro, rd;
    float fw = camera_ray(sc, sc.cam, smp, px, py, film_x, film_y, ro, rd);
    float thr[8];
    for (int i = 0; i < n; ++i) thr[i] = 1.0f;
    V3 L = path_li(sc, smp, w, ro, rd, 1e16f, thr, ip.max_depth, nullptr, nullptr);
    return {L.x * fw, L.y * fw, L.z * fw};
}

#include "restir.inc"

}  // namespace oracle

extern "C" {

int oracle_version(void) { return 2; }

// A prepared scene (the oracle's BVH is built once per handle).
void *oracle_open(const oracle_scene *s) { return new oracle::Scene(s); }
void oracle_close(void *h) { delete static_cast<oracle::Scene *>(h); }

// Closest hit for n rays (8 floats each: origin, unused, direction, tmax).
// hits: 4 uint32 per ray (inst, prim, u bits, v bits); t: -1 on a miss.
int oracle_trace_closest(void *handle, const float *rays, uint32_t n, uint32_t *hits, float *t) {
    const oracle::Scene &sc = *static_cast<oracle::Scene *>(handle);
    const oracle_scene *s = sc.s;
    for (uint32_t i = 0; i < n; ++i) {
        const float *r = rays + 8 * i;
        oracle::RayPre rp = oracle::precompute({r[0], r[1], r[2]}, {r[4], r[5], r[6]});
        oracle::HitRec h = oracle::closest(sc, rp, r[7]);
        if (h.prim == oracle::kInvalid) {
            hits[4 * i] = hits[4 * i + 1] = oracle::kInvalid;
            hits[4 * i + 2] = hits[4 * i + 3] = 0;
            t[i] = -1.0f;
        } else {
            hits[4 * i] = s->prim_inst[h.prim];
            hits[4 * i + 1] = h.prim;
            hits[4 * i + 2] = oracle::fbits(h.u);
            hits[4 * i + 3] = oracle::fbits(h.v);
            t[i] = h.t;
        }
    }
    return 0;
}

int oracle_trace_any(void *handle, const float *rays, uint32_t n, uint32_t *occ) {
    const oracle::Scene &sc = *static_cast<oracle::Scene *>(handle);
    for (uint32_t i = 0; i < n; ++i) {
        const float *r = rays + 8 * i;
        occ[i] = oracle::any_hit(sc, oracle::precompute({r[0], r[1], r[2]}, {r[4], r[5], r[6]}), r[7]) ? 1u : 0u;
    }
    return 0;
}

// Per-path radiance of the listed pixels for frames [frame_begin, frame_begin+frame_count):
// out[(f * npix_list + k) * 3 + c].
int oracle_paths(void *handle, const uint32_t *pixels, uint32_t npix_list, uint32_t frame_begin,
                 uint32_t frame_count, uint32_t threads, float *out) {
    const oracle::Scene &sc = *static_cast<oracle::Scene *>(handle);
    uint64_t total = static_cast<uint64_t>(npix_list) * frame_count;
    std::atomic<uint64_t> next{0};
    auto work = [&]() {
        while (true) {
            uint64_t j = next.fetch_add(64);
            if (j >= total) break;
            uint64_t e = std::min<uint64_t>(total, j + 64);
            for (uint64_t q = j; q < e; ++q) {
                uint32_t f = static_cast<uint32_t>(q / npix_list), k = static_cast<uint32_t>(q % npix_list);
                uint32_t pix = pixels[k];
                oracle::V3 L = oracle::trace_path(sc, pix % sc.cam.width, pix / sc.cam.width, frame_begin + f);
                out[3 * q] = L.x;
                out[3 * q + 1] = L.y;
                out[3 * q + 2] = L.z;
            }
        }
    };
    if (threads <= 1) {
        work();
    } else {
        std::vector<std::thread> th;
        for (uint32_t i = 0; i < threads; ++i) th.emplace_back(work);
        for (auto &x : th) x.join();
    }
    return 0;
}

// Full-frame render with the reference film semantics: FP32 running mean of
// zero_if_nan_inf(L) (normal.cpp:87-101) into film32 (4 floats per pixel) and,
// when film64 is non-null, FP64 sums (r, g, b, count) per pixel.
int oracle_render(void *handle, uint32_t frame_begin, uint32_t frame_count, uint32_t threads, float *film32,
                  double *film64) {
    const oracle::Scene &sc = *static_cast<oracle::Scene *>(handle);
    uint32_t npix = sc.cam.width * sc.cam.height;
    std::atomic<uint32_t> next{0};
    auto work = [&]() {
        while (true) {
            uint32_t p0 = next.fetch_add(16);
            if (p0 >= npix) break;
            for (uint32_t p = p0; p < std::min(npix, p0 + 16); ++p) {
                float *acc = film32 + 4 * p;
                if (frame_begin == 0) acc[0] = acc[1] = acc[2] = acc[3] = 0.0f;
                double *a64 = film64 ? film64 + 4 * p : nullptr;
                if (a64 && frame_begin == 0) a64[0] = a64[1] = a64[2] = a64[3] = 0.0;
                for (uint32_t f = frame_begin; f < frame_begin + frame_count; ++f) {
                    oracle::V3 L = oracle::trace_path(sc, p % sc.cam.width, p / sc.cam.width, f);
                    float v[4] = {L.x, L.y, L.z, 1.0f};
                    bool bad = false;
                    for (int c = 0; c < 3; ++c) bad = bad || std::isnan(v[c]) || std::isinf(v[c]);
                    if (bad) v[0] = v[1] = v[2] = v[3] = 0.0f;
                    float a = 1.0f / static_cast<float>(f + 1u);
                    for (int c = 0; c < 4; ++c) acc[c] = acc[c] + a * (v[c] - acc[c]);
                    if (a64) {
                        for (int c = 0; c < 3; ++c) a64[c] += bad ? 0.0 : v[c];
                        a64[3] += 1.0;
                    }
                }
            }
        }
    };
    if (threads <= 1) {
        work();
    } else {
        std::vector<std::thread> th;
        for (uint32_t i = 0; i < threads; ++i) th.emplace_back(work);
        for (auto &x : th) x.join();
    }
    return 0;
}

// TEA/LCG stream of the independent sampler, for golden-vector checks.
void oracle_sampler_stream(uint32_t px, uint32_t py, uint32_t sample, uint32_t dim, uint32_t kind, uint32_t seed,
                           uint32_t n, float *out) {
    oracle::Sampler s;
    s.start(px, py, sample, dim, kind, seed);
    for (uint32_t i = 0; i < n; ++i) out[i] = s.next();
}

uint32_t oracle_tea(uint32_t a, uint32_t b) { return oracle::tea(a, b); }

// Hero wavelengths and pdfs of one uniform sample.
void oracle_wavelengths(uint32_t n, float u, float *lambda, float *pdf) {
    oracle::Swl w = oracle::sample_wavelengths(static_cast<int>(n), u);
    for (uint32_t i = 0; i < n; ++i) {
        lambda[i] = w.lambda[i];
        pdf[i] = w.pdf[i];
    }
}

// Linear sRGB of a sampled spectrum.
void oracle_linear_srgb(uint32_t n, const float *lambda, const float *pdf, const float *s, float *rgb) {
    oracle::Swl w;
    w.n = static_cast<int>(n);
    for (uint32_t i = 0; i < n; ++i) {
        w.lambda[i] = lambda[i];
        w.pdf[i] = pdf[i];
    }
    oracle::V3 c = oracle::linear_srgb(s, w);
    rgb[0] = c.x; rgb[1] = c.y; rgb[2] = c.z;
}

float oracle_cie_y_integral(void) { return oracle::tables().y_integral; }

float oracle_spd_eval(const float *f, int n, float lambda) { return oracle::spd_eval(f, n, lambda); }

// Real-time ReSTIR state over an opened scene (restir.inc).
void *oracle_rt_open(void *handle, uint32_t width, uint32_t height) {
    return new oracle::rt::Frame(*static_cast<oracle::Scene *>(handle), width, height);
}
void oracle_rt_close(void *rt) { delete static_cast<oracle::rt::Frame *>(rt); }

// One frame with the given camera block (128 bytes) and parameter block
// (448 bytes, as vs_restir_params returns it).
int oracle_rt_frame(void *rt, const void *camera, const void *params, uint32_t film_index, uint32_t threads) {
    auto *f = static_cast<oracle::rt::Frame *>(rt);
    oracle::Camera cam;
    oracle::rt::Params p;
    std::memcpy(&cam, camera, sizeof(cam));
    std::memcpy(&p, params, sizeof(p));
    if (p.width * p.height != f->npix || p.di.s_count > oracle::rt::kMaxNeighbours ||
        p.gi.s_count > oracle::rt::kMaxNeighbours)
        return 1;
    f->run(cam, p, film_index, threads);
    return 0;
}

// SVGF over a film (4 floats per pixel) with the frame's camera and
// parameter blocks and the 48-byte SVGF settings (as vs_denoiser_params
// returns them).
int oracle_rt_svgf(void *rt, const void *camera, const void *params, const void *svgf_params, const float *radiance,
                   uint32_t threads) {
    auto *f = static_cast<oracle::rt::Frame *>(rt);
    oracle::Camera cam;
    oracle::rt::Params p;
    oracle::rt::Frame::SvParams sp;
    static_assert(sizeof(sp) == 48, "SVGF settings block");
    std::memcpy(&cam, camera, sizeof(cam));
    std::memcpy(&p, params, sizeof(p));
    std::memcpy(&sp, svgf_params, sizeof(sp));
    if (p.width * p.height != f->npix || sp.N > 10u || sp.mradius < 0 || sp.mradius > 5) return 1;
    f->svgf(cam, p, sp, radiance, threads);
    return 0;
}

// Per-pixel buffers of the last frame: 0 direct radiance, 1 indirect
// radiance, 2 motion, 3 surfaces, 4 direct reservoirs, 5 indirect
// reservoirs, 6 BSDF samples, 7 initial indirect samples, 8 film; of the
// last SVGF pass: 9 output, 10 G-buffer, 11 albedo, 12 emission, 13 filtered
// SVGFData, 14 G-buffer motion, 15 history.
int oracle_rt_buffer(void *rt, int which, void *dst, size_t bytes) {
    auto *f = static_cast<oracle::rt::Frame *>(rt);
    uint32_t c = f->cur();
    const void *src = nullptr;
    size_t n = 0;
    switch (which) {
        case 0: src = f->di_rad.data(); n = f->di_rad.size() * 4; break;
        case 1: src = f->gi_rad.data(); n = f->gi_rad.size() * 4; break;
        case 2: src = f->motion.data(); n = f->motion.size() * 4; break;
        case 3: src = f->surf[c].data(); n = f->surf[c].size() * sizeof(oracle::rt::Surface); break;
        case 4: src = f->di[c].data(); n = f->di[c].size() * sizeof(oracle::rt::DiRes); break;
        case 5: src = f->gi[c].data(); n = f->gi[c].size() * sizeof(oracle::rt::GiRes); break;
        case 6: src = f->hit_bsdf.data(); n = f->hit_bsdf.size() * sizeof(oracle::rt::HitBsdf); break;
        case 7: src = f->gi_init.data(); n = f->gi_init.size() * sizeof(oracle::rt::GiRes); break;
        case 8: src = f->film.data(); n = f->film.size() * 4; break;
        case 9: src = f->sout.data(); n = f->sout.size() * 4; break;
        case 10: src = f->sgeom[c].data(); n = f->sgeom[c].size() * sizeof(oracle::rt::Frame::SvGeom); break;
        case 11: src = f->salb.data(); n = f->salb.size() * 4; break;
        case 12: src = f->semi.data(); n = f->semi.size() * 4; break;
        case 13: src = f->sprev.data(); n = f->sprev.size() * sizeof(oracle::rt::Frame::SvData); break;
        case 14: src = f->smot.data(); n = f->smot.size() * 4; break;
        case 15: src = f->shist[c].data(); n = f->shist[c].size() * 4; break;
        default: return 1;
    }
    if (n != bytes) return 2;
    std::memcpy(dst, src, n);
    return 0;
}

}  // extern "C"

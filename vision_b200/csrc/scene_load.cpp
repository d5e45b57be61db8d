// vision_scene.json -> HostScene.
//
// Keeps the reference's schema (src/core/scene_desc.cpp:37-53,
// src/core/node_desc.cpp): top-level "shapes", "materials", "camera",
// "integrator", "spectrum", "sampler", "light_sampler", "render_setting";
// nodes are {"type", "name", "param"}; slots are a number, an array, a
// {"channels", "node"} pair or a {"type": "number", "param": {"value"}} node;
// emission hangs off a shape as {"emission": {"type": "area", "param"}}.
#include "vs_host.h"
#include "json.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "vs_image.h"
#include <map>
#include <numeric>
#include <stdexcept>

#include "data/spectral_tables.inc"

namespace vs {

void update_env_world(HostScene &s);
void rebuild_light_alias(HostScene &s);

const Cie5 &cie5() {
    static Cie5 c = [] {
        Cie5 r{};
        for (int i = 0; i < kSpd5Count; ++i) {
            r.x[i] = VS_CIE_X[5 * i];
            r.y[i] = VS_CIE_Y[5 * i];
            r.z[i] = VS_CIE_Z[5 * i];
            r.d65[i] = VS_CIE_D65[5 * i];
        }
        float sum = 0.0f;
        for (int i = 0; i < kSpd5Count; ++i) sum += 0.5f * (VS_CIE_Y[i * 5] + VS_CIE_Y[(i + 1) * 5]);
        r.y_integral = sum * 5.0f;
        return r;
    }();
    return c;
}

void build_alias(const std::vector<float> &weights, std::vector<AliasEntry> &table, std::vector<float> &pmf,
                 float *integral_out) {
    size_t n = weights.size();
    double sum = 0.0;
    for (float w : weights) sum += w;
    double ratio = static_cast<double>(n) / sum;
    std::vector<uint32_t> over, under;
    table.assign(n, AliasEntry{0.0f, 0u});
    for (uint32_t i = 0; i < n; ++i) {
        float p = static_cast<float>(weights[i] * ratio);
        table[i] = {p, i};
        (p > 1.0f ? over : under).push_back(i);
    }
    while (!over.empty() && !under.empty()) {
        uint32_t o = over.back(), u = under.back();
        over.pop_back();
        under.pop_back();
        table[o].prob -= 1.0f - table[u].prob;
        table[u].alias = o;
        if (table[o].prob > 1.0f) over.push_back(o);
        else if (table[o].prob < 1.0f) under.push_back(o);
    }
    for (uint32_t i : over) table[i] = {1.0f, i};
    for (uint32_t i : under) table[i] = {1.0f, i};
    float integral = static_cast<float>(sum / static_cast<double>(n));
    if (integral_out) *integral_out = integral;
    pmf.resize(n);
    for (size_t i = 0; i < n; ++i)
        pmf[i] = integral > 0.0f ? weights[i] / (integral * static_cast<float>(n)) : 0.0f;
}

// Filter::evaluate of the tabulated filters at p in [0, r]^2.
float filter_value(const Camera &c, float x, float y) {
    const float kPiF = 3.14159265358979323846f;
    if (c.filter == kFilterGaussian) {
        // GaussianFilter::evaluate (gaussian.cpp:36-40), gaussian() of math/util.h:37-42.
        const float sigma = c.filter_p0;
        auto g = [&](float v) {
            return 1.0f / std::sqrt(2.0f * kPiF * sigma * sigma) * std::exp(-(v * v) / (2.0f * sigma * sigma));
        };
        const float vx = g(x) - g(c.filter_rx), vy = g(y) - g(c.filter_ry);
        return std::max(0.0f, vx) * std::max(0.0f, vy);
    }
    if (c.filter == kFilterMitchell) {
        // MitchellFilter::mitchell_1d / evaluate (mitchell.cpp).
        const float b = c.filter_p0, cc = c.filter_p1;
        auto m1 = [&](float v) {
            v = std::fabs(v);
            if (v <= 1.0f)
                return ((12.0f - 9.0f * b - 6.0f * cc) * v * v * v + (-18.0f + 12.0f * b + 6.0f * cc) * v * v +
                        (6.0f - 2.0f * b)) * (1.0f / 6.0f);
            if (v <= 2.0f)
                return ((-b - 6.0f * cc) * v * v * v + (6.0f * b + 30.0f * cc) * v * v + (-12.0f * b - 48.0f * cc) * v +
                        (8.0f * b + 24.0f * cc)) * (1.0f / 6.0f);
            return 0.0f;
        };
        return m1(2.0f * x / c.filter_rx) * m1(2.0f * y / c.filter_ry);
    }
    // LanczosSincFilter::evaluate (sinc.cpp): windowed_sinc(x, r, tau) per axis, times 4.
    const float tau = c.filter_p0;
    auto sinc = [&](float v) {
        const float a = kPiF * v;
        return 1.0f + a * a == 1.0f ? 1.0f : std::sin(a) / a;
    };
    auto ws = [&](float v, float r) { return std::fabs(v) > r ? 0.0f : sinc(v) * sinc(v / tau); };
    return ws(x, c.filter_rx) * ws(y, c.filter_ry) * 4.0f;
}

// FilterSampler::build (fitted_curve.h:36-58): the filter at the centres of a
// kFilterTable^2 grid over [0, r]^2, normalised by its average, and the 2D
// alias warper over its absolute value (AliasTable2D::build, alias2d.cpp).
void build_filter_table(const Camera &c, std::vector<float> &tab, std::vector<AliasEntry> &alias, float &integral) {
    tab.clear();
    alias.clear();
    integral = 0.0f;
    if (c.filter != kFilterGaussian && c.filter != kFilterMitchell && c.filter != kFilterSinc) return;
    const uint32_t n = kFilterTable;
    std::vector<float> lut(n * n), func(n * n);
    for (uint32_t i = 0; i < n * n; ++i) {
        const uint32_t x = i % n, y = i / n;
        const float px = (static_cast<float>(x) + 0.5f) / static_cast<float>(n) * c.filter_rx;
        const float py = (static_cast<float>(y) + 0.5f) / static_cast<float>(n) * c.filter_ry;
        const float v = filter_value(c, px, py);
        func[i] = std::fabs(v);
        lut[i] = v;
    }
    float sum = 0.0f;
    for (float v : lut) sum += v;
    const float avg = sum / static_cast<float>(n * n);
    for (float &v : lut) v = v / avg;
    std::vector<float> marginal(n), cond_func;
    std::vector<AliasEntry> cond;
    for (uint32_t v = 0; v < n; ++v) {
        std::vector<float> row(func.begin() + v * n, func.begin() + (v + 1) * n);
        std::vector<AliasEntry> t;
        std::vector<float> pmf;
        float row_integral = 0.0f;
        build_alias(row, t, pmf, &row_integral);
        marginal[v] = row_integral;
        cond.insert(cond.end(), t.begin(), t.end());
        cond_func.insert(cond_func.end(), row.begin(), row.end());
    }
    std::vector<AliasEntry> mtab;
    std::vector<float> mpmf;
    build_alias(marginal, mtab, mpmf, &integral);
    tab = lut;
    tab.insert(tab.end(), marginal.begin(), marginal.end());
    tab.insert(tab.end(), cond_func.begin(), cond_func.end());
    alias = mtab;
    alias.insert(alias.end(), cond.begin(), cond.end());
}

namespace {

std::runtime_error unsupported(const std::string &what) {
    return std::runtime_error("unsupported: " + what);
}

m4 mat_from_columns(const Json &cols) {
    m4 m = m4_identity();
    if (!cols.is_array() || cols.size() != 4) throw std::runtime_error("matrix4x4 needs 4 columns");
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r) m.m[c][r] = cols[c][r].as_float();
    return m;
}

m4 translation(f3 t) {
    m4 m = m4_identity();
    m.m[3][0] = t.x; m.m[3][1] = t.y; m.m[3][2] = t.z;
    return m;
}
m4 scale_m(f3 s) {
    m4 m = m4_identity();
    m.m[0][0] = s.x; m.m[1][1] = s.y; m.m[2][2] = s.z;
    return m;
}
// Right-handed rotation by `deg` degrees about `axis` (Rodrigues):
// R e_j = cos e_j + sin (k x e_j) + (1 - cos) k k_j.
m4 rot_axis(f3 axis, float deg) {
    const f3 k = normalize(axis);
    const float a = deg * kPi / 180.0f, c = std::cos(a), sn = std::sin(a);
    const float kk[3] = {k.x, k.y, k.z};
    m4 m = m4_identity();
    for (int j = 0; j < 3; ++j) {
        f3 e = make3(j == 0 ? 1.0f : 0.0f, j == 1 ? 1.0f : 0.0f, j == 2 ? 1.0f : 0.0f);
        f3 col = e * c + cross(k, e) * sn + k * ((1.0f - c) * kk[j]);
        m.m[j][0] = col.x; m.m[j][1] = col.y; m.m[j][2] = col.z;
    }
    return m;
}
// Right-handed rotations about the axes, angle in degrees.
m4 rot_x(float deg) {
    float a = deg * kPi / 180.0f, c = std::cos(a), s = std::sin(a);
    m4 m = m4_identity();
    m.m[1][1] = c; m.m[1][2] = s; m.m[2][1] = -s; m.m[2][2] = c;
    return m;
}
m4 rot_y(float deg) {
    float a = deg * kPi / 180.0f, c = std::cos(a), s = std::sin(a);
    m4 m = m4_identity();
    m.m[0][0] = c; m.m[0][2] = -s; m.m[2][0] = s; m.m[2][2] = c;
    return m;
}
m4 rot_z(float deg) {
    float a = deg * kPi / 180.0f, c = std::cos(a), s = std::sin(a);
    m4 m = m4_identity();
    m.m[0][0] = c; m.m[0][1] = s; m.m[1][0] = -s; m.m[1][1] = c;
    return m;
}

// Inverse of an affine 4x4 (rotation/scale + translation).
m4 invert_affine(const m4 &m) {
    double a[3][3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) a[r][c] = m.m[c][r];
    double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                 a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
    double inv[3][3];
    inv[0][0] = (a[1][1] * a[2][2] - a[1][2] * a[2][1]) / det;
    inv[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) / det;
    inv[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) / det;
    inv[1][0] = (a[1][2] * a[2][0] - a[1][0] * a[2][2]) / det;
    inv[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) / det;
    inv[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) / det;
    inv[2][0] = (a[1][0] * a[2][1] - a[1][1] * a[2][0]) / det;
    inv[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) / det;
    inv[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) / det;
    m4 r = m4_identity();
    for (int row = 0; row < 3; ++row)
        for (int c = 0; c < 3; ++c) r.m[c][row] = static_cast<float>(inv[row][c]);
    for (int row = 0; row < 3; ++row) {
        double t = 0.0;
        for (int c = 0; c < 3; ++c) t -= inv[row][c] * m.m[3][c];
        r.m[3][row] = static_cast<float>(t);
    }
    return r;
}

f3 as_f3(const Json &j, f3 def) {
    if (!j.is_array() || j.size() < 3) return def;
    return {j[0].as_float(), j[1].as_float(), j[2].as_float()};
}

// Camera frame whose columns are right, up, forward, position; only used to
// recover yaw and pitch (Sensor::update_mat, sensor.cpp:78-83).
m4 look_at(f3 pos, f3 target, f3 up) {
    f3 fwd = normalize(target - pos);
    f3 right = normalize(cross(fwd, up));
    f3 up2 = cross(right, fwd);
    m4 m = m4_identity();
    m.m[0][0] = right.x; m.m[0][1] = right.y; m.m[0][2] = right.z;
    m.m[1][0] = up2.x; m.m[1][1] = up2.y; m.m[1][2] = up2.z;
    m.m[2][0] = fwd.x; m.m[2][1] = fwd.y; m.m[2][2] = fwd.z;
    m.m[3][0] = pos.x; m.m[3][1] = pos.y; m.m[3][2] = pos.z;
    return m;
}

// TransformDesc::init (node_desc.cpp:26-52).
m4 parse_transform(const Json &t) {
    if (t.is_null()) return m4_identity();
    std::string type = t["type"].as_string("matrix4x4");
    const Json &p = t["param"];
    if (type == "matrix4x4") return p.contains("matrix4x4") ? mat_from_columns(p["matrix4x4"]) : m4_identity();
    if (type == "look_at")
        return look_at(as_f3(p["position"], make3(0.0f)), as_f3(p["target_pos"], make3(0, 0, 1)), as_f3(p["up"], make3(0, 1, 0)));
    if (type == "Euler") {
        m4 yaw = rot_y(p["yaw"].as_float(0.0f));
        m4 roll = rot_z(p["roll"].as_float(0.0f));
        m4 pitch = rot_x(p["pitch"].as_float(0.0f));
        return translation(as_f3(p["position"], make3(0.0f))) * pitch * roll * yaw;
    }
    if (type == "trs") {
        // TransformDesc "trs" (node_desc.cpp:48-52): T * R * S, r = (axis, degrees).
        std::vector<float> r = p["r"].as_floats();
        if (r.size() < 4) r = {1.0f, 0.0f, 0.0f, 0.0f};
        return translation(as_f3(p["t"], make3(0.0f))) * rot_axis(make3(r[0], r[1], r[2]), r[3]) *
               scale_m(as_f3(p["s"], make3(1.0f)));
    }
    throw unsupported("transform type '" + type + "'");
}

// A shader node's type and parameters (ShaderNodeDesc::init,
// node_desc.cpp:292-320): {"type", "param"}, or the parameters inline, where
// an object naming a file ("fn") is an image node.
std::string node_type(const Json &n) {
    if (!n.is_object()) return "";
    if (n.contains("param")) return n["type"].as_string("number");
    return n["type"].as_string(n.contains("fn") ? "image" : "number");
}
const Json &node_param(const Json &n) { return n.contains("param") ? n["param"] : n; }

// Slot value as a flat float list (SlotDesc::init, node_desc.cpp:127-150).
std::vector<float> slot_values(const Json &j) {
    if (j.is_number() || j.is_array()) return j.as_floats();
    if (j.is_object()) {
        if (j.contains("channels")) return slot_values(j["node"]);
        std::string type = node_type(j);
        if (type == "number" || type == "constant") {
            const Json &p = j.contains("param") ? j["param"] : j;
            return p["value"].as_floats();
        }
        throw unsupported("shader node type '" + type + "'");
    }
    return {};
}

bool is_blackbody_slot(const Json &j) {
    const Json &n = j.is_object() && j.contains("channels") ? j["node"] : j;
    return n.is_object() && n["type"].as_string() == "blackbody";
}
const Json &slot_node(const Json &j) { return j.is_object() && j.contains("channels") ? j["node"] : j; }

f3 slot_rgb(const Json &j, f3 def) {
    std::vector<float> v = slot_values(j);
    if (v.empty()) return def;
    if (v.size() == 1) return make3(v[0]);
    return {v[0], v[1], v.size() > 2 ? v[2] : v[1]};
}
float slot_scalar(const Json &j, float def) {
    std::vector<float> v = slot_values(j);
    return v.empty() ? def : v[0];
}

// The file of an `image` shader node (image.cpp) as linear RGB texels (4
// floats each, RGB and 0): the sRGB transfer function removed for the colour
// space "srgb" (the default of 8-bit files; "linear" for Radiance HDR); a grey
// file replicated to three channels.
std::vector<float> load_texture_texels(const Json &node, const std::string &base_dir, uint32_t &w, uint32_t &h) {
    const Json &p = node_param(node);
    const std::string fn = p["fn"].as_string();
    if (fn.empty()) throw std::runtime_error("image node without 'fn'");
    const bool absolute = !fn.empty() && fn[0] == '/';
    const std::string path = absolute || base_dir.empty() ? fn : base_dir + "/" + fn;
    const size_t dot = path.find_last_of('.');
    std::string ext = dot == std::string::npos ? "" : path.substr(dot + 1);
    for (char &c : ext) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
    if (ext != "png" && ext != "jpg" && ext != "jpeg" && ext != "hdr" && ext != "exr")
        throw unsupported("image file format '" + ext + "' (" + fn + ")");
    std::string cs = p["color_space"].as_string("");
    if (cs.empty()) cs = ext == "hdr" || ext == "exr" ? "linear" : "srgb";
    if (cs != "srgb" && cs != "linear") throw unsupported("image colour space '" + cs + "'");
    const Image im = load_image(path);
    w = im.width;
    h = im.height;
    std::vector<float> t(static_cast<size_t>(w) * h * 4, 0.0f);
    for (size_t i = 0; i < static_cast<size_t>(w) * h; ++i) {
        for (int c = 0; c < 3; ++c) {
            const float v = im.data[i * im.channels + (im.channels >= 3 ? c : 0)];
            t[4 * i + c] = cs == "srgb" ? srgb_to_linear(v) : v;
        }
    }
    return t;
}

struct MeshData {
    std::vector<f3> p, n;
    std::vector<f2> uv;
    std::vector<uint32_t> idx;
};

// Quad::init (src/render_core/shapes/quad.cpp:21-50): unit quad in the xz plane
// facing +y, vertex normals set to the unnormalised geometric normal.
MeshData make_quad(float width, float height) {
    MeshData m;
    float w = width / 2, h = height / 2;
    m.p = {{w, 0, h}, {w, 0, -h}, {-w, 0, h}, {-w, 0, -h}};
    m.uv = {{1, 1}, {1, 0}, {0, 1}, {0, 0}};
    f3 ng = cross(m.p[0] - m.p[2], m.p[1] - m.p[2]);
    m.n.assign(4, ng);
    m.idx = {0, 1, 2, 2, 1, 3};
    return m;
}

// Cube::init (src/render_core/shapes/cube.cpp:20-71).
MeshData make_cube(float x, float y, float z) {
    y = y == 0 ? x : y;
    z = z == 0 ? y : z;
    x /= 2; y /= 2; z /= 2;
    MeshData m;
    m.p = {{-x, -y, z}, {x, -y, z}, {-x, y, z}, {x, y, z},     {-x, y, -z}, {x, y, -z}, {-x, -y, -z}, {x, -y, -z},
           {-x, y, z},  {x, y, z},  {-x, y, -z}, {x, y, -z},   {-x, -y, z}, {x, -y, z}, {-x, -y, -z}, {x, -y, -z},
           {x, -y, z},  {x, y, z},  {x, y, -z},  {x, -y, -z},  {-x, -y, z}, {-x, y, z}, {-x, y, -z},  {-x, -y, -z}};
    const f3 N[6] = {{0, 0, 1}, {0, 0, -1}, {0, 1, 0}, {0, -1, 0}, {1, 0, 0}, {-1, 0, 0}};
    for (int f = 0; f < 6; ++f)
        for (int k = 0; k < 4; ++k) m.n.push_back(N[f]);
    m.uv = {{0, 0}, {1, 0}, {0, 1}, {1, 1}, {0, 1}, {1, 1}, {0, 0}, {1, 0}, {0, 1}, {1, 1}, {0, 0}, {1, 0},
            {0, 1}, {1, 1}, {0, 0}, {1, 0}, {0, 1}, {1, 1}, {1, 0}, {0, 0}, {0, 1}, {1, 1}, {1, 0}, {0, 0}};
    m.idx = {0, 1, 3, 0, 3, 2, 6, 5, 7, 4, 5, 6, 10, 9, 11, 8, 9, 10, 13, 14, 15, 13, 12, 14, 18, 17, 19, 17, 16, 19, 21, 22, 23, 20, 21, 23};
    return m;
}

// Inline triangle mesh: {"positions": [x0,y0,z0,...], "indices": [...],
// optional "normals", "uvs"}.  Stand-in for the assimp "model" shape.
MeshData make_inline_mesh(const Json &p) {
    MeshData m;
    std::vector<float> P = p["positions"].as_floats();
    std::vector<float> Nn = p["normals"].as_floats();
    std::vector<float> UV = p["uvs"].as_floats();
    const Json &I = p["indices"];
    for (size_t i = 0; i + 2 < P.size(); i += 3) m.p.push_back({P[i], P[i + 1], P[i + 2]});
    for (size_t i = 0; i < m.p.size(); ++i) {
        m.n.push_back(Nn.size() >= 3 * (i + 1) ? f3{Nn[3 * i], Nn[3 * i + 1], Nn[3 * i + 2]} : f3{0, 0, 0});
        m.uv.push_back(UV.size() >= 2 * (i + 1) ? f2{UV[2 * i], UV[2 * i + 1]} : f2{0, 0});
    }
    for (size_t i = 0; i < I.size(); ++i) m.idx.push_back(I[i].as_uint());
    return m;
}

// Model (src/render_core/shapes/model.cpp:27-37) reads its file through
// AssimpParser (importers/assimp_parser.cpp:231-340, assimp's OBJ importer and
// post-processing).  Restated here for Wavefront OBJ:
//   * `v`, `vt`, `vn` records and `f` faces with `i`, `i/t`, `i//n`, `i/t/n`
//     references, 1-based or negative (relative to the end);
//   * every distinct (position, uv, normal) triple is one vertex, numbered in
//     order of first use (JoinIdenticalVertices);
//   * polygons are split as a fan from their first corner (Triangulate; the
//     two triangles of a quad are (0,1,2), (0,2,3) as in parse_meshes);
//   * a face without normals gets its geometric normal normalize((p1-p0) x
//     (p2-p0)): on its own vertices (GenNormals), or with `smooth`, summed
//     over the faces without normals that share the position record and
//     normalised (GenSmoothNormals);
//   * uv defaults to (0, 0); `flip_uv` (default true) maps v to 1 - v;
//     non-finite normals and uvs become zero (parse_meshes);
//   * `swap_handed` negates z of positions and normals and reverses the
//     winding (MakeLeftHanded | FlipWindingOrder);
//   * groups, objects and `usemtl` are ignored: the model is one mesh with the
//     shape's material.
MeshData load_obj(const std::string &path, bool smooth, bool flip_uv, bool swap_handed) {
    std::FILE *fp = std::fopen(path.c_str(), "rb");
    if (!fp) throw std::runtime_error("model: cannot open '" + path + "'");
    std::string text;
    char buf[1 << 16];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof(buf), fp)) > 0) text.append(buf, got);
    std::fclose(fp);

    std::vector<f3> P, N;
    std::vector<f2> T;
    struct Corner {
        int v, t, n;
    };
    std::vector<Corner> corners;    // triangle corners, 3 per triangle
    std::vector<uint32_t> tri_face;  // face number of each triangle
    uint32_t face_count = 0;
    auto fail = [&](size_t line, const std::string &why) {
        throw std::runtime_error("model '" + path + "' line " + std::to_string(line) + ": " + why);
    };
    size_t pos = 0, line_no = 0;
    std::vector<Corner> poly;
    while (pos < text.size()) {
        size_t end = text.find('\n', pos);
        if (end == std::string::npos) end = text.size();
        std::string line = text.substr(pos, end - pos);
        pos = end + 1;
        ++line_no;
        if (!line.empty() && line.back() == '\r') line.pop_back();
        const char *c = line.c_str();
        while (*c == ' ' || *c == '\t') ++c;
        auto floats = [&](const char *q, float *out, int n) {
            int k = 0;
            while (k < n) {
                char *e;
                float v = std::strtof(q, &e);
                if (e == q) break;
                out[k++] = v;
                q = e;
            }
            return k;
        };
        if (c[0] == 'v' && (c[1] == ' ' || c[1] == '\t')) {
            float v[3];
            if (floats(c + 2, v, 3) != 3) fail(line_no, "vertex needs 3 coordinates");
            P.push_back({v[0], v[1], v[2]});
        } else if (c[0] == 'v' && c[1] == 't' && (c[2] == ' ' || c[2] == '\t')) {
            float v[2] = {0.0f, 0.0f};
            if (floats(c + 3, v, 2) < 1) fail(line_no, "texture coordinate needs a value");
            T.push_back({v[0], v[1]});
        } else if (c[0] == 'v' && c[1] == 'n' && (c[2] == ' ' || c[2] == '\t')) {
            float v[3];
            if (floats(c + 3, v, 3) != 3) fail(line_no, "normal needs 3 components");
            N.push_back({v[0], v[1], v[2]});
        } else if (c[0] == 'f' && (c[1] == ' ' || c[1] == '\t')) {
            poly.clear();
            const char *q = c + 2;
            auto resolve = [&](long r, size_t count, const char *what) -> int {
                long i = r > 0 ? r - 1 : static_cast<long>(count) + r;
                if (r == 0 || i < 0 || i >= static_cast<long>(count)) fail(line_no, std::string(what) + " index out of range");
                return static_cast<int>(i);
            };
            while (*q) {
                while (*q == ' ' || *q == '\t') ++q;
                if (!*q) break;
                char *e;
                long vi = std::strtol(q, &e, 10);
                if (e == q) fail(line_no, "bad face corner");
                Corner k{resolve(vi, P.size(), "position"), -1, -1};
                q = e;
                if (*q == '/') {
                    ++q;
                    if (*q != '/') {
                        long ti = std::strtol(q, &e, 10);
                        if (e == q) fail(line_no, "bad texture index");
                        k.t = resolve(ti, T.size(), "texture coordinate");
                        q = e;
                    }
                    if (*q == '/') {
                        ++q;
                        long ni = std::strtol(q, &e, 10);
                        if (e == q) fail(line_no, "bad normal index");
                        k.n = resolve(ni, N.size(), "normal");
                        q = e;
                    }
                }
                if (*q && *q != ' ' && *q != '\t') fail(line_no, "bad face corner");
                poly.push_back(k);
            }
            if (poly.size() < 3) continue;  // points and lines carry no surface
            for (size_t i = 1; i + 1 < poly.size(); ++i) {
                corners.push_back(poly[0]);
                corners.push_back(poly[i]);
                corners.push_back(poly[i + 1]);
                tri_face.push_back(face_count);
            }
            ++face_count;
        }
    }
    if (swap_handed) {
        for (f3 &p : P) p.z = -p.z;
        for (f3 &n : N) n.z = -n.z;
        for (size_t t = 0; t < corners.size(); t += 3) std::swap(corners[t + 1], corners[t + 2]);
    }
    // Geometric normals of the triangles whose corners lack a normal.
    const size_t ntri = corners.size() / 3;
    std::vector<f3> tri_n(ntri, f3{0.0f, 0.0f, 0.0f});
    std::vector<f3> smooth_n;
    if (smooth) smooth_n.assign(P.size(), f3{0.0f, 0.0f, 0.0f});
    for (size_t t = 0; t < ntri; ++t) {
        const Corner *k = &corners[3 * t];
        if (k[0].n >= 0 && k[1].n >= 0 && k[2].n >= 0) continue;
        f3 g = cross(P[k[1].v] - P[k[0].v], P[k[2].v] - P[k[0].v]);
        const float l = length(g);
        tri_n[t] = l > 0.0f ? g / l : f3{0.0f, 0.0f, 0.0f};
        if (smooth)
            for (int i = 0; i < 3; ++i) smooth_n[k[i].v] = smooth_n[k[i].v] + tri_n[t];
    }
    auto finite3 = [](f3 v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); };
    MeshData m;
    std::map<std::array<int64_t, 3>, uint32_t> seen;
    for (size_t t = 0; t < ntri; ++t) {
        for (int i = 0; i < 3; ++i) {
            const Corner &k = corners[3 * t + i];
            // A generated flat normal belongs to its face: key it by face.
            const int64_t nkey = k.n >= 0 ? k.n : (smooth ? -1 : -2 - static_cast<int64_t>(tri_face[t]));
            const std::array<int64_t, 3> key{k.v, k.t, nkey};
            auto it = seen.find(key);
            if (it != seen.end()) {
                m.idx.push_back(it->second);
                continue;
            }
            const uint32_t id = static_cast<uint32_t>(m.p.size());
            seen.emplace(key, id);
            m.p.push_back(P[k.v]);
            f3 n;
            if (k.n >= 0) {
                n = N[k.n];
            } else if (smooth) {
                const f3 sum = smooth_n[k.v];
                const float l = length(sum);
                n = l > 0.0f ? sum / l : f3{0.0f, 0.0f, 0.0f};
            } else {
                n = tri_n[t];
            }
            m.n.push_back(finite3(n) ? n : f3{0.0f, 0.0f, 0.0f});
            f2 uv = k.t >= 0 ? T[k.t] : f2{0.0f, 0.0f};
            if (k.t >= 0 && flip_uv) uv.y = 1.0f - uv.y;
            if (!std::isfinite(uv.x) || !std::isfinite(uv.y)) uv = f2{0.0f, 0.0f};
            m.uv.push_back(uv);
            m.idx.push_back(id);
        }
    }
    if (m.idx.empty()) throw std::runtime_error("model '" + path + "': no faces");
    return m;
}

// Sphere (src/render_core/shapes/sphere.cpp:17-87): a UV sphere of `radius`
// with sub_div rings of latitude (default 60) and twice as many meridians;
// a pole vertex at +y, the rings from the top (ring i at theta = pi i / n,
// vertex j at phi = 2 pi j / m, normal = position / radius, uv = (j/m, i/n)),
// a pole vertex at -y, then the top fan, the bands (two triangles per quad,
// the last quad of a ring wrapping to its first vertex) and the bottom fan,
// in the reference's vertex and index order so the triangles are the same.
MeshData make_sphere(float radius, uint32_t n) {
    if (n < 2u) throw std::runtime_error("sphere sub_div must be at least 2");
    const uint32_t m = 2u * n;
    MeshData s;
    s.p.push_back({0.0f, radius, 0.0f});
    s.n.push_back({0.0f, 1.0f, 0.0f});
    s.uv.push_back({0.0f, 0.0f});
    for (uint32_t i = 1; i < n; ++i) {
        const float v = static_cast<float>(i) / static_cast<float>(n);
        const float theta = kPi * v;
        const float y = radius * std::cos(theta), r = radius * std::sin(theta);
        for (uint32_t j = 0; j < m; ++j) {
            const float u = static_cast<float>(j) / static_cast<float>(m);
            const float phi = u * 2.0f * kPi;
            const f3 q = j == 0 ? f3{r, y, 0.0f} : f3{std::cos(phi) * r, y, std::sin(phi) * r};
            s.p.push_back(q);
            s.n.push_back(normalize(q));
            s.uv.push_back({j == 0 ? 0.0f : u, v});
        }
    }
    s.p.push_back({0.0f, -radius, 0.0f});
    s.n.push_back({0.0f, -1.0f, 0.0f});
    s.uv.push_back({0.0f, 1.0f});
    auto tri = [&](uint32_t a, uint32_t b, uint32_t c) {
        s.idx.push_back(a);
        s.idx.push_back(b);
        s.idx.push_back(c);
    };
    for (uint32_t i = 0; i < m; ++i) tri(0u, (i + 1u) % m + 1u, i + 1u);
    for (uint32_t i = 0; i + 2u < n; ++i) {
        uint32_t vs = 1u + i * m;
        for (uint32_t j = 0; j < m; ++j, ++vs) {
            if (j != m - 1u) {
                tri(vs, vs + 1u, vs + m);
                tri(vs + 1u, vs + m + 1u, vs + m);
            } else {
                tri(vs, vs + 1u - m, vs + m);
                tri(vs + 1u - m, vs + 1u, vs + m);
            }
        }
    }
    const uint32_t last = static_cast<uint32_t>(s.p.size()) - 1u;
    for (uint32_t i = 0; i < m; ++i) tri(last, last - ((1u + i) % m + 1u), last - (i + 1u));
    return s;
}

// Lattice value noise in [-1, 1] with smoothstep-weighted trilinear
// interpolation of hashed corner values.
float value_noise(f3 p, uint32_t seed) {
    auto hash = [&](int x, int y, int z) {
        uint32_t h = static_cast<uint32_t>(x) * 0x8da6b343u ^ static_cast<uint32_t>(y) * 0xd8163841u ^
                     static_cast<uint32_t>(z) * 0xcb1ab31fu ^ seed * 0x165667b1u;
        h ^= h >> 13;
        h *= 0x5bd1e995u;
        h ^= h >> 15;
        return static_cast<float>(h & 0xffffffu) * (2.0f / 16777215.0f) - 1.0f;
    };
    float fx = std::floor(p.x), fy = std::floor(p.y), fz = std::floor(p.z);
    int x = static_cast<int>(fx), y = static_cast<int>(fy), z = static_cast<int>(fz);
    float tx = p.x - fx, ty = p.y - fy, tz = p.z - fz;
    auto ss = [](float t) { return t * t * (3.0f - 2.0f * t); };
    tx = ss(tx); ty = ss(ty); tz = ss(tz);
    auto l = [](float t, float a, float b) { return a + t * (b - a); };
    float c00 = l(tx, hash(x, y, z), hash(x + 1, y, z)), c10 = l(tx, hash(x, y + 1, z), hash(x + 1, y + 1, z));
    float c01 = l(tx, hash(x, y, z + 1), hash(x + 1, y, z + 1)), c11 = l(tx, hash(x, y + 1, z + 1), hash(x + 1, y + 1, z + 1));
    return l(tz, l(ty, c00, c10), l(ty, c01, c11));
}

// Subdivided icosahedron on the unit sphere scaled to `radius`, displaced
// along the radius by `amplitude * radius * value_noise(frequency * p)`, with
// area-weighted smooth vertex normals and spherical uv.
MeshData make_icosphere(const Json &p) {
    uint32_t sub = p["subdivisions"].as_uint(4u);
    if (sub > 9) throw unsupported("icosphere subdivisions > 9");
    float radius = p["radius"].as_float(1.0f);
    const Json &dj = p["displacement"];
    float amp = dj["amplitude"].as_float(0.0f);
    float freq = dj["frequency"].as_float(4.0f);
    uint32_t seed = dj["seed"].as_uint(1u);
    const float t = (1.0f + std::sqrt(5.0f)) / 2.0f;
    std::vector<f3> v = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
                         {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
    for (f3 &q : v) q = normalize(q);
    std::vector<uint32_t> f = {0, 11, 5, 0, 5, 1, 0, 1, 7, 0, 7, 10, 0, 10, 11, 1, 5, 9, 5, 11, 4, 11, 10, 2, 10, 7, 6, 7, 1, 8,
                               3, 9, 4, 3, 4, 2, 3, 2, 6, 3, 6, 8, 3, 8, 9, 4, 9, 5, 2, 4, 11, 6, 2, 10, 8, 6, 7, 9, 8, 1};
    for (uint32_t level = 0; level < sub; ++level) {
        std::map<uint64_t, uint32_t> mid;
        auto midpoint = [&](uint32_t a, uint32_t b) {
            uint64_t key = a < b ? (static_cast<uint64_t>(a) << 32 | b) : (static_cast<uint64_t>(b) << 32 | a);
            auto it = mid.find(key);
            if (it != mid.end()) return it->second;
            uint32_t i = static_cast<uint32_t>(v.size());
            v.push_back(normalize((v[a] + v[b]) * 0.5f));
            mid[key] = i;
            return i;
        };
        std::vector<uint32_t> nf;
        nf.reserve(f.size() * 4);
        for (size_t k = 0; k + 2 < f.size(); k += 3) {
            uint32_t a = f[k], b = f[k + 1], c = f[k + 2];
            uint32_t ab = midpoint(a, b), bc = midpoint(b, c), ca = midpoint(c, a);
            uint32_t tris[12] = {a, ab, ca, b, bc, ab, c, ca, bc, ab, bc, ca};
            nf.insert(nf.end(), tris, tris + 12);
        }
        f.swap(nf);
    }
    MeshData m;
    m.p.resize(v.size());
    m.uv.resize(v.size());
    for (size_t i = 0; i < v.size(); ++i) {
        float r = radius * (1.0f + amp * value_noise(v[i] * freq, seed));
        m.p[i] = v[i] * r;
        float theta = std::acos(clampf(v[i].y, -1.0f, 1.0f));
        float phi = std::atan2(v[i].z, v[i].x);
        m.uv[i] = {phi * kInv2Pi + 0.5f, theta * kInvPi};
    }
    // Faces wind counter-clockwise seen from outside: cross(p0 - p2, p1 - p2)
    // points outward.
    m.idx = f;
    m.n.assign(v.size(), make3(0.0f));
    for (size_t k = 0; k + 2 < f.size(); k += 3) {
        f3 n = cross(m.p[f[k]] - m.p[f[k + 2]], m.p[f[k + 1]] - m.p[f[k + 2]]);
        for (int j = 0; j < 3; ++j) m.n[f[k + j]] += n;
    }
    return m;
}

// Regular grid in the xz plane, facing +y: nx x nz quads over size_x x size_z.
MeshData make_grid(const Json &p) {
    uint32_t nx = p["nx"].as_uint(1u), nz = p["nz"].as_uint(1u);
    if (nx == 0 || nz == 0 || static_cast<uint64_t>(nx) * nz > (1ull << 26)) throw unsupported("grid resolution");
    float sx = p["size_x"].as_float(1.0f), sz = p["size_z"].as_float(1.0f);
    MeshData m;
    for (uint32_t j = 0; j <= nz; ++j)
        for (uint32_t i = 0; i <= nx; ++i) {
            float u = static_cast<float>(i) / nx, w = static_cast<float>(j) / nz;
            m.p.push_back({(u - 0.5f) * sx, 0.0f, (w - 0.5f) * sz});
            m.n.push_back({0.0f, 1.0f, 0.0f});
            m.uv.push_back({u, w});
        }
    for (uint32_t j = 0; j < nz; ++j)
        for (uint32_t i = 0; i < nx; ++i) {
            uint32_t a = j * (nx + 1) + i, b = a + 1, c = a + nx + 1, d = c + 1;
            uint32_t q[6] = {c, b, a, c, d, b};
            m.idx.insert(m.idx.end(), q, q + 6);
        }
    return m;
}

// Normal-matrix transform (inverse transpose of the upper 3x3).
f3 xform_normal(const m4 &m, f3 n) {
    double a[3][3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) a[r][c] = m.m[c][r];
    double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                 a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
    double inv[3][3];
    inv[0][0] = (a[1][1] * a[2][2] - a[1][2] * a[2][1]) / det;
    inv[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) / det;
    inv[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) / det;
    inv[1][0] = (a[1][2] * a[2][0] - a[1][0] * a[2][2]) / det;
    inv[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) / det;
    inv[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) / det;
    inv[2][0] = (a[1][0] * a[2][1] - a[1][1] * a[2][0]) / det;
    inv[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) / det;
    inv[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) / det;
    // (inv)^T * n
    return {static_cast<float>(inv[0][0] * n.x + inv[1][0] * n.y + inv[2][0] * n.z),
            static_cast<float>(inv[0][1] * n.x + inv[1][1] * n.y + inv[2][1] * n.z),
            static_cast<float>(inv[0][2] * n.x + inv[1][2] * n.y + inv[2][2] * n.z)};
}

// calculate_alpha (src/base/scattering/microfacet.h:43-58).
void alpha_aniso(float a, float aniso, float &ax, float &ay) {
    if (std::fabs(aniso) <= 1e-4f) {
        ax = ay = a;
        return;
    }
    ax = aniso < 0.0f ? a / (1.0f + aniso) : a * (1.0f - aniso);
    ay = aniso < 0.0f ? a * (1.0f + aniso) : a / (1.0f - aniso);
}

// SPD::to_list (src/base/color/spd.h:41-47): samples every 5 nm from 360 nm
// while below 830 nm (94 samples).
template <typename F>
std::vector<float> to_list(F &&f) {
    std::vector<float> v;
    for (float l = kLambdaMin; l < kLambdaMax; l += 5.0f) v.push_back(f(l));
    return v;
}

// Named glasses (Sellmeier fits of glass.cpp:104-134; Schott catalogue data).
std::vector<float> sellmeier_curve(const std::string &name) {
    struct Coef { float b1, b2, b3, c1, c2, c3; };
    Coef c;
    if (name == "LASF9") c = {2.00029547f, 0.298926886f, 1.80691843f, 0.0121426017f, 0.0538736236f, 156.530829f};
    else c = {1.03961212f, 0.231792344f, 1.01046945f, 0.00600069867f, 0.0200179144f, 103.560653f};  // BK7 and unknown
    return to_list([&](float lambda) {
        float l = lambda / 1000.0f;
        float l2 = l * l;
        float f = c.b1 * l2 / (l2 - c.c1) + c.b2 * l2 / (l2 - c.c2) + c.b3 * l2 / (l2 - c.c3);
        return std::sqrt(f + 1.0f);
    });
}

// Cauchy dispersion n(lambda) = A + B / lambda^2, lambda in micrometres.  The
// reference has no Cauchy curve; it is expressed as an spd ior slot.
std::vector<float> cauchy_curve(float A, float B) {
    return to_list([&](float lambda) {
        float l = lambda / 1000.0f;
        return A + B / (l * l);
    });
}

// Procedural HDR sky in lat-long layout (row 0 at the zenith): a
// horizon-to-zenith gradient above the horizon, a dim ground below, and a sun
// lobe of `sun_radius` degrees whose radiance peaks at `sun_peak`.
std::vector<float> make_sky(const Json &p, uint32_t &W, uint32_t &H) {
    W = p["width"].as_uint(2048u);
    H = p["height"].as_uint(1024u);
    f3 zenith = as_f3(p["zenith"], make3(0.25f, 0.45f, 1.0f));
    f3 horizon = as_f3(p["horizon"], make3(1.0f, 0.95f, 0.85f));
    f3 ground = as_f3(p["ground"], make3(0.3f, 0.28f, 0.25f));
    float elev = p["sun_elevation"].as_float(35.0f) * kPi / 180.0f;
    float azim = p["sun_azimuth"].as_float(40.0f) * kPi / 180.0f;
    float radius = p["sun_radius"].as_float(5.0f) * kPi / 180.0f;
    float peak = p["sun_peak"].as_float(5e4f);
    f3 sun = {std::cos(elev) * std::cos(azim), std::cos(elev) * std::sin(azim), std::sin(elev)};
    std::vector<float> tex(static_cast<size_t>(W) * H * 4, 0.0f);
    for (uint32_t y = 0; y < H; ++y) {
        float theta = (y + 0.5f) / H * kPi;
        float e = 0.5f * kPi - theta;
        for (uint32_t x = 0; x < W; ++x) {
            float phi = (x + 0.5f) / W * k2Pi;
            f3 d = {std::sin(theta) * std::cos(phi), std::sin(theta) * std::sin(phi), std::cos(theta)};
            f3 c;
            if (e >= 0.0f) {
                float t = std::sqrt(e / (0.5f * kPi));
                c = horizon + (zenith - horizon) * t;
            } else {
                c = ground;
            }
            float ang = std::acos(clampf(dot(d, sun), -1.0f, 1.0f));
            if (ang < radius) c += make3(peak * 0.5f * (1.0f + std::cos(kPi * ang / radius)));
            float *t4 = &tex[(static_cast<size_t>(y) * W + x) * 4];
            t4[0] = c.x; t4[1] = c.y; t4[2] = c.z; t4[3] = 0.0f;
        }
    }
    return tex;
}

struct Loader {
    HostScene &s;
    const float *table;
    std::map<std::string, uint32_t> mat_by_name;
    std::string base_dir;  // model files are relative to the scene's folder
    bool srgb = false;     // RGB spectrum: colour slots are stored as RGB
    std::map<std::string, uint32_t> tex_by_key;  // texture ids by file and colour space
    std::vector<f3> tex_avg;                      // mean texel of each texture (ShaderNode::average)

    // The texture of an `image` node, loaded once per file and colour space.
    uint32_t texture(const Json &node) {
        const Json &p = node_param(node);
        const std::string key = p["fn"].as_string() + "|" + p["color_space"].as_string("");
        auto it = tex_by_key.find(key);
        if (it != tex_by_key.end()) return it->second;
        uint32_t w = 0, h = 0;
        std::vector<float> t = load_texture_texels(node, base_dir, w, h);
        TextureRec r{static_cast<uint32_t>(s.tex_texels.size() / 4), w, h, 0u};
        s.tex_texels.insert(s.tex_texels.end(), t.begin(), t.end());
        const uint32_t id = static_cast<uint32_t>(s.textures.size());
        s.textures.push_back(r);
        double sum[3] = {0.0, 0.0, 0.0};
        for (size_t i = 0; i < t.size(); i += 4)
            for (int c = 0; c < 3; ++c) sum[c] += t[i + c];
        const double n = static_cast<double>(w) * h;
        tex_avg.push_back({static_cast<float>(sum[0] / n), static_cast<float>(sum[1] / n), static_cast<float>(sum[2] / n)});
        tex_by_key[key] = id;
        return id;
    }

    // A colour slot that is an `image` node, or a `multiply` node (math.cpp)
    // of an image node and a constant: the texture and the constant factor.
    bool texture_slot(const Json &slot, uint32_t &id, f3 &factor) {
        const Json &n = slot_node(slot);
        if (!n.is_object()) return false;
        const std::string t = node_type(n);
        if (t == "image") {
            id = texture(n);
            factor = make3(1.0f);
            return true;
        }
        if (t != "multiply") return false;
        const Json &lhs = slot_node(n["param"]["lhs"]), &rhs = slot_node(n["param"]["rhs"]);
        const bool li = node_type(lhs) == "image";
        const bool ri = node_type(rhs) == "image";
        if (li == ri) throw unsupported("multiply node other than an image times a constant");
        id = texture(li ? lhs : rhs);
        factor = slot_rgb(n["param"][li ? "rhs" : "lhs"], make3(1.0f));
        return true;
    }

    // A material's colour slot: a constant stored through albedo_coef, or a
    // texture (flag kMatFlagTexture, id in p[7]) whose constant factor is
    // stored as RGB in coef; the device decodes each lookup.  Returns the
    // slot's average colour (the texture's mean texel times the factor).
    f3 colour_slot(const Json &slot, f3 def, Material &mat) {
        uint32_t id;
        f3 factor;
        if (texture_slot(slot, id, factor)) {
            mat.flags |= kMatFlagTexture;
            mat.p[7] = bits_float(id);
            mat.coef[0] = factor.x;
            mat.coef[1] = factor.y;
            mat.coef[2] = factor.z;
            mat.coef[3] = 0.0f;
            return {tex_avg[id].x * factor.x, tex_avg[id].y * factor.y, tex_avg[id].z * factor.z};
        }
        const f3 rgb = slot_rgb(slot, def);
        const float in[3] = {rgb.x, rgb.y, rgb.z};
        albedo_coef(in, mat.coef);
        return rgb;
    }

    // A colour slot as the material record stores it: sigmoid coefficients
    // for the hero spectrum (RGBAlbedoSpectrum), the colour itself for the
    // RGB spectrum (SRGBSpectrum::albedo_params, srgb.cpp:26-28).
    void albedo_coef(const float rgb[3], float out[4]) const {
        if (srgb) {
            out[0] = rgb[0];
            out[1] = rgb[1];
            out[2] = rgb[2];
            out[3] = 0.0f;
        } else {
            rgb2spec_decode_albedo(table, rgb, out);
        }
    }

    uint32_t add_spd(const float *v, int n) {
        uint32_t off = static_cast<uint32_t>(s.spd.size());
        s.spd.push_back(static_cast<float>(n));
        s.spd.insert(s.spd.end(), v, v + n);
        return off;
    }

    void load_material(const Json &m) {
        std::string type = m["type"].as_string("diffuse");
        std::string name = m["name"].as_string();
        const Json &p = m["param"];
        Material mat{};
        mat.spd0 = mat.spd1 = kInvalid;
        f3 rgb = make3(0.0f);
        if (type == "mix" || type == "add") {
            // MixMaterial / AddMaterial (mix.cpp:20-68, add.cpp:12-59): two
            // inline material nodes (MaterialDesc::init, node_desc.cpp:155-161)
            // loaded as records of their own (named after this one), and the
            // mix fraction slot (default 0.5).
            mat.type = kMatMix;
            if (type == "add") mat.flags |= kMatFlagAdd;
            else mat.p[0] = slot_scalar(p["frac"], 0.5f);
            uint32_t child[2];
            for (int k = 0; k < 2; ++k) {
                Json c = p[k == 0 ? "mat0" : "mat1"];
                if (!c.is_object()) throw std::runtime_error("material '" + name + "': missing mat" + std::to_string(k));
                const std::string ct = c["type"].as_string("diffuse");
                if (ct == "mix" || ct == "add") throw unsupported("mix / add material inside a mix / add (" + name + ")");
                if (ct == "black_body") throw unsupported("black_body inside a mix / add material (" + name + ")");
                c.set("name", Json::string(name + "/mat" + std::to_string(k)));
                load_material(c);
                child[k] = static_cast<uint32_t>(s.materials.size()) - 1u;
            }
            mat.spd0 = child[0];
            mat.spd1 = child[1];
        } else if (type == "diffuse") {
            // DiffuseMaterial: colour slot, default 0.5 (diffuse.cpp:37-44).
            mat.type = kMatDiffuse;
            rgb = colour_slot(p["color"], make3(0.5f), mat);
        } else if (type == "black_body") {
            mat.type = kMatBlackBody;
        } else if (type == "metal") {
            // MetalMaterial (metal.cpp:40-156): complex IOR of a named metal as
            // SPDs, GGX roughness remapped to alpha = r^2, anisotropy.
            mat.type = kMatMetal;
            std::string metal = p["material_name"].as_string();
            const float *eta = nullptr, *k = nullptr;
            static const struct {
                const char *name;
                const float *eta, *k;
            } kMetals[] = {
                {"Ag", VS_METAL_AG_ETA, VS_METAL_AG_K},       {"Al", VS_METAL_AL_ETA, VS_METAL_AL_K},
                {"Au", VS_METAL_AU_ETA, VS_METAL_AU_K},       {"Cu", VS_METAL_CU_ETA, VS_METAL_CU_K},
                {"CuZn", VS_METAL_CUZN_ETA, VS_METAL_CUZN_K}, {"Fe", VS_METAL_FE_ETA, VS_METAL_FE_K},
                {"Ti", VS_METAL_TI_ETA, VS_METAL_TI_K},       {"V", VS_METAL_V_ETA, VS_METAL_V_K},
                {"VN", VS_METAL_VN_ETA, VS_METAL_VN_K},       {"Li", VS_METAL_LI_ETA, VS_METAL_LI_K},
            };
            // An unknown or empty name falls back to silver.
            eta = VS_METAL_AG_ETA;
            k = VS_METAL_AG_K;
            for (const auto &mt : kMetals)
                if (metal == mt.name) {
                    eta = mt.eta;
                    k = mt.k;
                }
            mat.spd0 = add_spd(eta, 95);
            mat.spd1 = add_spd(k, 95);
            float r = clampf(slot_scalar(p["roughness"], 0.01f), 0.0001f, 1.0f);
            float aniso = clampf(slot_scalar(p["anisotropic"], 0.0f), -0.9f, 0.9f);
            bool remap = p["remapping_roughness"].as_bool(true);
            float a = remap ? r * r : r;
            alpha_aniso(a, aniso, mat.p[0], mat.p[1]);
            s.needs_luts = true;
        } else if (type == "metallic") {
            // MetallicMaterial (metallic.cpp:26-60): MetallicLobe, a
            // compensated GGX reflection with kr = colour and the F82-tint
            // Fresnel (F0 = colour, F82 = edge tint); roughness clamped to
            // [0.01, 1] and always remapped to alpha = r^2.
            mat.type = kMatMetal;
            mat.flags |= kMatFlagF82;
            rgb = colour_slot(p["color"], make3(1.0f), mat);
            const f3 et = slot_rgb(p["edge_tint"], make3(1.0f));
            const float ein[3] = {et.x, et.y, et.z};
            float ec[4];
            albedo_coef(ein, ec);
            mat.p[2] = ec[0];
            mat.p[3] = ec[1];
            mat.p[4] = ec[2];
            const float r = clampf(slot_scalar(p["roughness"], 0.5f), 0.01f, 1.0f);
            const float aniso = clampf(slot_scalar(p["anisotropic"], 0.0f), -0.9f, 0.9f);
            alpha_aniso(r * r, aniso, mat.p[0], mat.p[1]);
            s.needs_luts = true;
        } else if (type == "glass") {
            // GlassMaterial (glass.cpp:169-257): colour, ior (number, spd node,
            // named Sellmeier glass, or a Cauchy curve), roughness, anisotropy.
            mat.type = kMatGlass;
            rgb = colour_slot(p["color"], make3(1.0f), mat);
            std::string glass = p["material_name"].as_string();
            const Json &ior = p["ior"];
            const Json &ion = slot_node(ior);
            std::vector<float> curve;
            if (!glass.empty()) {
                curve = sellmeier_curve(glass);
            } else if (ion.is_object() && ion["type"].as_string() == "spd") {
                curve = (ion.contains("param") ? ion["param"]["value"] : ion["value"]).as_floats();
            } else if (ion.is_object() && ion["type"].as_string() == "cauchy") {
                const Json &cp = ion["param"];
                curve = cauchy_curve(cp["A"].as_float(1.5f), cp["B"].as_float(0.0f));
            }
            if (!curve.empty()) {
                if (curve.size() < 2) throw std::runtime_error("glass '" + name + "': ior spd needs >= 2 samples");
                mat.spd0 = add_spd(curve.data(), static_cast<int>(curve.size()));
                mat.flags |= kMatFlagDispersive;
            } else {
                mat.p[2] = slot_scalar(ior, 1.5f);
            }
            float r = clampf(slot_scalar(p["roughness"], 0.5f), 0.01f, 1.0f);
            float aniso = clampf(slot_scalar(p["anisotropic"], 0.0f), -0.9f, 0.9f);
            bool remap = p["remapping_roughness"].as_bool(true);
            float a = remap ? r * r : r;
            alpha_aniso(a, aniso, mat.p[0], mat.p[1]);
            s.needs_luts = true;
        } else if (type == "principled_bsdf") {
            // PrincipledBSDF (principled_bsdf.cpp:263-461).
            mat.type = kMatPrincipled;
            rgb = colour_slot(p["color"], make3(1.0f), mat);
            float r = clampf(slot_scalar(p["roughness"], 0.5f), 0.0001f, 1.0f);
            float aniso = slot_scalar(p["anisotropic"], 0.0f);
            float aspect = std::sqrt(1.0f - aniso * 0.9f);
            mat.p[0] = std::max(0.001f, r * r / aspect);
            mat.p[1] = std::max(0.001f, r * r * aspect);
            mat.p[2] = slot_scalar(p["metallic"], 0.0f);
            mat.p[3] = slot_scalar(p["ior"], 1.5f);
            f3 tint = slot_rgb(p["spec_tint"], make3(1.0f));
            float tin[3] = {tint.x, tint.y, tint.z}, tc[4];
            albedo_coef(tin, tc);
            mat.p[4] = tc[0]; mat.p[5] = tc[1]; mat.p[6] = tc[2];
            // Sheen, coat and transmission layers (initialize_slots,
            // principled_bsdf.cpp:287-302): when any weight is non-zero their
            // parameters go to a 12-float block of the SPD table at spd0:
            // sheen weight, roughness, tint (3 coefficients); coat weight,
            // roughness, ior, tint (3 coefficients); transmission weight.
            const float sheen_w = slot_scalar(p["sheen_weight"], 0.0f);
            const float coat_w = slot_scalar(p["coat_weight"], 0.0f);
            const float trans_w = slot_scalar(p["transmission_weight"], 0.0f);
            if (sheen_w != 0.0f || coat_w != 0.0f || trans_w != 0.0f) {
                f3 st = slot_rgb(p["sheen_tint"], make3(1.0f)), ct = slot_rgb(p["coat_tint"], make3(1.0f));
                float sin3[3] = {st.x, st.y, st.z}, cin3[3] = {ct.x, ct.y, ct.z}, sc[4], cc[4];
                albedo_coef(sin3, sc);
                albedo_coef(cin3, cc);
                const float block[12] = {sheen_w, slot_scalar(p["sheen_roughness"], 0.5f), sc[0], sc[1], sc[2],
                                         coat_w, slot_scalar(p["coat_roughness"], 0.2f),
                                         slot_scalar(p["coat_ior"], 1.5f), cc[0], cc[1], cc[2], trans_w};
                mat.spd0 = add_spd(block, 12);
            }
            s.needs_luts = true;
        } else if (type == "mirror") {
            // MirrorMaterial (mirror.cpp:18-74): the compensated GGX
            // reflection lobe of a metal with a constant Fresnel term and the
            // colour slot as kr; roughness default 0.001, remapped to r^2.
            mat.type = kMatMetal;
            mat.flags |= kMatFlagConstantFresnel;
            rgb = colour_slot(p["color"], make3(1.0f), mat);
            float r = clampf(slot_scalar(p["roughness"], 0.001f), 0.0001f, 1.0f);
            float aniso = clampf(slot_scalar(p["anisotropic"], 0.0f), -0.9f, 0.9f);
            float a = p["remapping_roughness"].as_bool(true) ? r * r : r;
            alpha_aniso(a, aniso, mat.p[0], mat.p[1]);
            s.needs_luts = true;
        } else if (type == "plastic") {
            // PlasticMaterial (plastic.cpp:80-129): colour (Rd, default 1), spec
            // (Rs, default 0.05), ior (default 1.3), roughness (default 0.5)
            // remapped twice like the substrate's; Schlick F0 = F0(ior) * Rs.
            mat.type = kMatSubstrate;
            mat.flags |= kMatFlagPlastic;
            rgb = colour_slot(p["color"], make3(1.0f), mat);
            f3 spec = slot_rgb(p["spec"], make3(0.05f));
            float sin[3] = {spec.x, spec.y, spec.z}, sc[4];
            albedo_coef(sin, sc);
            mat.p[2] = sc[0]; mat.p[3] = sc[1]; mat.p[4] = sc[2];
            mat.p[5] = clampf(slot_scalar(p["ior"], 1.3f), 1.003f, 5.0f);
            float r = clampf(slot_scalar(p["roughness"], 0.5f), 0.0001f, 1.0f);
            float aniso = clampf(slot_scalar(p["anisotropic"], 0.0f), -0.9f, 0.9f);
            const bool remap = p["remapping_roughness"].as_bool(true);
            alpha_aniso(remap ? r * r : r, aniso, mat.p[0], mat.p[1]);
            if (remap) {
                mat.p[0] = mat.p[0] * mat.p[0];
                mat.p[1] = mat.p[1] * mat.p[1];
            }
            mat.p[0] = clampf(mat.p[0], 0.0001f, 1.0f);
            mat.p[1] = clampf(mat.p[1], 0.0001f, 1.0f);
        } else if (type == "substrate") {
            // SubstrateMaterial (substrate.cpp:96-148): colour (Rd, default 1)
            // and spec (Rs, default 0.05) slots, roughness default 0.5.  With
            // remapping the reference squares the roughness and then the
            // anisotropic alphas once more; alphas clamp to [1e-4, 1].
            mat.type = kMatSubstrate;
            rgb = colour_slot(p["color"], make3(1.0f), mat);
            f3 spec = slot_rgb(p["spec"], make3(0.05f));
            float sin[3] = {spec.x, spec.y, spec.z}, sc[4];
            albedo_coef(sin, sc);
            mat.p[2] = sc[0]; mat.p[3] = sc[1]; mat.p[4] = sc[2];
            float r = clampf(slot_scalar(p["roughness"], 0.5f), 0.0001f, 1.0f);
            float aniso = clampf(slot_scalar(p["anisotropic"], 0.0f), -0.9f, 0.9f);
            const bool remap = p["remapping_roughness"].as_bool(true);
            alpha_aniso(remap ? r * r : r, aniso, mat.p[0], mat.p[1]);
            if (remap) {
                mat.p[0] = mat.p[0] * mat.p[0];
                mat.p[1] = mat.p[1] * mat.p[1];
            }
            mat.p[0] = clampf(mat.p[0], 0.0001f, 1.0f);
            mat.p[1] = clampf(mat.p[1], 0.0001f, 1.0f);
        } else {
            throw unsupported("material type '" + type + "' (" + name + ")");
        }
        mat_by_name[name] = static_cast<uint32_t>(s.materials.size());
        s.materials.push_back(mat);
        s.material_names.push_back(name);
        s.material_rgb.push_back(rgb);
    }

    uint32_t black_body_material() {
        auto it = mat_by_name.find("__black_body__");
        if (it != mat_by_name.end()) return it->second;
        Json j = Json::parse("{\"type\":\"black_body\",\"name\":\"__black_body__\",\"param\":{}}");
        load_material(j);
        return mat_by_name["__black_body__"];
    }

    // The object-space mesh of a new instance: an existing mesh with the same
    // positions and triangles, or a new one.
    uint32_t register_mesh(const MeshData &mesh) {
        uint64_t h = 1469598103934665603ull;
        auto mix = [&](const void *p, size_t n) {
            const unsigned char *c = static_cast<const unsigned char *>(p);
            for (size_t i = 0; i < n; ++i) h = (h ^ c[i]) * 1099511628211ull;
        };
        mix(mesh.p.data(), mesh.p.size() * sizeof(f3));
        mix(mesh.idx.data(), mesh.idx.size() * sizeof(uint32_t));
        for (uint32_t m = 0; m < s.meshes.size(); ++m) {
            const HostScene::MeshRec &r = s.meshes[m];
            if (r.hash != h || r.vertex_count != mesh.p.size() || 3u * r.tri_count != mesh.idx.size()) continue;
            if (std::memcmp(&s.mesh_pos[r.first_vertex], mesh.p.data(), mesh.p.size() * sizeof(f3)) == 0 &&
                std::memcmp(&s.mesh_idx[3u * r.first_tri], mesh.idx.data(), mesh.idx.size() * sizeof(uint32_t)) == 0)
                return m;
        }
        HostScene::MeshRec r{static_cast<uint32_t>(s.mesh_pos.size()), static_cast<uint32_t>(mesh.p.size()),
                             static_cast<uint32_t>(s.mesh_idx.size() / 3), static_cast<uint32_t>(mesh.idx.size() / 3), h};
        s.mesh_pos.insert(s.mesh_pos.end(), mesh.p.begin(), mesh.p.end());
        s.mesh_idx.insert(s.mesh_idx.end(), mesh.idx.begin(), mesh.idx.end());
        s.meshes.push_back(r);
        return static_cast<uint32_t>(s.meshes.size() - 1);
    }

    void add_mesh(const MeshData &mesh, const m4 &o2w, uint32_t mat, const std::string &name, const Json *emission) {
        uint32_t inst_id = static_cast<uint32_t>(s.instances.size());
        uint32_t vbase = static_cast<uint32_t>(s.pos.size());
        s.inst_mesh.push_back(register_mesh(mesh));
        s.inst_w2o.push_back(invert_affine(o2w));
        for (size_t i = 0; i < mesh.p.size(); ++i) {
            s.pos.push_back(xform_point(o2w, mesh.p[i]));
            s.nrm.push_back(is_zero(mesh.n[i]) ? mesh.n[i] : xform_normal(o2w, mesh.n[i]));
            s.uv.push_back(mesh.uv[i]);
        }
        Instance inst{};
        inst.mat_id = mat;
        inst.light_id = kInvalid;
        inst.first_prim = static_cast<uint32_t>(s.prim_inst.size());
        inst.prim_count = static_cast<uint32_t>(mesh.idx.size() / 3);
        for (size_t t = 0; t + 2 < mesh.idx.size(); t += 3) {
            for (int k = 0; k < 3; ++k) {
                uint32_t vi = mesh.idx[t + k];
                if (vi >= mesh.p.size()) throw std::runtime_error("mesh '" + name + "': index out of range");
                s.idx.push_back(vbase + vi);
            }
            s.prim_inst.push_back(inst_id);
        }
        if (emission) {
            inst.light_id = static_cast<uint32_t>(s.lights.size());
            add_area_light(*emission, inst_id, inst);
        }
        s.instances.push_back(inst);
        s.instance_names.push_back(name);
    }

    // Light::Light (light.cpp:10-17) + AreaLight (area.cpp:33-177).
    void add_area_light(const Json &em, uint32_t inst_id, const Instance &inst) {
        std::string type = em["type"].as_string("area");
        if (type != "area") throw unsupported("emission type '" + type + "'");
        const Json &p = em["param"];
        AreaLight L{};
        L.inst = inst_id;
        L.first_prim = inst.first_prim;
        L.prim_count = inst.prim_count;
        L.two_sided = p["two_sided"].as_bool(false) ? 1u : 0u;
        L.shape = kLightArea;
        emitter_colour(p, L);
        // Per-primitive alias table over world-space triangle areas.
        std::vector<float> areas;
        float total = 0.0f;
        for (uint32_t t = 0; t < inst.prim_count; ++t) {
            uint32_t pr = inst.first_prim + t;
            f3 p0 = s.pos[s.idx[3 * pr]], p1 = s.pos[s.idx[3 * pr + 1]], p2 = s.pos[s.idx[3 * pr + 2]];
            float a = 0.5f * length(cross(p0 - p2, p1 - p2));
            areas.push_back(a);
            total += a;
        }
        std::vector<AliasEntry> tab;
        std::vector<float> pmf;
        build_alias(areas, tab, pmf);
        L.alias_offset = static_cast<uint32_t>(s.prim_alias.size());
        s.prim_alias.insert(s.prim_alias.end(), tab.begin(), tab.end());
        s.prim_pmf.insert(s.prim_pmf.end(), pmf.begin(), pmf.end());
        // AreaLight::power (area.cpp:87-89).
        f3 power = L.two_sided ? make3(2.0f) * make3(L.rgb_avg[0], L.rgb_avg[1], L.rgb_avg[2]) * (total * kPi)
                               : make3(L.rgb_avg[0], L.rgb_avg[1], L.rgb_avg[2]) * (total * kPi);
        L.lum_power = linear_srgb_to_y(power);
        s.lights.push_back(L);
    }

    // PointLight (lights/point.cpp:20-43) and SpotLight (lights/spot.cpp:19-70)
    // of the light sampler's list: colour slot and scale as an area light's,
    // position; a spot adds its axis, cone angle (degrees, clamped to
    // [1, 89]) and falloff range (degrees, clamped to [0, angle]).
    void add_point_light(const std::string &type, const Json &p) {
        AreaLight L{};
        L.inst = L.first_prim = L.prim_count = L.alias_offset = kInvalid;
        L.shape = type == "spot" ? kLightSpot : kLightPoint;
        emitter_colour(p, L);
        const f3 pos = as_f3(p["position"], make3(0.0f));
        L.pos[0] = pos.x; L.pos[1] = pos.y; L.pos[2] = pos.z;
        const f3 avg = make3(L.rgb_avg[0], L.rgb_avg[1], L.rgb_avg[2]);
        if (L.shape == kLightPoint) {
            // PointLight::power: 4 pi * average.
            L.lum_power = linear_srgb_to_y(avg * (4.0f * kPi));
        } else {
            const f3 d = normalize(as_f3(p["direction"], make3(0.0f, 0.0f, 1.0f)));
            L.dir[0] = d.x; L.dir[1] = d.y; L.dir[2] = d.z;
            const float angle = clampf(p["angle"].as_float(45.0f), 1.0f, 89.0f) * kPi / 180.0f;
            const float falloff = std::min(std::max(p["falloff"].as_float(10.0f) * kPi / 180.0f, 0.0f), angle);
            L.cos_angle = std::cos(angle);
            L.cos_start = std::cos(std::max(0.0f, angle - falloff));
            // SpotLight::power: 2 pi * average * (1 - (2 angle + falloff) / 2), angles in radians.
            L.lum_power = linear_srgb_to_y(avg * (2.0f * kPi * (1.0f - 0.5f * (angle * 2.0f + falloff))));
        }
        s.lights.push_back(L);
    }

    // Projector (projector.cpp:30-126): a delta-position light at the origin
    // of `o2w` that projects its colour slot (an image node, alone or times a
    // constant, or a constant colour) through a pinhole looking along +z,
    // vertical half-angle `angle` (degrees, clamped to [1, 89]), width over
    // height `ratio` (0: the image's aspect).
    void add_projector(const Json &p) {
        AreaLight L{};
        L.inst = L.first_prim = L.prim_count = kInvalid;
        L.shape = kLightProjector;
        uint32_t tex = kInvalid;
        f3 factor = make3(1.0f);
        if (texture_slot(p["color"], tex, factor)) {
            // The texel times the factor is decoded per lookup as an
            // illumination (decode_to_illumination); an image is not
            // normalised (Light::Light applies NumberNode::normalize only).
            const float scale = p["scale"].is_number() ? p["scale"].as_float() : 1.0f;
            const f3 avg = {tex_avg[tex].x * factor.x, tex_avg[tex].y * factor.y, tex_avg[tex].z * factor.z};
            L.kind = kEmitRGB;
            L.scale = scale;
            L.coef[0] = factor.x;
            L.coef[1] = factor.y;
            L.coef[2] = factor.z;
            L.coef[3] = 0.0f;
            L.rgb_avg[0] = avg.x * scale;
            L.rgb_avg[1] = avg.y * scale;
            L.rgb_avg[2] = avg.z * scale;
            s.light_rgb.push_back(avg);
        } else {
            emitter_colour(p, L);
        }
        const m4 o2w = parse_transform(p["o2w"]);
        const m4 w2o = invert_affine(o2w);
        L.pos[0] = o2w.m[3][0];
        L.pos[1] = o2w.m[3][1];
        L.pos[2] = o2w.m[3][2];
        const f3 d = normalize(make3(o2w.m[2][0], o2w.m[2][1], o2w.m[2][2]));
        L.dir[0] = d.x;
        L.dir[1] = d.y;
        L.dir[2] = d.z;
        float ratio = p["ratio"].as_float(1.0f);
        if (ratio == 0.0f)
            ratio = tex != kInvalid ? static_cast<float>(s.textures[tex].width) / static_cast<float>(s.textures[tex].height)
                                    : 1.0f;
        const float angle = clampf(p["angle"].as_float(45.0f), 1.0f, 89.0f) * (kPi / 180.0f);
        const float tan_y = std::tan(angle);
        float block[kProjectorBlock] = {};
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 4; ++c) block[4 * r + c] = w2o.m[c][r];
        block[12] = ratio * tan_y;
        block[13] = tan_y;
        block[14] = bits_float(tex);
        L.alias_offset = static_cast<uint32_t>(s.spd.size());
        s.spd.insert(s.spd.end(), block, block + kProjectorBlock);
        // Projector::power (projector.cpp:60-90): the solid angle of a
        // frustum with 45-degree corners (the reference's formula, which does
        // not depend on `angle`) over 4 pi, times two, times the average.
        const float y = std::sqrt(1.0f / (ratio * ratio + 1.0f));
        const float x = ratio * y;
        const float z = std::sqrt(x * x + y * y);
        const f3 p0 = {x, y, z}, p1 = {x, -y, z}, p2 = {-x, -y, z};
        f3 c01 = cross(p0, p1), c12 = cross(p1, p2), c20 = cross(p2, p0);
        if (length_sq(c01) > 0.0f) c01 = normalize(c01);
        if (length_sq(c12) > 0.0f) c12 = normalize(c12);
        if (length_sq(c20) > 0.0f) c20 = normalize(c20);
        const float solid = std::fabs(std::acos(clampf(dot(c01, -c12), -1.0f, 1.0f)) +
                                      std::acos(clampf(dot(c12, -c20), -1.0f, 1.0f)) +
                                      std::acos(clampf(dot(c20, -c01), -1.0f, 1.0f)) - kPi);
        const f3 avg = make3(L.rgb_avg[0], L.rgb_avg[1], L.rgb_avg[2]);
        L.lum_power = linear_srgb_to_y(avg * ((2.0f * solid) / (4.0f * kPi)));
        s.lights.push_back(L);
    }

    // Light::Light (light.cpp:10-17): the colour slot (RGB illumination or the
    // blackbody emitter) and the scale, with RGB colours normalised so that
    // the largest channel is folded into the scale; also the average colour.
    void emitter_colour(const Json &p, AreaLight &L) {
        float scale = p["scale"].is_number() ? p["scale"].as_float() : 1.0f;
        f3 avg;
        if (is_blackbody_slot(p["color"])) {
            // New emitter: Planck spectrum normalised to a peak of one.
            const Json &n = slot_node(p["color"]);
            float T = n["param"]["temperature"].as_float(6500.0f);
            L.kind = kEmitBlackbody;
            L.coef[0] = T;
            L.coef[1] = 1.0f / planck(planck_peak_nm(T), T);
            // Average colour: linear sRGB of the normalised spectrum.
            double xyz[3] = {0, 0, 0};
            for (int i = 0; i < kCieSamples; ++i) {
                double e = planck(360.0f + i, T) * L.coef[1];
                xyz[0] += e * VS_CIE_X[i];
                xyz[1] += e * VS_CIE_Y[i];
                xyz[2] += e * VS_CIE_Z[i];
            }
            double yi = cie5().y_integral;
            avg = xyz_to_linear_srgb(make3(float(xyz[0] / yi), float(xyz[1] / yi), float(xyz[2] / yi)));
            s.light_rgb.push_back(avg);
        } else {
            f3 rgb = slot_rgb(p["color"], make3(1.0f));
            // NumberArray::normalize (number.cpp:40-48): fold the max channel into the scale.
            float mx = std::max(rgb.x, std::max(rgb.y, rgb.z));
            if (mx >= 1.0f) {
                rgb = rgb / mx;
                scale *= mx;
            }
            L.kind = kEmitRGB;
            float in[3] = {rgb.x, rgb.y, rgb.z};
            rgb2spec_decode_unbound(table, in, L.coef);
            avg = rgb;
            s.light_rgb.push_back(rgb);
        }
        L.scale = scale;
        L.rgb_avg[0] = avg.x * scale;
        L.rgb_avg[1] = avg.y * scale;
        L.rgb_avg[2] = avg.z * scale;
    }

    MeshData load_model(const Json &p) {
        if (p["subdiv_level"].as_uint(0u) != 0u) throw unsupported("model subdiv_level (Catmull-Clark subdivision)");
        const std::string fn = p["fn"].as_string();
        if (fn.empty()) throw std::runtime_error("model shape needs 'fn'");
        const bool absolute = fn[0] == '/';
        const std::string path = absolute || base_dir.empty() ? fn : base_dir + "/" + fn;
        const std::string ext = fn.size() >= 4 ? fn.substr(fn.size() - 4) : std::string();
        if (ext != ".obj" && ext != ".OBJ") throw unsupported("model format of '" + fn + "' (only Wavefront .obj)");
        return load_obj(path, p["smooth"].as_bool(false), p["flip_uv"].as_bool(true), p["swap_handed"].as_bool(false));
    }

    void load_shape(const Json &sh) {
        std::string type = sh["type"].as_string();
        std::string name = sh["name"].as_string();
        const Json &p = sh["param"];
        m4 o2w = parse_transform(p["transform"]);
        MeshData mesh;
        if (type == "quad") mesh = make_quad(p["width"].as_float(1.0f), p["height"].as_float(1.0f));
        else if (type == "cube") mesh = make_cube(p["x"].as_float(1.0f), p["y"].as_float(1.0f), p["z"].as_float(1.0f));
        else if (type == "mesh") mesh = make_inline_mesh(p);
        else if (type == "icosphere") mesh = make_icosphere(p);
        else if (type == "grid") mesh = make_grid(p);
        else if (type == "model") mesh = load_model(p);
        else if (type == "sphere") mesh = make_sphere(p["radius"].as_float(1.0f), p["sub_div"].as_uint(60u));
        else throw unsupported("shape type '" + type + "' (" + name + ")");
        const Json *emission = p.contains("emission") ? &p["emission"] : nullptr;
        uint32_t mat = kInvalid;
        std::string mname = p["material"].as_string();
        if (!mname.empty()) {
            auto it = mat_by_name.find(mname);
            if (it == mat_by_name.end()) throw std::runtime_error("shape '" + name + "': unknown material '" + mname + "'");
            mat = it->second;
        } else if (emission) {
            mat = black_body_material();
        }
        if (mat == kInvalid) mat = black_body_material();
        add_mesh(mesh, o2w, mat, name, emission);
    }
};

}  // namespace

// VisionRenderer::add_instance (src/sdk/vision.cpp:160-188, from_sdk_instance:
// vertices, triangles and the column-major o2w of an sdk::Instance) on the
// flattened scene: the mesh goes to world space like a JSON shape's.  The
// material is the name of a material of the scene, a material node as JSON
// text ({"type", "name", "param"}, MaterialDesc as the reference parses it),
// or empty for a default diffuse material.
uint32_t scene_add_instance(HostScene &s, const float *vertices40, uint32_t vert_num, const uint32_t *triangles,
                            uint32_t tri_num, const m4 &o2w, const std::string &material) {
    Loader ld{s, rgb2spec_table(""), {}, ""};
    ld.srgb = s.ip.srgb != 0u;
    for (size_t i = 0; i < s.material_names.size(); ++i) ld.mat_by_name[s.material_names[i]] = static_cast<uint32_t>(i);
    uint32_t mat = kInvalid;
    if (material.empty()) {
        auto it = ld.mat_by_name.find("__sdk_default__");
        if (it == ld.mat_by_name.end()) {
            ld.load_material(Json::parse("{\"type\":\"diffuse\",\"name\":\"__sdk_default__\",\"param\":{}}"));
            it = ld.mat_by_name.find("__sdk_default__");
        }
        mat = it->second;
    } else if (material[0] == '{') {
        Json m = Json::parse(material);
        std::string name = m["name"].as_string();
        if (!m.is_object()) throw std::runtime_error("add_instance: material JSON must be an object");
        if (name.empty() || ld.mat_by_name.count(name)) {
            name = "__sdk_material_" + std::to_string(s.materials.size()) + "__";
            m.set("name", Json::string(name));
        }
        ld.load_material(m);
        mat = ld.mat_by_name[name];
    } else {
        auto it = ld.mat_by_name.find(material);
        if (it == ld.mat_by_name.end()) throw std::runtime_error("add_instance: unknown material '" + material + "'");
        mat = it->second;
    }
    MeshData mesh;
    mesh.p.resize(vert_num);
    mesh.n.resize(vert_num);
    mesh.uv.resize(vert_num);
    for (uint32_t i = 0; i < vert_num; ++i) {
        const float *v = vertices40 + 10u * i;  // sdk::Vertex: pos[3], n[3], uv[2], uv2[2]
        mesh.p[i] = {v[0], v[1], v[2]};
        mesh.n[i] = {v[3], v[4], v[5]};
        mesh.uv[i] = {v[6], v[7]};
    }
    mesh.idx.assign(triangles, triangles + 3u * static_cast<size_t>(tri_num));
    const uint32_t inst = static_cast<uint32_t>(s.instances.size());
    ld.add_mesh(mesh, o2w, mat, "__sdk_instance_" + std::to_string(inst) + "__", nullptr);
    update_env_world(s);
    rebuild_light_alias(s);
    return inst;
}

// Pipeline::clear_geometry as the SDK's clear_geometries calls it
// (src/sdk/vision.cpp:120-123): every shape instance and the area lights they
// carry go; point, spot and environment lights stay, as do the materials.
void scene_clear_geometries(HostScene &s) {
    s.pos.clear();
    s.nrm.clear();
    s.uv.clear();
    s.idx.clear();
    s.prim_inst.clear();
    s.instances.clear();
    s.instance_names.clear();
    s.mesh_pos.clear();
    s.mesh_idx.clear();
    s.meshes.clear();
    s.inst_mesh.clear();
    s.inst_w2o.clear();
    s.tlas_inst.clear();
    s.blas_root.clear();
    s.two_level = false;
    std::vector<AreaLight> keep;
    std::vector<f3> keep_rgb;
    for (size_t i = 0; i < s.lights.size(); ++i)
        if (s.lights[i].shape != kLightArea) {
            keep.push_back(s.lights[i]);
            keep_rgb.push_back(s.light_rgb[i]);
        }
    s.lights = keep;
    s.light_rgb = keep_rgb;
    s.prim_alias.clear();
    s.prim_pmf.clear();
    s.nodes.clear();
    s.tri_v.clear();
    s.bvh_depth = 0;
    update_env_world(s);
    rebuild_light_alias(s);
}

void update_camera(HostScene &s, uint32_t width, uint32_t height) { s.cam = camera_at_resolution(s.cam, width, height); }

Camera camera_at_resolution(const Camera &base, uint32_t width, uint32_t height) {
    Camera c = base;
    c.width = width;
    c.height = height;
    // RadianceCollector::update_screen_window (radiance_collector.cpp:33-42).
    float ratio = static_cast<float>(width) / static_cast<float>(height);
    float lo_x = -1.0f, hi_x = 1.0f, lo_y = -1.0f, hi_y = 1.0f;
    if (ratio > 1.0f) {
        lo_x = -ratio; hi_x = ratio;
    } else {
        lo_y = -1.0f / ratio; hi_y = 1.0f / ratio;
    }
    c.screen_lo_x = lo_x;
    c.screen_hi_y = hi_y;
    c.screen_span_x = hi_x - lo_x;
    c.screen_span_y = hi_y - lo_y;
    return c;
}

// SphericalMap (spherical.cpp:26-215) with a procedural sky image and its
// AliasTable2D (alias2d.cpp:30-66) built from luminance * sin(theta) weights
// (calculate_weights, spherical.cpp:187-213).
static void load_spherical(const Json &p, const Json &root, HostScene &s, const std::string &base_dir) {
    const Json &cn = slot_node(p["color"]);
    const std::string ct = node_type(cn);
    if (ct != "sky" && ct != "image")
        throw unsupported("spherical light colour other than an 'image' or a procedural 'sky' node");
    uint32_t W, H;
    // The map's texels as the image node gives them (width along phi, height
    // along theta), or the procedural sky.
    s.env_tex = ct == "sky" ? make_sky(cn["param"], W, H) : load_texture_texels(cn, base_dir, W, H);
    EnvLight &e = s.env;
    e.width = W;
    e.height = H;
    e.scale = p["scale"].is_number() ? p["scale"].as_float() : 1.0f;
    // o2w_ = o2w * rotation_x(-90) * scale(1, -1, 1) (flip_u false); w2o = inverse.
    m4 o2w = parse_transform(p["o2w"]);
    bool flip_u = p["flip_u"].as_bool(false);
    m4 rx = rot_x(-90.0f) * scale_m(make3(1.0f, flip_u ? 1.0f : -1.0f, 1.0f));
    e.o2w = o2w * rx;
    e.w2o = invert_affine(e.o2w);
    // Warper weights.
    std::vector<float> weights(static_cast<size_t>(W) * H);
    double avg[3] = {0, 0, 0};
    for (size_t idx = 0; idx < weights.size(); ++idx) {
        const float *t = &s.env_tex[idx * 4];
        float v = static_cast<float>(idx / H) + 0.5f;
        float theta = v / W;
        float sin_theta = std::sin(kPi * theta);
        weights[idx] = linear_srgb_to_y(make3(t[0], t[1], t[2])) * sin_theta;
        for (int c = 0; c < 3; ++c) avg[c] += t[c];
    }
    std::vector<float> marginal_func(H);
    s.env_cond.clear();
    s.env_cond_func.clear();
    for (uint32_t v = 0; v < H; ++v) {
        std::vector<float> row(weights.begin() + static_cast<size_t>(v) * W, weights.begin() + static_cast<size_t>(v + 1) * W);
        std::vector<AliasEntry> tab;
        std::vector<float> pmf;
        float integral = 0.0f;
        build_alias(row, tab, pmf, &integral);
        marginal_func[v] = integral;
        s.env_cond.insert(s.env_cond.end(), tab.begin(), tab.end());
        s.env_cond_func.insert(s.env_cond_func.end(), row.begin(), row.end());
    }
    std::vector<float> mpmf;
    build_alias(marginal_func, s.env_marginal, mpmf, &e.integral);
    s.env_marginal_func = marginal_func;
    s.min_world_radius = root["render_setting"]["min_world_radius"].as_float(10.0f);
    double n = static_cast<double>(W) * H;
    s.env_avg = make3(float(avg[0] / n), float(avg[1] / n), float(avg[2] / n)) * e.scale;
    s.has_env = true;
    update_env_world(s);
}

void update_env_world(HostScene &s) {
    if (!s.has_env) return;
    EnvLight &e = s.env;
    // World bounds (Scene::world_radius: max(aabb radius, min_world_radius)).
    f3 lo = make3(3.4e38f), hi = make3(-3.4e38f);
    for (const f3 &q : s.pos) {
        lo = vmin(lo, q);
        hi = vmax(hi, q);
    }
    float radius = s.pos.empty() ? s.min_world_radius : std::max(0.5f * length(hi - lo), s.min_world_radius);
    e.world_diameter = 2.0f * radius;
    // SphericalMap::power (spherical.cpp:58-61).
    e.lum_power = linear_srgb_to_y(s.env_avg * (kPi * radius * radius));
}

// LightSampler::prepare with PowerLightSampler weights (power.cpp:16-30):
// one alias table over the lights' luminance powers, the environment last.
void rebuild_light_alias(HostScene &s) {
    std::vector<float> w;
    for (const AreaLight &L : s.lights) w.push_back(L.lum_power);
    if (s.has_env) w.push_back(s.env.lum_power);
    s.ip.light_count = static_cast<uint32_t>(w.size());
    s.light_alias.clear();
    s.light_pmf.clear();
    if (!w.empty()) build_alias(w, s.light_alias, s.light_pmf);
}

namespace {

// ReSTIR::ReSTIR with SpatialResamplingParam / TemporalResamplingParam
// (ReSTIR/common.h:19-67,91-98); thresholds as cos(radians(theta)).
RtStage load_rt_stage(const Json &d) {
    RtStage st{};
    st.open = d["open"].as_bool(true) ? 1u : 0u;
    st.diff_factor = d["diffuse_factor"].as_float(0.3f);
    st.max_age = d["max_age"].as_uint(30u);
    const Json &sp = d["spatial"];
    bool s_open = sp["open"].as_bool(true);
    st.spatial = s_open ? 1u : 0u;
    st.s_count = s_open ? sp["sample_num"].as_uint(1u) : 1u;
    if (st.s_count > kMaxSpatialNeighbours)
        throw unsupported("spatial sample_num above " + std::to_string(kMaxSpatialNeighbours));
    st.s_dot = std::cos(sp["theta"].as_float(35.0f) * (kPi / 180.0f));
    st.s_depth = sp["depth"].as_float(0.3f);
    st.s_radius = sp["radius"].as_float(30.0f);
    const Json &tp = d["temporal"];
    st.temporal = tp["open"].as_bool(true) ? 1u : 0u;
    st.history_limit = tp["history_limit"].as_uint(5u);
    st.t_count = tp["N"].as_uint(9u);
    st.t_mis = tp["mis"].as_bool(false) ? 1u : 0u;
    st.t_dot = std::cos(tp["theta"].as_float(35.0f) * (kPi / 180.0f));
    st.t_depth = tp["depth"].as_float(0.3f);
    st.t_radius = tp["radius"].as_float(8.0f);
    return st;
}

// RealTimeIntegrator (rt.cpp:24-31) with ReSTIRDI (direct.cpp:9-15) and
// ReSTIRGI (indirect.cpp:9-12).  The integrator keeps max_depth - 1 for the
// paths of the indirect samples.
void load_rt(const Json &ip, HostScene &s) {
    if (s.ip.spectrum_dim != 3) throw unsupported("rt integrator with a hero dimension other than 3");
    for (const Material &m : s.materials)
        if (m.type == kMatMix) throw unsupported("mix / add materials with the rt integrator");
    if (s.ip.max_depth < 3) throw unsupported("rt integrator with max_depth below 3");
    s.rt = true;
    s.ip.max_depth -= 1u;
    const Json &dj = ip["direct"];
    s.rt_di = load_rt_stage(dj);
    s.rt_gi = load_rt_stage(ip["indirect"]);
    // The denoiser node (SVGF::SVGF, svgf.h:41-51).  The reference turns SVGF
    // on from its GUI only; here vs_denoiser_enable does.  The OIDN and OptiX
    // denoisers are not built.
    const Json &dn = ip["denoiser"];
    if (dn.is_object()) {
        const std::string t = dn["type"].as_string();
        if (t != "svgf") throw unsupported("denoiser type '" + t + "'");
        const Json &dp = dn["param"];
        s.svgf.N = dp["N"].as_uint(3u);
        if (s.svgf.N > 10u) throw unsupported("SVGF with more than 10 a-trous iterations");
        s.svgf.alpha = dp["alpha"].as_float(0.05f);
        s.svgf.moments_alpha = dp["moments_alpha"].as_float(0.2f);
        s.svgf.history_limit = dp["history_limit"].as_uint(32u);
        s.svgf.moments_radius = dp["moments_filter_radius"].as_int(3);
        if (s.svgf.moments_radius < 0 || s.svgf.moments_radius > 5)
            throw unsupported("SVGF moments_filter_radius outside 0..5");
        s.svgf.sigma_rt = dp["sigma_rt"].as_float(10.0f);
        s.svgf.sigma_normal = dp["sigma_normal"].as_float(30.0f);
        s.svgf.reproject = dp["reproject"].as_bool(true) ? 1u : 0u;
        s.svgf.filter_moments = dp["filter_moments"].as_bool(true) ? 1u : 0u;
    }
    s.rt_gi.t_mis = 0u;
    s.rt_M_light = dj["M_light"].as_uint(10u);
    s.rt_M_bsdf = dj["M_bsdf"].as_uint(1u);
    s.rt_max_recursion = dj["max_recursion"].as_uint(5u);
    s.rt_pairwise = dj["pairwise"].as_bool(false) ? 1u : 0u;
}

}  // namespace

void load_scene_json(const std::string &text, const std::string &base_dir, const std::string &table_cache,
                     HostScene &s) {
    Json root = Json::parse(text);
    if (!table_cache.empty()) {
        size_t slash = table_cache.find_last_of('/');
        s.lut_cache = (slash == std::string::npos ? std::string() : table_cache.substr(0, slash + 1)) + "microfacet_luts.bin";
    }
    Loader ld{s, rgb2spec_table(table_cache), {}, base_dir};
    // Spectrum (SpectrumDesc, node_desc.cpp:346-350; hero.cpp:239).
    const Json &sp = root["spectrum"];
    // The schema's default is the RGB spectrum (SpectrumDesc::init: "srgb").
    s.spectrum_type = sp["type"].as_string("srgb");
    if (s.spectrum_type == "srgb") {
        // SRGBSpectrum: three RGB channels (Spectrum::dimension, spectrum.h:264).
        s.ip.srgb = 1u;
        s.ip.spectrum_dim = 3u;
    } else if (s.spectrum_type == "hero") {
        s.ip.srgb = 0u;
        s.ip.spectrum_dim = sp["param"]["dimension"].as_uint(3u);
        if (s.ip.spectrum_dim < 1 || s.ip.spectrum_dim > 4)
            throw unsupported("hero dimension " + std::to_string(s.ip.spectrum_dim));
    } else {
        throw unsupported("spectrum type '" + s.spectrum_type + "'");
    }
    ld.srgb = s.ip.srgb != 0u;
    {
        const Json &inst = root["render_setting"]["instancing"];
        s.instancing = inst.is_bool() ? (inst.as_bool() ? 2 : 0) : (inst.as_string("auto") == "auto" ? 1 : 0);
        // How the BVH8 picks each wide node's children (an extension key of
        // this library: the reference hands its triangles to OptiX).
        const std::string collapse = root["render_setting"]["bvh_collapse"].as_string("sah");
        if (collapse != "greedy" && collapse != "sah") throw unsupported("bvh_collapse '" + collapse + "'");
        s.bvh_sah_collapse = collapse == "sah";
        const Json &lj = root["render_setting"]["bvh_leaf_size"];
        if (lj.is_number()) {
            const uint32_t leaf = lj.as_uint(1u);
            if (leaf < 1u || leaf > 3u) throw unsupported("bvh_leaf_size " + std::to_string(leaf) + " (1 to 3)");
            s.bvh_leaf_size = leaf;
        } else if (lj.as_string("auto") != "auto") {
            throw unsupported("bvh_leaf_size '" + lj.as_string() + "' (1 to 3 or \"auto\")");
        } else {
            s.bvh_leaf_size = 0;
        }
    }
    // Materials, then shapes (which reference materials by name).
    for (const Json &m : root["materials"].elements()) ld.load_material(m);
    for (const Json &sh : root["shapes"].elements()) ld.load_shape(sh);
    if (s.prim_inst.empty()) throw std::runtime_error("scene has no primitives");
    // Light sampler (LightSamplerDesc, node_desc.cpp:318-328).
    const Json &lsj = root["light_sampler"];
    std::string lst = lsj["type"].as_string("uniform");
    if (lst == "uniform") s.ip.light_sampler = kLightSamplerUniform;
    else if (lst == "power") s.ip.light_sampler = kLightSamplerPower;
    else throw unsupported("light sampler '" + lst + "'");
    for (const Json &l : lsj["param"]["lights"].elements()) {
        std::string lt = l["type"].as_string("area");
        if (lt == "point" || lt == "spot") {
            ld.add_point_light(lt, l["param"]);
            continue;
        }
        if (lt == "projector") {
            ld.add_projector(l["param"]);
            continue;
        }
        if (lt != "spherical") throw unsupported("light type '" + lt + "' in light_sampler");
        if (s.has_env) throw unsupported("more than one environment light");
        load_spherical(l["param"], root, s, ld.base_dir);
    }
    s.ip.light_count = static_cast<uint32_t>(s.lights.size()) + (s.has_env ? 1u : 0u);
    if (s.ip.light_count == 0) throw unsupported("scene without lights");
    rebuild_light_alias(s);
    // Integrator (IlluminationIntegrator ctor, integrator.cpp:60-67).
    const Json &ij = root["integrator"];
    std::string it = ij["type"].as_string("pt");
    if (it != "pt" && it != "rt") throw unsupported("integrator type '" + it + "'");
    const Json &ip = ij["param"];
    s.ip.max_depth = ip["max_depth"].as_uint(16u);
    s.ip.min_depth = ip["min_depth"].as_uint(5u);
    s.ip.rr_threshold = ip["rr_threshold"].as_float(1.0f);
    s.ip.mis_mode = ip["mis_mode"].as_uint(0u);
    if (it == "rt") load_rt(ip, s);
    // Sampler.
    const Json &smp = root["sampler"];
    std::string st = smp["type"].as_string("independent");
    if (st == "independent") s.ip.sampler = kSamplerIndependent;
    else if (st == "pcg") s.ip.sampler = kSamplerPCG;
    else throw unsupported("sampler type '" + st + "'");
    s.ip.seed = smp["param"]["seed"].as_uint(0u);
    bool dispersive = false;
    for (const Material &m : s.materials) dispersive = dispersive || (m.flags & kMatFlagDispersive);
    // RGB transport has no dispersion (a glass IOR curve is read at one wavelength).
    s.ip.scatter_pdf_dim = dispersive && !s.ip.srgb ? s.ip.spectrum_dim : 1u;
    // Camera (SensorDesc, node_desc.cpp:84-95; Sensor::init, sensor.cpp:20-26).
    const Json &cj = root["camera"];
    std::string ct = cj["type"].as_string("pinhole");
    if (ct != "pinhole" && ct != "thin_lens") throw unsupported("camera type '" + ct + "'");
    const Json &cp = cj["param"];
    float fov = std::min(std::max(cp["fov_y"].as_float(20.0f), 15.0f), 120.0f);
    m4 m = parse_transform(cp["transform"]);
    float pitch = std::atan2(m.m[1][2], m.m[1][1]) * 180.0f / kPi;
    float yaw = std::atan2(m.m[2][0], m.m[0][0]) * 180.0f / kPi;
    f3 position = {m.m[3][0], m.m[3][1], m.m[3][2]};
    // Sensor::camera_to_world (sensor.cpp:163-172): T * scale(1,1,-1) * Ry(yaw) * Rx(-pitch).
    s.cam.c2w = translation(position) * scale_m(make3(1, 1, -1)) * rot_y(yaw) * rot_x(-pitch);
    s.cam.tan_half_fov = std::tan(fov * kPi / 180.0f * 0.5f);
    const Json &rc = cp["radiance_collector"]["param"];
    std::vector<float> res = rc["resolution"].as_floats();
    uint32_t w = res.size() >= 2 ? static_cast<uint32_t>(res[0]) : 1280u;
    uint32_t h = res.size() >= 2 ? static_cast<uint32_t>(res[1]) : 720u;
    s.cam.exposure = rc["exposure"].as_float(1.0f);
    // ToneMapperDesc (node_desc.cpp:201-207): radiance_collector.param.tone_mapper.type.
    const std::string tm = rc["tone_mapper"]["type"].as_string("linear");
    if (tm == "linear") s.tone_mapper = kToneLinear;
    else if (tm == "aces") s.tone_mapper = kToneAces;
    else if (tm == "reinhard") s.tone_mapper = kToneReinhard;
    else throw unsupported("tone mapper '" + tm + "'");
    // ThinLensCamera (thin_lens.cpp:11-20): lens radius and focal distance.
    s.cam.thin_lens = ct == "thin_lens" ? 1u : 0u;
    s.cam.lens_radius = cp["lens_radius"].as_float(0.0f);
    s.cam.focal_distance = cp["focal_distance"].as_float(5.0f);
    // FilterDesc (node_desc.cpp): type and radius, plus the fitted filters'
    // parameters (gaussian.cpp:18-24, mitchell.cpp, sinc.cpp).
    const Json &fj = cp["filter"];
    std::string ft = fj["type"].as_string("box");
    const Json &fp = fj["param"];
    std::vector<float> rad = fp["radius"].as_floats();
    s.cam.filter_rx = rad.size() >= 1 ? rad[0] : 0.5f;
    s.cam.filter_ry = rad.size() >= 2 ? rad[1] : s.cam.filter_rx;
    s.cam.filter_p0 = s.cam.filter_p1 = 0.0f;
    if (ft == "box") {
        s.cam.filter = kFilterBox;
    } else if (ft == "triangle") {
        s.cam.filter = kFilterTriangle;
    } else if (ft == "gaussian") {
        s.cam.filter = kFilterGaussian;
        s.cam.filter_p0 = fp["sigma"].as_float(1.0f);
    } else if (ft == "mitchell") {
        s.cam.filter = kFilterMitchell;
        s.cam.filter_p0 = fp["b"].as_float(1.0f / 3.0f);
        s.cam.filter_p1 = fp["c"].as_float(1.0f / 3.0f);
    } else if (ft == "sinc") {
        s.cam.filter = kFilterSinc;
        s.cam.filter_p0 = fp["tau"].as_float(3.0f);
    } else {
        throw unsupported("filter type '" + ft + "'");
    }
    build_filter_table(s.cam, s.filter_tab, s.filter_alias, s.filter_integral);
    update_camera(s, w, h);
}

}  // namespace vs

// Host-side scene representation and builders (C++17, no CUDA types).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "vs_math.h"
#include "vs_restir.h"
#include "vs_scene.h"
#include "vs_spectral.h"

namespace vs {

// Everything the kernels need, flattened: world-space vertices, primitives in
// instance order, materials, emitters, sampling tables, sensor and integrator
// settings.  Built from the scene JSON by load_scene_json().
struct HostScene {
    // Geometry (world space).
    std::vector<f3> pos;
    std::vector<f3> nrm;       // world-space vertex normals (not normalised)
    std::vector<f2> uv;
    std::vector<uint32_t> idx;  // 3 per primitive
    std::vector<uint32_t> prim_inst;
    std::vector<Instance> instances;
    std::vector<std::string> instance_names;
    // Materials.
    std::vector<Material> materials;
    std::vector<std::string> material_names;
    std::vector<f3> material_rgb;  // colour slot value before the uplift
    // Area lights (one per emissive instance) and their sampling tables.
    std::vector<AreaLight> lights;
    std::vector<f3> light_rgb;     // normalised colour slot value
    std::vector<AliasEntry> prim_alias;
    std::vector<float> prim_pmf;
    std::vector<AliasEntry> light_alias;
    std::vector<float> light_pmf;
    // Spectral samples of named SPDs (metal eta/k, glass ior), concatenated.
    std::vector<float> spd;
    // Spherical environment light (at most one) and its 2D alias warper.
    bool has_env = false;
    EnvLight env{};
    std::vector<float> env_tex;  // 4 floats (RGB, 0) per texel, row-major from the zenith
    // Textures of `image` shader nodes (colour slots): 4 floats per texel.
    std::vector<float> tex_texels;
    std::vector<TextureRec> textures;
    std::vector<AliasEntry> env_marginal, env_cond;
    std::vector<float> env_marginal_func, env_cond_func;
    f3 env_avg{};                  // average texel colour times the light's scale
    float min_world_radius = 10.0f; // render_setting.min_world_radius
    // Tabulated pixel filter (DeviceScene::filter_tab layout); empty for box
    // and triangle.
    std::vector<float> filter_tab;
    std::vector<AliasEntry> filter_alias;
    float filter_integral = 0.0f;
    // Tone mapper of the radiance collector (ToneMapper).
    uint32_t tone_mapper = 0;
    bool needs_luts = false;
    std::string lut_cache;
    Camera cam{};
    IntegratorParams ip{};
    // Real-time ReSTIR integrator (integrator type "rt", rt.cpp:24-31): the
    // settings of its direct and indirect stages.
    bool rt = false;
    RtStage rt_di{}, rt_gi{};
    uint32_t rt_M_light = 10, rt_M_bsdf = 1, rt_max_recursion = 5, rt_pairwise = 0;
    // SVGF denoiser settings (the integrator's "denoiser" node; svgf.h:41-51 defaults).
    SvgfParams svgf{3u, 0.05f, 0.2f, 32u, 3, 10.0f, 30.0f, 1u, 1u, {0u, 0u, 0u}};
    std::string spectrum_type = "hero";
    // Compressed BVH8 over the primitives.
    std::vector<Bvh8Node> nodes;
    std::vector<float> tri_v;  // 12 floats per primitive in leaf order
    uint32_t bvh_depth = 0;
    // Instancing (Geometry::build_accel builds one BLAS per mesh and an IAS
    // over the instances, geometry.cpp:20-52): the distinct object-space
    // meshes (shapes with equal vertices and triangles share one) and each
    // instance's mesh and world-to-object transform.  With instancing 2 (JSON
    // render_setting.instancing true) whenever some mesh has several
    // instances, and with 1 (the default, "auto") when the scene has at least
    // 2^20 triangles and 8 times those of its distinct meshes, build_bvh8 builds a
    // bottom-level BVH8 per mesh over its object-space
    // triangles (tri_v w = the triangle's index in its mesh) and a top-level
    // BVH8 over the instances' world boxes whose leaf entries index tlas_inst.
    struct MeshRec {
        uint32_t first_vertex, vertex_count, first_tri, tri_count;
        uint64_t hash;
    };
    std::vector<f3> mesh_pos;
    std::vector<uint32_t> mesh_idx;  // 3 per triangle, relative to the mesh's first vertex
    std::vector<MeshRec> meshes;
    std::vector<uint32_t> inst_mesh;  // per instance
    std::vector<m4> inst_w2o;         // per instance
    int instancing = 1;  // 0: one world-space BVH8; 1: auto; 2: two levels when any mesh is shared
    bool bvh_sah_collapse = true;  // wide-node children: SAH-optimal (true) or greedy (false)
    uint32_t bvh_leaf_size = 0;    // most triangles (or instances) per leaf child, 1..3; 0: by tree size
    bool two_level = false;
    uint32_t tlas_root = 0;
    std::vector<uint32_t> tlas_inst;  // top-level leaf entries: instance ids
    std::vector<uint32_t> blas_root;  // per mesh: root node index
};

// Parses a vision_scene.json document.  Throws std::runtime_error with a
// message naming the offending key or plugin type.
void load_scene_json(const std::string &text, const std::string &base_dir, const std::string &table_cache,
                     HostScene &scene);

// SDK geometry edits (src/sdk/vision.h:66-80): append a mesh instance
// (sdk::Vertex records of 10 floats, triangles as index triples, a column-major
// object-to-world matrix, a material name, JSON material node or "") and return
// its instance id; remove every shape instance and its area light.  Both keep
// the light sampler's tables and the environment's world bounds current; the
// scene needs build_bvh8 (vs_scene_build_accel) afterwards.
uint32_t scene_add_instance(HostScene &scene, const float *vertices40, uint32_t vert_num, const uint32_t *triangles,
                            uint32_t tri_num, const m4 &o2w, const std::string &material);
void scene_clear_geometries(HostScene &scene);
// Environment world diameter and power from the current geometry bounds;
// light-sampler alias table from the current lights.
void update_env_world(HostScene &scene);
void rebuild_light_alias(HostScene &scene);

// Sets resolution / camera-derived fields after load or on update.
void update_camera(HostScene &scene, uint32_t width, uint32_t height);
// A sensor at another resolution: same transform, filter and field of view,
// screen window of the new aspect ratio (radiance_collector.cpp:33-42).
Camera camera_at_resolution(const Camera &base, uint32_t width, uint32_t height);

// Builds the compressed BVH8 (nodes, tri_v) from pos/idx.
void build_bvh8(HostScene &scene);

// Vose alias table with the reference's layout and float arithmetic
// (src/render_core/warpers/alias.h:86-122); fills entries and the PMF of every
// entry (func / (integral * size)).
void build_alias(const std::vector<float> &weights, std::vector<AliasEntry> &entries, std::vector<float> &pmf,
                 float *integral = nullptr);

// RGB -> spectrum coefficient table (3 x 64^3 x float4) and its decoders.
const float *rgb2spec_table(const std::string &cache_path);
void rgb2spec_decode_albedo(const float *table, const float rgb[3], float out[4]);
void rgb2spec_decode_unbound(const float *table, const float rgb[3], float out[4]);

// Albedo tables of the compensated lobes (layout in vs_microfacet.h): the
// reference's shipped values, and the same tables regenerated from the lobe
// definitions (built on first use, cached in `cache_path`).
const float *microfacet_luts();
// The principled BSDF's tables as shipped by the reference: CoatLobe albedo
// (precomputed_table.h, 32^3) and the SheenLTC fits (ltc_sheen_table.h,
// Approximate mode, 32^2 x 4).
const float *coat_lut();
const float *sheen_ltc_lut();
const float *regenerate_microfacet_luts(const std::string &cache_path);

// CIE tables downsampled to the reference's 94-entry 5 nm SPDs and the CIE Y
// integral (src/base/color/spd.cpp:14-38).
struct Cie5 {
    float x[kSpd5Count], y[kSpd5Count], z[kSpd5Count], d65[kSpd5Count];
    float y_integral;
};
const Cie5 &cie5();

}  // namespace vs

// Device view of an uploaded scene, passed by value as a kernel parameter.
#pragma once

#include <cuda_runtime.h>
#include "vs_scene.h"

namespace vs {

// Everything a render kernel reads, passed by value as a kernel parameter.
struct DeviceScene {
    const uint4 *nodes;          // Bvh8Node array (5 uint4 per node)
    const float4 *tri_v;         // leaf-ordered triangles: 3 float4 each, w0 = prim id bits
    const float4 *vtx;           // 2 float4 per vertex: (pos.xyz, u), (normal.xyz, v)
    const uint4 *prims;          // per primitive: vertex indices i, j, k and instance id
    const Instance *instances;
    const Material *materials;
    const AreaLight *lights;
    const AliasEntry *prim_alias; // per-light alias tables over primitives
    const float *prim_pmf;        // PMF of each entry of prim_alias
    const AliasEntry *light_alias;// power light sampler
    const float *light_pmf;
    const float *spd;             // concatenated SPD sample arrays ([n, v0..v(n-1)] each)
    const float *luts;            // albedo tables of the compensated lobes (vs_microfacet.h offsets)
    // Environment light (only when has_env): texels as float4 RGB, the warper's
    // marginal / conditional alias tables and weights, the RGB->spectrum table.
    EnvLight env;
    uint32_t has_env;
    uint32_t env_index;           // light index of the environment (last)
    const float4 *env_tex;
    const float4 *tex_texels;     // textures of image nodes (TextureRec offsets)
    const uint4 *textures;        // TextureRec per texture
    const AliasEntry *env_marginal;
    const float *env_marginal_func;
    const AliasEntry *env_cond;
    const float *env_cond_func;
    const float4 *rgb2spec;       // 3 x 64^3 coefficient table
    // Tabulated pixel filter (Gaussian, Mitchell, sinc): kFilterTable^2 table
    // values over the filter's integral, the marginal function (kFilterTable)
    // and the conditional functions (kFilterTable^2); the marginal alias table
    // (kFilterTable) and the conditional ones (kFilterTable^2); the integral.
    const float *filter_tab;
    const AliasEntry *filter_alias;
    float filter_integral;
    Camera cam;
    IntegratorParams ip;
    uint32_t node_count;
    uint32_t prim_count;
    // Two-level scenes (instancing): node 0 is the top level's root, whose
    // leaf entries index tlas_inst (instance ids); per instance, inst_xf holds
    // 4 float4: the world-to-object rows (x' = r.x x + r.y y + r.z z + r.w)
    // and (root node of its mesh's BVH8, first global primitive, -, -) as bits.
    uint32_t two_level;
    const uint32_t *tlas_inst;
    const float4 *inst_xf;
    // Optional traversal counters (null in normal launches): [0] ray segments
    // traced, [1] BVH8 nodes visited, [2] triangle tests.
    unsigned long long *stats;
};

}  // namespace vs

// Per-pixel records and parameters of the real-time ReSTIR frame
// (src/render_core/integrators/rt.cpp, ReSTIR/direct.cpp, ReSTIR/indirect.cpp).
// POD, fixed size, 16-byte aligned so the kernels move them with vector loads.
// Reservoir weight sums are FP64; everything else is FP32.
#pragma once

#include "vs_math.h"
#include "vs_scene.h"
#include <cstdint>
#include <vector_types.h>

namespace vs {

// Upper bound on neighbours of one spatial pass (sample_num).
constexpr uint32_t kMaxSpatialNeighbours = 16;

// SurfaceData (src/base/scattering/interaction.h:15-44), 64 bytes.  `hit` is
// the last surface of the primary chain (after near-specular vertices);
// normal, linear depth and position are those of the first surface.
struct alignas(16) RtSurface {
    Hit hit;                    // inst_id == kInvalid: miss
    float nx, ny, nz, depth;    // normal_depth
    float px, py, pz, diffuse;  // pos_diff (position, diffuse factor)
    uint32_t is_replaced;
    uint32_t flag;              // BxDFFlag of the last surface's lobe set
    uint32_t pad0, pad1;
};
static_assert(sizeof(RtSurface) == 64, "RtSurface must be 64 bytes");

// SurfaceExtend (interaction.h:47-56), 32 bytes.
struct alignas(16) RtSurfaceExt {
    float tx, ty, tz;        // throughput of the near-specular chain
    float vx, vy, vz;        // view position seen by the last surface
    float t_max;             // accumulated chain distance along the camera ray
    uint32_t pad;
};
static_assert(sizeof(RtSurfaceExt) == 32, "RtSurfaceExt must be 32 bytes");

// HitBSDF (interaction.h:59-80), 32 bytes.
struct alignas(16) RtHitBsdf {
    float wx, wy, wz;
    float fx, fy, fz;  // first three channels of f (includes |cos|)
    float pdf;         // -1 when unset
    uint32_t pad;
};
static_assert(sizeof(RtHitBsdf) == 32, "RtHitBsdf must be 32 bytes");

// DIReservoir + DISample (src/render_core/integrators/ReSTIR/reservoir.h:15-115),
// 64 bytes.
struct alignas(16) DiReservoir {
    double weight_sum;
    float C, W;
    uint32_t light_index;  // kInvalid: no sample
    uint32_t prim_id;
    float bary_u, bary_v;
    uint32_t age;
    float p_hat;
    float pos[3];
    uint32_t pad[3];
};
static_assert(sizeof(DiReservoir) == 64, "DiReservoir must be 64 bytes");

// GIReservoir + GISample (reservoir.h:157-223), 64 bytes.
struct alignas(16) GiReservoir {
    double weight_sum;
    float C, W;
    float sp_pos[3];
    float sp_ng[3];
    float Lo[3];
    float age;
    uint32_t pad[2];
};
static_assert(sizeof(GiReservoir) == 64, "GiReservoir must be 64 bytes");

// Spatial / temporal resampling settings of one ReSTIR stage
// (common.h:19-67 with DIParam / GIParam, direct.h:14-38, indirect.h).
struct RtStage {
    uint32_t open;
    uint32_t spatial;        // spatial pass on
    uint32_t s_count;        // neighbours per spatial pass (sample_num)
    uint32_t temporal;       // temporal pass on
    uint32_t history_limit;
    uint32_t t_count;        // temporal fallback candidates (N)
    uint32_t t_mis;          // temporal pairwise MIS (direct only)
    uint32_t max_age;
    float diff_factor;
    float s_dot, s_depth, s_radius;
    float t_dot, t_depth, t_radius;
    uint32_t pad;
};

// Everything a ReSTIR kernel needs beyond the scene.
struct RtParams {
    RtStage di, gi;
    uint32_t M_light, M_bsdf;
    uint32_t max_recursion;
    uint32_t pairwise;        // direct spatial reuse: pairwise MIS combine
    uint32_t gi_max_depth;    // path length of the indirect sample (max_depth - 1)
    uint32_t frame;           // frame index (reservoir / surface buffer parity)
    uint32_t width, height;
    m4 w2c;                   // world -> camera of this frame (linear depth)
    m4 prev_w2c;              // world -> camera of the previous frame
    Camera prev_cam;          // previous frame's sensor (raster mapping)
    f3 view_pos;              // camera position of this frame
    f3 prev_view_pos;
    float di_factor, gi_factor;  // combine weights (ReSTIR::factor: open ? 1 : 0)
};

// Buffers of one ReSTIR frame.  Surfaces and reservoirs are double-buffered
// by frame parity: frame f writes index (f+1)&1 and reads the previous
// frame's data at f&1 (direct.h:136-145).  `*_pass` are the passthrough
// reservoirs between the temporal and the spatial pass.
struct RtBuffers {
    RtSurface *surf[2];
    RtSurfaceExt *ext[2];
    RtHitBsdf *hit_bsdf;
    float2 *motion;
    DiReservoir *di[2];
    DiReservoir *di_pass;
    GiReservoir *gi[2];
    GiReservoir *gi_pass;
    GiReservoir *gi_init;    // initial GI samples (GISample; W and C unused)
    float4 *di_radiance;
    float4 *gi_radiance;
    // Staged direct pass (null: one kernel): per pixel 4 float4 of sampler
    // state, wavelengths, film position and primary-ray direction; 2 float4
    // of the pending ray; the BSDF candidate's hit; the list of pixels that
    // see a surface; its length and the two traversal stages' fetch counters.
    float4 *di_stage;
    float4 *di_ray;
    Hit *di_hit;
    uint32_t *di_list;
    uint32_t *di_count;
    // Staged indirect spatial pass, kMaxSpatialNeighbours entries per pixel: neighbour index (bits) and weight; visibility ray;
    // visibility; the queued entries, their count and the fetch counter.
    float2 *gs_nb;
    float4 *gs_ray;
    uint8_t *gs_vis;
    uint32_t *gs_list;
    uint32_t *gs_count;
};

// SVGF denoiser of the real-time frame (src/render_core/denoisers/SVGF/).
// Settings (svgf.h:28-51; reproject / filter_moments are its pass switches),
// 48 bytes.
struct SvgfParams {
    uint32_t N;               // a-trous iterations (step widths 1, 2, 4, ...)
    float alpha;              // temporal blend of the illumination
    float moments_alpha;      // temporal blend of the moments
    uint32_t history_limit;
    int32_t moments_radius;   // spatial variance estimate while history < 4
    float sigma_rt;           // luminance edge stop
    float sigma_normal;       // normal edge stop (exponent)
    uint32_t reproject;
    uint32_t filter_moments;
    uint32_t pad[3];
};
static_assert(sizeof(SvgfParams) == 48, "SvgfParams must be 48 bytes");

// PixelGeometry (frame_buffer.h:15-21), 32 bytes: shading normal and its
// screen-space width, film position, depth gradient, linear depth (-1: the
// camera ray left the scene).
struct alignas(16) SvgfGeom {
    float nx, ny, nz, fwidth;
    float px, py;
    float depth_gradient;
    float linear_depth;
};
static_assert(sizeof(SvgfGeom) == 32, "SvgfGeom must be 32 bytes");

// SVGFData (utils.h:19-24), 32 bytes: demodulated illumination and its
// variance, history length, first and second luminance moments.
struct alignas(16) SvgfData {
    float ix, iy, iz, var;
    float history;
    float m1, m2;
    float pad;
};
static_assert(sizeof(SvgfData) == 32, "SvgfData must be 32 bytes");

// Buffers of the denoiser.  The G-buffer and the history lengths are
// double-buffered by frame parity (frame f writes (f+1)&1, reads f&1); the
// three SVGFData buffers rotate: `prev` holds the last frame's filtered
// result, `cur` and `tmp` take this frame's passes in turn.
struct SvgfBuffers {
    SvgfGeom *geom[2];
    float *history[2];
    float2 *motion;
    float4 *albedo;
    float4 *emission;
    SvgfData *data[3];
    const float4 *radiance;  // the frame's film (running mean), demodulated
    float4 *out;             // the denoised frame
};

}  // namespace vs

// Flat scene layout shared by the host builder, the device kernels and the
// scene export used by the tests.  Every struct here is POD and has a fixed
// size so it can be copied to HBM as is.
#pragma once

#include "vs_math.h"
#include <cstdint>

namespace vs {

// Material plugin types (reference: src/render_core/materials/*.cpp).
enum MaterialType : uint32_t {
    kMatDiffuse = 0,     // diffuse.cpp
    kMatBlackBody = 1,   // black_body.cpp: non-scattering emitter surface
    kMatMetal = 2,       // metal.cpp: GGX conductor with complex Fresnel
    kMatGlass = 3,       // glass.cpp: rough dielectric, optionally dispersive
    kMatPrincipled = 4,  // principled_bsdf.cpp
    kMatSubstrate = 5,   // substrate.cpp: FresnelBlend (glossy coat over diffuse)
    kMatMix = 6,         // mix.cpp / add.cpp: two materials' lobe sets; spd0 / spd1 hold their indices
};

enum MaterialFlag : uint32_t {
    kMatFlagDispersive = 1u,
    kMatFlagRemapRoughness = 2u,
    kMatFlagConstantFresnel = 4u,  // kMatMetal written by a `mirror` (mirror.cpp): F = 1, kr = colour
    kMatFlagPlastic = 8u,          // kMatSubstrate written by a `plastic` (plastic.cpp): PlasticLobe
    kMatFlagAdd = 16u,             // kMatMix written by an `add` (add.cpp): weights 1, sample weights 1/2
    kMatFlagTexture = 32u,         // colour slot from an `image` node: texture id in p[7] (bits), coef = RGB factor
    kMatFlagF82 = 64u,             // kMatMetal written by a `metallic` (metallic.cpp): F82 tint, edge tint in p[2..4]
};

// A texture of the `image` shader node: linear RGB texels (float4) at
// `offset` in the scene's texel array, width x height, row 0 the top.
struct TextureRec {
    uint32_t offset, width, height, pad;
};

// 64 bytes.  `coef` holds RGB->spectrum sigmoid coefficients (c0, c1, c2) of
// the albedo/colour slot; `p` holds the per-type scalar parameters.
struct alignas(16) Material {
    uint32_t type;
    uint32_t flags;
    uint32_t spd0;  // index into the SPD table (metal eta, glass ior) or kInvalid
    uint32_t spd1;  // metal k or kInvalid
    float coef[4];
    float p[8];
};

// Emission colour encodings of an area light.
enum EmitterKind : uint32_t {
    kEmitRGB = 0,        // RGB illumination slot: sigmoid(c) * scale2 * D65
    kEmitBlackbody = 1,  // Planck spectrum at temperature T, peak-normalised
};

// Shape of a light record: an emissive instance, or one of the delta
// lights of the light sampler's list (IPointLight, light.h:220-249).
// A projector keeps, at `alias_offset` in the SPD table, a 16-float block:
// world-to-light rows (3 x 4), tan of the horizontal and vertical
// half-angles, the texture id (bits; kInvalid for a constant colour) and 0.
enum LightShape : uint32_t { kLightArea = 0, kLightPoint = 1, kLightSpot = 2, kLightProjector = 3 };
constexpr uint32_t kProjectorBlock = 16;

// 112 bytes.  Point and spot lights leave the instance fields unused.
struct alignas(16) AreaLight {
    uint32_t inst;         // emitting instance
    uint32_t first_prim;   // first global primitive of the instance
    uint32_t prim_count;
    uint32_t alias_offset; // offset of this light's per-primitive alias table
    uint32_t two_sided;
    uint32_t kind;         // EmitterKind
    float scale;           // light scale after colour normalisation
    float lum_power;       // luminance of the light power (power light sampler)
    float coef[4];         // RGB: (c0, c1, c2, scale2); blackbody: (T, 1/peak, 0, 0)
    float rgb_avg[4];      // average colour * scale (reference Light::average)
    uint32_t shape;        // LightShape
    float cos_angle;       // spot: cos of the cone half-angle
    float cos_start;       // spot: cos of the angle where the falloff starts
    uint32_t pad;
    float pos[4];          // point, spot: position
    float dir[4];          // spot: unit axis
};

// One instance of a mesh in the flattened scene.
struct alignas(16) Instance {
    uint32_t mat_id;
    uint32_t light_id;    // kInvalid if not emissive
    uint32_t first_prim;
    uint32_t prim_count;
};

// Spherical environment map (src/render_core/lights/environments/spherical.cpp)
// with its 2D alias warper (src/render_core/warpers/alias2d.cpp).
struct alignas(16) EnvLight {
    m4 w2o;               // world -> map space (includes the map's x-rotation)
    m4 o2w;
    uint32_t width, height;
    float scale;
    float integral;       // marginal integral of the 2D warper
    float world_diameter; // distance of sampled light points
    float lum_power;      // luminance of pi r^2 * average colour (power light sampler)
    uint32_t pad0, pad1;
};

// Alias-table entry (reference src/render_core/warpers/alias.h AliasEntry).
struct AliasEntry {
    float prob;
    uint32_t alias;
};

// Pixel filters (src/render_core/filters): box and triangle sample in closed
// form; Gaussian, Mitchell and Lanczos-sinc through a 20 x 20 table of the
// filter over [0, r]^2 and a 2D alias warper (fitted_curve.h).
// Tone mappers of the radiance collector (tonemappers/impl.cpp).
enum ToneMapper : uint32_t { kToneLinear = 0, kToneAces = 1, kToneReinhard = 2 };

enum FilterType : uint32_t { kFilterBox = 0, kFilterTriangle = 1, kFilterGaussian = 2, kFilterMitchell = 3,
                             kFilterSinc = 4 };
constexpr uint32_t kFilterTable = 20;

// Pinhole or thin-lens sensor (pinhole.cpp, thin_lens.cpp) with its pixel
// filter.  Directions are built from the screen window the way
// src/base/sensor/sensor.cpp:44-76 builds raster_to_sensor.
struct alignas(16) Camera {
    m4 c2w;
    float tan_half_fov;
    float screen_lo_x, screen_hi_y;   // screen window lower.x, upper.y
    float screen_span_x, screen_span_y;
    float filter_rx, filter_ry;       // filter radius
    uint32_t width, height;
    float exposure;
    uint32_t filter;                  // FilterType
    uint32_t thin_lens;               // 1: ThinLensCamera (lens sample), 0: pinhole
    float lens_radius, focal_distance;
    float filter_p0, filter_p1;       // sigma (Gaussian), b and c (Mitchell), tau (sinc)
};
static_assert(sizeof(Camera) == 128, "Camera layout");

enum SamplerType : uint32_t { kSamplerIndependent = 0, kSamplerPCG = 1 };
enum LightSamplerType : uint32_t { kLightSamplerUniform = 0, kLightSamplerPower = 1 };

struct alignas(16) IntegratorParams {
    uint32_t max_depth;
    uint32_t min_depth;
    float rr_threshold;
    uint32_t mis_mode;        // 0 both, 1 light only, 2 BSDF only
    uint32_t spectrum_dim;    // hero wavelengths per path
    uint32_t scatter_pdf_dim; // spectrum_dim if any dispersive material else 1
    uint32_t sampler;         // SamplerType
    uint32_t seed;            // PCG seed
    uint32_t light_sampler;   // LightSamplerType
    uint32_t light_count;
    uint32_t srgb;            // 1: SRGBSpectrum (three RGB channels), 0: hero wavelengths
    uint32_t pad1;
};

// Compressed 8-wide BVH node: 80 bytes = 5 x 16-byte words.
//   w0: origin p (3 floats) | e[3] (biased float exponents of the grid step) | imask
//   w1: base_child | base_tri | meta[8]
//   w2..w4: qlo_x[8] qlo_y[8] qlo_z[8] qhi_x[8] qhi_y[8] qhi_z[8]
// Internal children of a node are stored contiguously from base_child in slot
// order; leaf children keep their triangles contiguously from base_tri and
// encode (count as unary bits << 5 | offset) in meta.
struct alignas(16) Bvh8Node {
    float px, py, pz;
    uint8_t e[3];
    uint8_t imask;
    uint32_t base_child;
    uint32_t base_tri;
    uint8_t meta[8];
    uint8_t qlo[3][8];
    uint8_t qhi[3][8];
};
static_assert(sizeof(Bvh8Node) == 80, "BVH8 node must be 80 bytes");

// Result of a closest-hit query (reference TriangleHit{inst_id, prim_id, bary}).
struct alignas(16) Hit {
    uint32_t inst_id;
    uint32_t prim_id;  // global primitive index in the flattened scene
    float u, v;        // barycentrics of vertex 1 and vertex 2
};

}  // namespace vs

// Small vector / matrix toolkit shared by host C++ (scene build, BVH build) and
// the sm_100a kernels.  Plain structs, no virtuals, usable in __constant__ and
// in device buffers.
#pragma once

#include <cstdint>
#include <cmath>

#if defined(__CUDACC__)
#define VS_HD __host__ __device__ __forceinline__
#else
#define VS_HD inline
#endif

namespace vs {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.31830988618379067154f;
constexpr float kInv2Pi = 0.15915494309189533577f;
constexpr float kInv4Pi = 0.07957747154594766788f;
constexpr float k2Pi = 6.28318530717958647692f;
// Largest float below one (0x1.fffffep-1).
constexpr float kOneMinusEpsilon = 0.99999994039535522461f;
// Shadow rays stop this far short of the light point (parametric, pbrt value).
constexpr float kShadowEpsilon = 0.0001f;
constexpr uint32_t kInvalid = 0xffffffffu;

// A product the device compiler may not fuse into a multiply-add: where a
// sum of products is shared by several inlined call sites, the choice of
// which product to fuse can differ between kernels, and with it the last
// bit of the result.
#if defined(__CUDA_ARCH__)
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
#else
inline float mul_rn(float a, float b) { return a * b; }
#endif

struct f2 { float x, y; };
struct f3 { float x, y, z; };
struct alignas(16) f4 { float x, y, z, w; };

VS_HD f2 make2(float x, float y) { return {x, y}; }
VS_HD f3 make3(float x, float y, float z) { return {x, y, z}; }
VS_HD f3 make3(float s) { return {s, s, s}; }
VS_HD f4 make4(float x, float y, float z, float w) { return {x, y, z, w}; }

VS_HD f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
VS_HD f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
VS_HD f3 operator-(f3 a) { return {-a.x, -a.y, -a.z}; }
VS_HD f3 operator*(f3 a, f3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
VS_HD f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
VS_HD f3 operator*(float s, f3 a) { return {a.x * s, a.y * s, a.z * s}; }
VS_HD f3 operator/(f3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
VS_HD f3 &operator+=(f3 &a, f3 b) { a = a + b; return a; }
VS_HD f2 operator+(f2 a, f2 b) { return {a.x + b.x, a.y + b.y}; }
VS_HD f2 operator-(f2 a, f2 b) { return {a.x - b.x, a.y - b.y}; }
VS_HD f2 operator*(f2 a, float s) { return {a.x * s, a.y * s}; }

VS_HD float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
VS_HD f3 cross(f3 a, f3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
VS_HD float length_sq(f3 a) { return dot(a, a); }
VS_HD float length(f3 a) { return sqrtf(dot(a, a)); }
VS_HD f3 normalize(f3 a) { return a * (1.0f / sqrtf(dot(a, a))); }
VS_HD float comp(f3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
VS_HD f3 vmin(f3 a, f3 b) { return {fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)}; }
VS_HD f3 vmax(f3 a, f3 b) { return {fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }
VS_HD float max3(f3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }
VS_HD float sqr(float x) { return x * x; }
VS_HD float pow5(float x) { const float x2 = x * x; return x2 * x2 * x; }
VS_HD float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
VS_HD float lerpf(float t, float a, float b) { return a + t * (b - a); }
VS_HD float safe_sqrt(float x) { return sqrtf(fmaxf(x, 0.0f)); }
VS_HD float safe_div(float a, float b) { return b == 0.0f ? 0.0f : a / b; }
VS_HD bool is_zero(f3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }
VS_HD f3 face_forward(f3 v, f3 ref) { return dot(v, ref) < 0.0f ? -v : v; }

VS_HD uint32_t float_bits(float f) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    uint32_t u; __builtin_memcpy(&u, &f, 4); return u;
#endif
}
VS_HD float bits_float(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f; __builtin_memcpy(&f, &u, 4); return f;
#endif
}

// Column-major 4x4 (m[c][r]); matches the scene schema, where the fourth JSON
// column holds the translation.
struct m4 {
    float m[4][4];
};

VS_HD m4 m4_identity() {
    m4 r{};
    for (int i = 0; i < 4; ++i) r.m[i][i] = 1.0f;
    return r;
}
VS_HD m4 operator*(const m4 &a, const m4 &b) {
    m4 r{};
    for (int c = 0; c < 4; ++c)
        for (int rr = 0; rr < 4; ++rr) {
            float s = 0.0f;
            for (int k = 0; k < 4; ++k) s += a.m[k][rr] * b.m[c][k];
            r.m[c][rr] = s;
        }
    return r;
}
VS_HD f3 xform_point(const m4 &a, f3 p) {
    float x = a.m[0][0] * p.x + a.m[1][0] * p.y + a.m[2][0] * p.z + a.m[3][0];
    float y = a.m[0][1] * p.x + a.m[1][1] * p.y + a.m[2][1] * p.z + a.m[3][1];
    float z = a.m[0][2] * p.x + a.m[1][2] * p.y + a.m[2][2] * p.z + a.m[3][2];
    float w = a.m[0][3] * p.x + a.m[1][3] * p.y + a.m[2][3] * p.z + a.m[3][3];
    if (w != 1.0f) return {x / w, y / w, z / w};
    return {x, y, z};
}
VS_HD f3 xform_vector(const m4 &a, f3 v) {
    return {a.m[0][0] * v.x + a.m[1][0] * v.y + a.m[2][0] * v.z,
            a.m[0][1] * v.x + a.m[1][1] * v.y + a.m[2][1] * v.z,
            a.m[0][2] * v.x + a.m[1][2] * v.y + a.m[2][2] * v.z};
}

// Orthonormal shading basis; to_local / to_world are plain projections.
struct Frame {
    f3 x, y, z;
    VS_HD f3 to_local(f3 v) const { return {dot(v, x), dot(v, y), dot(v, z)}; }
    VS_HD f3 to_world(f3 v) const { return x * v.x + y * v.y + z * v.z; }
};

}  // namespace vs

// Spherical environment light on the device: lookup, evaluation for escaped
// rays and importance sampling through the 2D alias warper.
// Restates src/render_core/lights/environments/spherical.cpp,
// src/render_core/warpers/alias2d.cpp and alias.h, and the RGB -> spectrum
// decode of RGBToSpectrumTable::decode_unbound (hero.cpp:92-141).
#pragma once

#include "vs_texture.cuh"

namespace vs {

// Bilinear lookup of the map (texel centres at (i + 0.5) / size, u wraps,
// v clamps).
__device__ __forceinline__ f3 env_texel(const DeviceScene &s, float u, float v) {
    const int W = static_cast<int>(s.env.width), H = static_cast<int>(s.env.height);
    float x = u * W - 0.5f, y = v * H - 0.5f;
    float fx = floorf(x), fy = floorf(y);
    float tx = x - fx, ty = y - fy;
    int x0 = static_cast<int>(fx), y0 = static_cast<int>(fy);
    int x1 = x0 + 1, y1 = y0 + 1;
    x0 = ((x0 % W) + W) % W;
    x1 = ((x1 % W) + W) % W;
    y0 = y0 < 0 ? 0 : (y0 > H - 1 ? H - 1 : y0);
    y1 = y1 < 0 ? 0 : (y1 > H - 1 ? H - 1 : y1);
    float4 a = __ldg(&s.env_tex[y0 * W + x0]), b = __ldg(&s.env_tex[y0 * W + x1]);
    float4 c = __ldg(&s.env_tex[y1 * W + x0]), d = __ldg(&s.env_tex[y1 * W + x1]);
    auto bl = [&](float p, float q, float r, float t) { return lerpf(ty, lerpf(tx, p, q), lerpf(tx, r, t)); };
    return {bl(a.x, b.x, c.x, d.x), bl(a.y, b.y, c.y, d.y), bl(a.z, b.z, c.z, d.z)};
}

// SphericalMap::L: the map's RGB decoded as an illumination spectrum.
template <int N>
__device__ __forceinline__ Spec<N> env_L(const DeviceScene &s, float u, float v, const Wavelengths<N> &wl) {
    f3 rgb = env_texel(s, u, v);
    Spec<N> r;
    if (is_rgb(wl)) {
        const float ch[3] = {rgb.x, rgb.y, rgb.z};
#pragma unroll
        for (int i = 0; i < N; ++i) r.v[i] = ch[i < 3 ? i : 2] * s.env.scale;
        return r;
    }
    float c[4];
    rgb2spec_unbound(s.rgb2spec, rgb, c);
#pragma unroll
    for (int i = 0; i < N; ++i)
        r.v[i] = sigmoid_poly(c[0], c[1], c[2], wl.lambda[i]) * c[3] * cie_spd(c_spec.d65, wl.lambda[i]) * s.env.scale;
    return r;
}

// AliasTable2D::PDF (alias2d.cpp:94-98).
__device__ __forceinline__ float env_map_pdf(const DeviceScene &s, float u, float v) {
    uint32_t W = s.env.width, H = s.env.height;
    uint32_t iu = min(static_cast<uint32_t>(fmaxf(u * W, 0.0f)), W - 1u);
    uint32_t iv = min(static_cast<uint32_t>(fmaxf(v * H, 0.0f)), H - 1u);
    return s.env.integral > 0.0f ? __ldg(&s.env_cond_func[iv * W + iu]) / s.env.integral : 0.0f;
}

// spherical_theta / spherical_phi of a map-space direction.
__device__ __forceinline__ void env_uv(f3 local, float &u, float &v, float &sin_theta) {
    float theta = acosf(clampf(local.z, -1.0f, 1.0f));
    float phi = atan2f(local.y, local.x);
    if (phi < 0.0f) phi += k2Pi;
    u = phi * kInv2Pi;
    v = theta * kInvPi;
    sin_theta = sinf(theta);
}

// SphericalMap::evaluate_wi for a world direction (escaped rays).
template <int N>
__device__ VS_OUTLINE void env_eval(const DeviceScene &s, f3 world_dir, const Wavelengths<N> &wl, Spec<N> &L,
                                         float &pdf) {
    f3 local = xform_vector(s.env.w2o, world_dir);
    float u, v, st;
    env_uv(local, u, v, st);
    L = env_L<N>(s, u, v, wl);
    float p = env_map_pdf(s, u, v) / (k2Pi * kPi * st);
    pdf = st == 0.0f ? 0.0f : p;
}

// AliasTable::sample_continuous (alias.h:148-181) over one alias table.
__device__ __forceinline__ float alias_continuous(const AliasEntry *table, uint32_t size, float u, uint32_t &ofs) {
    u = u * static_cast<float>(size);
    uint32_t idx = min(static_cast<uint32_t>(u), size - 1u);
    u = fminf(u - static_cast<float>(idx), kOneMinusEpsilon);
    AliasEntry e = table[idx];
    bool keep = u < e.prob;
    float ur = keep ? fminf(u / e.prob, kOneMinusEpsilon) : fminf((1.0f - u) / (1.0f - e.prob), kOneMinusEpsilon);
    ofs = keep ? idx : e.alias;
    return (static_cast<float>(ofs) + ur) / static_cast<float>(size);
}

// SphericalMap::sample_wi -> AliasTable2D::sample_continuous (alias2d.cpp:100-120)
// and SphericalMap::evaluate (spherical.cpp:117-138).
template <int N>
__device__ VS_OUTLINE void env_sample(const DeviceScene &s, f3 p_ref, f2 u, const Wavelengths<N> &wl, Spec<N> &L,
                                           float &pdf, f3 &p_light) {
    uint32_t W = s.env.width, H = s.env.height;
    uint32_t iv;
    float fv = alias_continuous(s.env_marginal, H, u.y, iv);
    float pdf_v = s.env.integral > 0.0f ? __ldg(&s.env_marginal_func[iv]) / s.env.integral : 0.0f;
    uint32_t iu;
    float fu = alias_continuous(s.env_cond + static_cast<size_t>(iv) * W, W, u.x, iu);
    float integral_u = __ldg(&s.env_marginal_func[iv]);
    float func_u = __ldg(&s.env_cond_func[static_cast<size_t>(iv) * W + iu]);
    float pdf_u = integral_u > 0.0f ? func_u / integral_u : 0.0f;
    float pdf_map = pdf_u * pdf_v;
    float theta = fv * kPi, phi = fu * k2Pi;
    float st = sinf(theta), ct = cosf(theta);
    f3 local = {st * cosf(phi), st * sinf(phi), ct};
    f3 world_dir = normalize(xform_vector(s.env.o2w, local));
    float p = pdf_map / (k2Pi * kPi * st);
    pdf = isinf(p) ? 0.0f : p;
    L = env_L<N>(s, fu, fv, wl);
    p_light = p_ref + world_dir * s.env.world_diameter;
}

// SphericalMap::sample_only (spherical.cpp:127-132): the map coordinates of a
// sampled direction alone (the light-surface point a reservoir stores).
__device__ __forceinline__ f2 env_sample_uv(const DeviceScene &s, f2 u) {
    uint32_t iv, iu;
    const float fv = alias_continuous(s.env_marginal, s.env.height, u.y, iv);
    const float fu = alias_continuous(s.env_cond + static_cast<size_t>(iv) * s.env.width, s.env.width, u.x, iu);
    return {fu, fv};
}

// SphericalMap::evaluate_point -> evaluate (spherical.cpp:105-125,134-141) for
// stored map coordinates: the radiance, the solid-angle pdf from the map's
// own PDF(uv), and the world direction (compute_light_eval_context,
// spherical.cpp:148-160, places the light point world_diameter along it).
template <int N>
__device__ __forceinline__ void env_eval_uv(const DeviceScene &s, float u, float v, const Wavelengths<N> &wl,
                                            Spec<N> &L, float &pdf, f3 &world_dir) {
    const float theta = v * kPi, phi = u * k2Pi;
    const float st = sinf(theta), ct = cosf(theta);
    const f3 local = {st * cosf(phi), st * sinf(phi), ct};
    world_dir = normalize(xform_vector(s.env.o2w, local));
    const float p = env_map_pdf(s, u, v) / (k2Pi * kPi * st);
    pdf = isinf(p) ? 0.0f : p;
    L = env_L<N>(s, u, v, wl);
}

// Environment::convert_to_bary (spherical.cpp:70-73): map coordinates of a
// world direction.
__device__ __forceinline__ f2 env_dir_uv(const DeviceScene &s, f3 world_dir) {
    float u, v, st;
    env_uv(normalize(xform_vector(s.env.w2o, world_dir)), u, v, st);
    return {u, v};
}

}  // namespace vs

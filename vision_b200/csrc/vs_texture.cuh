// Colour slots on the device: the RGB -> spectrum decode of the coefficient
// table (RGBToSpectrumTable::decode_albedo / decode_unbound, hero.cpp:92-141)
// and the `image` shader node's texture lookup (shadernodes/image.cpp:80-88)
// with the albedo decode a material applies to it
// (ShaderNodeSlot::eval_albedo_spectrum, shader_node.cpp:299-303).
#pragma once

#include "vs_device.cuh"

namespace vs {

// RGBToSpectrumTable::decode_albedo: sigmoid coefficients of rgb clamped to
// [0, 1], by the table's trilinear interpolation (the host loader's
// rgb2spec_decode_albedo with the same operation order).
__device__ __forceinline__ void rgb2spec_albedo(const float4 *table, f3 rgb_in, float c[3]) {
    const f3 q = {clampf(rgb_in.x, 0.0f, 1.0f), clampf(rgb_in.y, 0.0f, 1.0f), clampf(rgb_in.z, 0.0f, 1.0f)};
    if (q.x == q.y && q.y == q.z) {
        c[0] = 0.0f;
        c[1] = 0.0f;
        c[2] = (q.x - 0.5f) / sqrtf(q.x * (1.0f - q.x));
        return;
    }
    const int res = 64;
    uint32_t maxc = (q.x > q.y) ? ((q.x > q.z) ? 0u : 2u) : ((q.y > q.z) ? 1u : 2u);
    float z = comp(q, maxc);
    float x = comp(q, (maxc + 1u) % 3u) * (res - 1u) / z;
    float y = comp(q, (maxc + 2u) % 3u) * (res - 1u) / z;
    auto inv_ss = [](float v) { return 0.5f - sinf(asinf(1.0f - 2.0f * v) * (1.0f / 3.0f)); };
    float zz = inv_ss(inv_ss(z)) * (res - 1u);
    uint32_t xi = min(static_cast<uint32_t>(x), static_cast<uint32_t>(res - 2));
    uint32_t yi = min(static_cast<uint32_t>(y), static_cast<uint32_t>(res - 2));
    uint32_t zi = min(static_cast<uint32_t>(zz), static_cast<uint32_t>(res - 2));
    float dx = x - xi, dy = y - yi, dz = zz - zi;
    auto co = [&](int ox, int oy, int oz) {
        return __ldg(&table[(((static_cast<size_t>(maxc) * res + (zi + oz)) * res + (yi + oy)) * res + (xi + ox))]);
    };
    float4 c000 = co(0, 0, 0), c100 = co(1, 0, 0), c010 = co(0, 1, 0), c110 = co(1, 1, 0);
    float4 c001 = co(0, 0, 1), c101 = co(1, 0, 1), c011 = co(0, 1, 1), c111 = co(1, 1, 1);
    auto tri = [&](float a000, float a100, float a010, float a110, float a001, float a101, float a011, float a111) {
        float x00 = lerpf(dx, a000, a100), x10 = lerpf(dx, a010, a110);
        float x01 = lerpf(dx, a001, a101), x11 = lerpf(dx, a011, a111);
        return lerpf(dz, lerpf(dy, x00, x10), lerpf(dy, x01, x11));
    };
    c[0] = tri(c000.x, c100.x, c010.x, c110.x, c001.x, c101.x, c011.x, c111.x);
    c[1] = tri(c000.y, c100.y, c010.y, c110.y, c001.y, c101.y, c011.y, c111.y);
    c[2] = tri(c000.z, c100.z, c010.z, c110.z, c001.z, c101.z, c011.z, c111.z);
}

// RGBToSpectrumTable::decode_unbound: the coefficients of rgb / (2 max) and
// the scale 2 max in c[3].
__device__ __forceinline__ void rgb2spec_unbound(const float4 *table, f3 rgb_in, float c[4]) {
    f3 rgb = vmax(rgb_in, make3(0.0f));
    float m = max3(rgb);
    float scale = 2.0f * m;
    f3 q = scale == 0.0f ? make3(0.0f) : rgb / scale;
    c[3] = scale;
    rgb2spec_albedo(table, q, c);
}

// The texel of an `image` node's texture at uv: bilinear between the four
// nearest texel centres ((i + 0.5) / size), both axes repeating, row 0 of
// the file at v = 0.
__device__ __forceinline__ f3 texture_rgb(const DeviceScene &s, uint32_t id, f2 uv) {
    const uint4 r = __ldg(&s.textures[id]);
    const int W = static_cast<int>(r.y), H = static_cast<int>(r.z);
    const float4 *t = s.tex_texels + r.x;
    float x = (uv.x - floorf(uv.x)) * W - 0.5f, y = (uv.y - floorf(uv.y)) * H - 0.5f;
    float fx = floorf(x), fy = floorf(y);
    float tx = x - fx, ty = y - fy;
    int x0 = static_cast<int>(fx), y0 = static_cast<int>(fy);
    int x1 = x0 + 1, y1 = y0 + 1;
    x0 = x0 < 0 ? x0 + W : (x0 >= W ? x0 - W : x0);
    x1 = x1 < 0 ? x1 + W : (x1 >= W ? x1 - W : x1);
    y0 = y0 < 0 ? y0 + H : (y0 >= H ? y0 - H : y0);
    y1 = y1 < 0 ? y1 + H : (y1 >= H ? y1 - H : y1);
    const float4 a = __ldg(&t[y0 * W + x0]), b = __ldg(&t[y0 * W + x1]);
    const float4 c = __ldg(&t[y1 * W + x0]), d = __ldg(&t[y1 * W + x1]);
    auto bl = [&](float p, float q, float u, float v) { return lerpf(ty, lerpf(tx, p, q), lerpf(tx, u, v)); };
    return {bl(a.x, b.x, c.x, d.x), bl(a.y, b.y, c.y, d.y), bl(a.z, b.z, c.z, d.z)};
}

// A material's colour slot at uv: the record's constant (albedo_spectrum of
// its coefficients), or for kMatFlagTexture the texture lookup times the
// constant factor held in coef, decoded as an albedo (the RGB spectrum keeps
// the colour itself, SRGBSpectrum::decode_to_albedo, srgb.cpp:50-52).
template <int N>
__device__ __forceinline__ Spec<N> colour_spectrum(const DeviceScene &s, const Material &m, f2 uv,
                                                   const Wavelengths<N> &wl) {
    if (!(m.flags & kMatFlagTexture)) return albedo_spectrum<N>(m.coef, wl);
    const f3 t = texture_rgb(s, __float_as_uint(m.p[7]), uv);
    const f3 rgb = {t.x * m.coef[0], t.y * m.coef[1], t.z * m.coef[2]};
    Spec<N> r;
    if (is_rgb(wl)) {
        const float ch[3] = {rgb.x, rgb.y, rgb.z};
#pragma unroll
        for (int i = 0; i < N; ++i) r.v[i] = ch[i < 3 ? i : 2];
        return r;
    }
    float c[3];
    rgb2spec_albedo(s.rgb2spec, rgb, c);
#pragma unroll
    for (int i = 0; i < N; ++i) r.v[i] = sigmoid_poly(c[0], c[1], c[2], wl.lambda[i]);
    return r;
}

}  // namespace vs

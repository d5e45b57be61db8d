// sm_100a kernels of the SVGF denoiser of the real-time frame
// (src/render_core/denoisers/SVGF/, SVGF::dispatch svgf.cpp:86-101), one
// thread per pixel on 16 x 16 tiles:
//   k_svgf_geom      the G-buffer: film position, shading normal, linear depth,
//                    material albedo, emission, motion vector
//                    (FrameBuffer::compute_geom, frame_buffer.cpp:72-122)
//   k_svgf_gradient  normal width and depth gradient over the 3 x 3
//                    neighbourhood (FrameBuffer::compute_gradient, :124-171)
//   k_svgf_demod     illumination = (radiance - emission) / albedo
//                    (Modulator demodulate, modulator.cpp:26-36)
//   k_svgf_reproject temporal accumulation of illumination and moments with
//                    history (Reproject, reproject.cpp:13-160)
//   k_svgf_moments   spatial variance estimate while history < 4
//                    (FilterMoments, filter_moments.cpp:13-66)
//   k_svgf_atrous    edge-stopping a-trous pass, one launch per step width
//                    (AtrousFilter, atrous.cpp:13-94)
//   k_svgf_mod       output = illumination * albedo + emission
//                    (Modulator modulate, modulator.cpp:15-24)
// The reference's moment filter and a-trous passes write the buffer whose
// neighbouring pixels they read, and its reprojection writes the history
// buffer it reads at the reprojected pixel, so its results depend on thread
// scheduling.  Here every pass reads one buffer and writes another (the
// published algorithm, Schied et al. 2017) and the history is double-buffered
// by frame parity, so the result is deterministic.
#include "vs_integrator.cuh"
#include "vs_launch.h"
#include "vs_restir.h"

namespace vs {

namespace {

constexpr int kSvgfTile = 16;

__device__ __forceinline__ bool svgf_pixel(const RtParams &p, int &x, int &y) {
    x = static_cast<int>(blockIdx.x * kSvgfTile + threadIdx.x);
    y = static_cast<int>(blockIdx.y * kSvgfTile + threadIdx.y);
    return x < static_cast<int>(p.width) && y < static_cast<int>(p.height);
}

__device__ __forceinline__ uint32_t pix(const RtParams &p, int x, int y) {
    return static_cast<uint32_t>(y) * p.width + static_cast<uint32_t>(x);
}

__device__ __forceinline__ bool in_screen(const RtParams &p, int x, int y) {
    return x >= 0 && y >= 0 && x < static_cast<int>(p.width) && y < static_cast<int>(p.height);
}

// make_int2 of a float: toward zero, saturating.
__device__ __forceinline__ int f2i_rz(float v) { return __float2int_rz(v); }

__device__ __forceinline__ f3 nrm(const SvgfGeom &g) { return {g.nx, g.ny, g.nz}; }
__device__ __forceinline__ f3 illum(const SvgfData &d) { return {d.ix, d.iy, d.iz}; }

// The hero wavelengths the real-time frame samples for a pixel (its own
// sampler stream; RGB transport keeps the sRGB primaries).
__device__ __forceinline__ Wavelengths<3> frame_wavelengths(const DeviceScene &s, uint32_t x, uint32_t y,
                                                            uint32_t frame) {
    if (s.ip.srgb) return rgb_wavelengths<3>();
    Sampler w;
    w.start(x, y, frame, 0xffffffffu, s.ip.sampler, s.ip.seed);
    return sample_wavelengths<3>(w.next());
}

// Sensor::prev_raster_coord (sensor.cpp:105-110): the previous frame's raster
// position of a world point.
__device__ __forceinline__ f2 prev_raster(const RtParams &p, f3 world) {
    f3 c = xform_point(p.prev_w2c, world);
    float a = c.x / c.z, b = c.y / c.z;
    const Camera &k = p.prev_cam;
    float sx = a / k.tan_half_fov, sy = b / k.tan_half_fov;
    return {(sx - k.screen_lo_x) / k.screen_span_x * static_cast<float>(k.width),
            (k.screen_hi_y - sy) / k.screen_span_y * static_cast<float>(k.height)};
}

// SVGF::cal_weight (svgf.cpp:68-77).
__device__ __forceinline__ float cal_weight(float z, float zn, float sigma_z, f3 n, f3 nn, float sigma_n, float l,
                                            float ln, float sigma_l) {
    const float w_normal = powf(clampf(dot(n, nn), 0.0f, 1.0f), sigma_n);
    const float w_depth = sigma_z == 0.0f ? 0.0f : fabsf(z - zn) / sigma_z;
    const float w_illum = fabsf(l - ln) / sigma_l;
    return expf(-(fmaxf(w_illum, 0.0f) + fmaxf(w_depth, 0.0f))) * w_normal;
}

__device__ __forceinline__ float lerp_to(float t, float a, float b) { return a + t * (b - a); }

__global__ void __launch_bounds__(256) k_svgf_geom(const __grid_constant__ DeviceScene s,
                                                   const __grid_constant__ RtParams p,
                                                   const __grid_constant__ SvgfBuffers b) {
    int x, y;
    if (!svgf_pixel(p, x, y)) return;
    const uint32_t idx = pix(p, x, y), cur = (p.frame + 1u) & 1u;
    const Wavelengths<3> wl = frame_wavelengths(s, x, y, p.frame);
    Sampler smp;
    smp.start(x, y, p.frame, 0u, s.ip.sampler, s.ip.seed);
    f2 p_film;
    f3 ro, rd;
    (void)camera_ray(s, s.cam, smp, x, y, p_film, ro, rd);
    SvgfGeom g{0.0f, 0.0f, 0.0f, 0.0f, p_film.x, p_film.y, 0.0f, -1.0f};
    f3 albedo = make3(0.0f), emission = make3(0.0f);
    f2 mv = make2(0.0f, 0.0f);
    Hit h;
    float t;
    if (trace_closest(s, precompute_ray(ro, rd), 3.402823466e+38f, h, t)) {
        const Interaction it = surface_interaction(s, h, rd, true);
        const f3 n = it.shading.z;
        g.nx = n.x;
        g.ny = n.y;
        g.nz = n.z;
        g.linear_depth = xform_point(p.w2c, it.pos).z;
        if (it.mat != kInvalid) {
            const Bsdf<3> bsdf = make_bsdf<3>(s, s.materials[it.mat], it.shading, it.ng, it.wo, it.uv, wl);
            albedo = linear_srgb<3>(bsdf.albedo(dot(n, it.wo)), wl);
        }
        if (it.light != kInvalid) {
            // LightSampler::evaluate_hit_wi with p_ref at the ray origin.
            Spec<3> Le;
            float pdf;
            eval_hit_light<3>(s, it, ro, wl, Le, pdf);
            emission = linear_srgb<3>(Le, wl);
        }
        // FrameBuffer::compute_motion_vec (frame_buffer.cpp:325-333).
        mv = p_film - prev_raster(p, it.pos);
    }
    b.geom[cur][idx] = g;
    b.motion[idx] = make_float2(mv.x, mv.y);
    b.albedo[idx] = make_float4(albedo.x, albedo.y, albedo.z, 1.0f);
    b.emission[idx] = make_float4(emission.x, emission.y, emission.z, 1.0f);
}

// Writes only the width and gradient fields, which no neighbour reads.
__global__ void __launch_bounds__(256) k_svgf_gradient(const __grid_constant__ RtParams p,
                                                       const __grid_constant__ SvgfBuffers b) {
    int x, y;
    if (!svgf_pixel(p, x, y)) return;
    SvgfGeom *geom = b.geom[(p.frame + 1u) & 1u];
    const SvgfGeom c = geom[pix(p, x, y)];
    uint32_t xn = 0u, yn = 0u;
    f3 ndx = make3(0.0f), ndy = make3(0.0f);
    float ddx = 0.0f, ddy = 0.0f;
    const int x0 = max(0, x - 1), x1 = min(x + 1, static_cast<int>(p.width) - 1);
    const int y0 = max(0, y - 1), y1 = min(y + 1, static_cast<int>(p.height) - 1);
    for (int qx = x0; qx <= x1; ++qx) {
        for (int qy = y0; qy <= y1; ++qy) {
            const SvgfGeom q = geom[pix(p, qx, qy)];
            if (x > qx) {
                xn += 1u;
                ndx = ndx + (nrm(c) - nrm(q));
                ddx += c.linear_depth - q.linear_depth;
            } else if (qx > x) {
                xn += 1u;
                ndx = ndx + (nrm(q) - nrm(c));
                ddx += q.linear_depth - c.linear_depth;
            }
            if (y > qy) {
                yn += 1u;
                ndy = ndy + (nrm(c) - nrm(q));
                ddy += c.linear_depth - q.linear_depth;
            } else if (qy > y) {
                yn += 1u;
                ndy = ndy + (nrm(q) - nrm(c));
                ddy += q.linear_depth - c.linear_depth;
            }
        }
    }
    const float fx = static_cast<float>(xn), fy = static_cast<float>(yn);
    ndx = make3(ndx.x / fx, ndx.y / fx, ndx.z / fx);
    ndy = make3(ndy.x / fy, ndy.y / fy, ndy.z / fy);
    const f3 fw = make3(fabsf(ndx.x) + fabsf(ndy.x), fabsf(ndx.y) + fabsf(ndy.y), fabsf(ndx.z) + fabsf(ndy.z));
    SvgfGeom *o = geom + pix(p, x, y);
    o->fwidth = length(fw);
    o->depth_gradient = fabsf(ddx / fx) + fabsf(ddy / fy);
}

__global__ void __launch_bounds__(256) k_svgf_demod(const __grid_constant__ RtParams p,
                                                    const __grid_constant__ SvgfBuffers b, uint32_t cur_d) {
    int x, y;
    if (!svgf_pixel(p, x, y)) return;
    const uint32_t idx = pix(p, x, y);
    const float4 r = b.radiance[idx], e = b.emission[idx], a = b.albedo[idx];
    SvgfData d{};
    d.ix = (r.x - e.x) / fmaxf(a.x, 0.001f);
    d.iy = (r.y - e.y) / fmaxf(a.y, 0.001f);
    d.iz = (r.z - e.z) / fmaxf(a.z, 0.001f);
    b.data[cur_d][idx] = d;
}

// Reproject::is_valid_reproject (reproject.cpp:13-28).
__device__ __forceinline__ bool valid_reproject(const RtParams &p, const SvgfGeom &c, const SvgfGeom &q) {
    const bool inside = in_screen(p, f2i_rz(q.px), f2i_rz(q.py));
    const bool z_ok = (fabsf(c.linear_depth - q.linear_depth) / (c.depth_gradient + 1e-2f)) < 10.0f;
    const bool n_ok = (length(nrm(c) - nrm(q)) / (c.fwidth + 1e-2f)) < 16.0f;
    return inside && z_ok && n_ok;
}

__global__ void __launch_bounds__(256) k_svgf_reproject(const __grid_constant__ RtParams p,
                                                        const __grid_constant__ SvgfParams sp,
                                                        const __grid_constant__ SvgfBuffers b, uint32_t cur_d,
                                                        uint32_t prev_d) {
    int x, y;
    if (!svgf_pixel(p, x, y)) return;
    const uint32_t idx = pix(p, x, y);
    const uint32_t cur = (p.frame + 1u) & 1u, prev = p.frame & 1u;
    const SvgfGeom g = b.geom[cur][idx];
    SvgfData d = b.data[cur_d][idx];
    f3 il = illum(d);
    const float2 mv = b.motion[idx];
    // Reproject::load_prev_data (reproject.cpp:30-120).
    const float ppx = g.px - mv.x, ppy = g.py - mv.y;
    const int px = f2i_rz(ppx - 0.5f), py = f2i_rz(ppy - 0.5f);
    const bool inside = in_screen(p, px, py);
    f3 prev_il = make3(0.0f);
    float pm1 = 0.0f, pm2 = 0.0f;
    bool v[4] = {false, false, false, false};
    bool valid = false;
    const int ox[4] = {0, 1, 0, 1}, oy[4] = {0, 0, 1, 1};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int qx = px + ox[i], qy = py + oy[i];
        if (in_screen(p, qx, qy)) {
            v[i] = valid_reproject(p, g, b.geom[prev][pix(p, qx, qy)]);
            valid = valid || v[i];
        }
    }
    if (valid) {
        float wsum = 0.0f;
        const float fx = ppx - floorf(ppx), fy = ppy - floorf(ppy);
        const float w[4] = {(1.0f - fx) * (1.0f - fy), fx * (1.0f - fy), (1.0f - fx) * fy, fx * fy};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int qx = px + ox[i], qy = py + oy[i];
            if (v[i] && in_screen(p, qx, qy)) {
                const SvgfData q = b.data[prev_d][pix(p, qx, qy)];
                prev_il = prev_il + illum(q) * w[i];
                pm1 += w[i] * q.m1;
                pm2 += w[i] * q.m2;
                wsum += w[i];
            }
        }
        valid = wsum >= 0.01f;
        prev_il = valid ? prev_il / wsum : make3(0.0f);
        pm1 = valid ? pm1 / wsum : 0.0f;
        pm2 = valid ? pm2 / wsum : 0.0f;
    }
    if (!valid) {
        // Any valid pixel of the 3 x 3 neighbourhood of the reprojected pixel.
        float n = 0.0f;
        const int x0 = max(0, px - 1), x1 = min(px + 1, static_cast<int>(p.width) - 1);
        const int y0 = max(0, py - 1), y1 = min(py + 1, static_cast<int>(p.height) - 1);
        for (int qx = x0; qx <= x1; ++qx) {
            for (int qy = y0; qy <= y1; ++qy) {
                const uint32_t q = pix(p, qx, qy);
                if (valid_reproject(p, g, b.geom[prev][q])) {
                    const SvgfData pd = b.data[prev_d][q];
                    prev_il = prev_il + illum(pd);
                    pm1 += pd.m1;
                    pm2 += pd.m2;
                    n += 1.0f;
                }
            }
        }
        if (n > 0.0f) {
            valid = true;
            prev_il = prev_il / n;
            pm1 /= n;
            pm2 /= n;
        }
    }
    float history;
    if (valid && inside) {
        history = b.history[prev][pix(p, px, py)];
    } else {
        history = 0.0f;
        prev_il = make3(0.0f);
        pm1 = pm2 = 0.0f;
    }
    history = fminf(static_cast<float>(sp.history_limit), valid ? history + 1.0f : 1.0f);
    b.history[cur][idx] = history;
    const float alpha = valid ? fmaxf(sp.alpha, 1.0f / history) : 1.0f;
    const float malpha = valid ? fmaxf(sp.moments_alpha, 1.0f / history) : 1.0f;
    float m1 = linear_srgb_to_y(il);
    float m2 = m1 * m1;
    m1 = lerp_to(malpha, pm1, m1);
    m2 = lerp_to(malpha, pm2, m2);
    const float var = fmaxf(0.0f, m2 - m1 * m1);
    il = make3(lerp_to(alpha, prev_il.x, il.x), lerp_to(alpha, prev_il.y, il.y), lerp_to(alpha, prev_il.z, il.z));
    d.ix = il.x;
    d.iy = il.y;
    d.iz = il.z;
    d.var = var;
    d.m1 = m1;
    d.m2 = m2;
    d.history = history;
    b.data[cur_d][idx] = d;
}

__global__ void __launch_bounds__(256) k_svgf_moments(const __grid_constant__ RtParams p,
                                                      const __grid_constant__ SvgfParams sp,
                                                      const __grid_constant__ SvgfBuffers b, uint32_t src,
                                                      uint32_t dst) {
    int x, y;
    if (!svgf_pixel(p, x, y)) return;
    const uint32_t idx = pix(p, x, y), cur = (p.frame + 1u) & 1u;
    const SvgfData *in = b.data[src];
    SvgfData c = in[idx];
    const SvgfGeom g = b.geom[cur][idx];
    const float history = b.history[cur][idx];
    if (history < 4.0f || g.linear_depth < 0.0f) {
        b.data[dst][idx] = c;
        return;
    }
    const float sigma_depth = fmaxf(g.depth_gradient, 1e-8f) * 3.0f;
    const float lum = linear_srgb_to_y(illum(c));
    const int r = sp.moments_radius;
    float wsum = 0.0f, s1 = 0.0f, s2 = 0.0f;
    f3 si = make3(0.0f);
    const int x0 = max(0, x - r), x1 = min(x + r, static_cast<int>(p.width) - 1);
    const int y0 = max(0, y - r), y1 = min(y + r, static_cast<int>(p.height) - 1);
    for (int qx = x0; qx <= x1; ++qx) {
        for (int qy = y0; qy <= y1; ++qy) {
            const uint32_t q = pix(p, qx, qy);
            const SvgfData qd = in[q];
            const SvgfGeom qg = b.geom[cur][q];
            const f3 qi = illum(qd);
            const float w = cal_weight(g.linear_depth, qg.linear_depth, sigma_depth, nrm(g), nrm(qg), sp.sigma_normal,
                                       lum, linear_srgb_to_y(qi), sp.sigma_rt);
            wsum += w;
            si = si + qi * w;
            s1 += qd.m1 * w;
            s2 += qd.m2 * w;
        }
    }
    wsum = fmaxf(wsum, 1e-6f);
    si = si / wsum;
    s1 /= wsum;
    s2 /= wsum;
    float var = s2 - s1 * s1;
    var *= 4.0f / history;
    c.ix = si.x;
    c.iy = si.y;
    c.iz = si.z;
    c.var = var;
    b.data[dst][idx] = c;
}

__global__ void __launch_bounds__(256) k_svgf_atrous(const __grid_constant__ RtParams p,
                                                     const __grid_constant__ SvgfParams sp,
                                                     const __grid_constant__ SvgfBuffers b, uint32_t src,
                                                     uint32_t dst, int step) {
    int x, y;
    if (!svgf_pixel(p, x, y)) return;
    const uint32_t idx = pix(p, x, y), cur = (p.frame + 1u) & 1u;
    const SvgfData *in = b.data[src];
    SvgfData c = in[idx];
    const float lum = linear_srgb_to_y(illum(c));
    // 3 x 3 Gaussian of the variance (atrous.cpp:17-31).
    float variance = 0.0f;
    {
        const float tab[2][2] = {{1.0f / 4, 1.0f / 8}, {1.0f / 8, 1.0f / 16}};
        const int x0 = max(0, x - 1), x1 = min(x + 1, static_cast<int>(p.width) - 1);
        const int y0 = max(0, y - 1), y1 = min(y + 1, static_cast<int>(p.height) - 1);
        for (int qx = x0; qx <= x1; ++qx)
            for (int qy = y0; qy <= y1; ++qy) variance += in[pix(p, qx, qy)].var * tab[abs(qx - x)][abs(qy - y)];
    }
    const SvgfGeom g = b.geom[cur][idx];
    if (g.linear_depth < 0.0f) {
        b.data[dst][idx] = c;
        return;
    }
    const float kw[3] = {1.0f, 2.0f / 3, 1.0f / 6};
    const float sigma_depth = fmaxf(g.depth_gradient, 1e-8f) * static_cast<float>(step);
    const float sigma_l = sp.sigma_rt * sqrtf(fmaxf(0.0f, 1e-10f + variance));
    float wsum = 1.0f;
    float4 sum = make_float4(c.ix, c.iy, c.iz, c.var);
    const int x0 = max(0, x - 2), x1 = min(x + 2, static_cast<int>(p.width) - 1);
    const int y0 = max(0, y - 2), y1 = min(y + 2, static_cast<int>(p.height) - 1);
    for (int nx = x0; nx <= x1; ++nx) {
        for (int ny = y0; ny <= y1; ++ny) {
            const int ox = x - nx, oy = y - ny;
            if (ox == 0 && oy == 0) continue;
            const int tx = x + ox * step, ty = y + oy * step;
            if (!in_screen(p, tx, ty)) continue;
            const uint32_t q = pix(p, tx, ty);
            const SvgfGeom qg = b.geom[cur][q];
            const SvgfData qd = in[q];
            const float len = sqrtf(static_cast<float>(ox * ox + oy * oy));
            const float w = cal_weight(g.linear_depth, qg.linear_depth, sigma_depth * len, nrm(g), nrm(qg),
                                       sp.sigma_normal, lum, linear_srgb_to_y(illum(qd)), sigma_l);
            const float iw = w * (kw[abs(ox)] * kw[abs(oy)]);
            wsum += iw;
            sum.x += iw * qd.ix;
            sum.y += iw * qd.iy;
            sum.z += iw * qd.iz;
            sum.w += (iw * iw) * qd.var;
        }
    }
    c.ix = sum.x / wsum;
    c.iy = sum.y / wsum;
    c.iz = sum.z / wsum;
    c.var = sum.w / (wsum * wsum);
    b.data[dst][idx] = c;
}

__global__ void __launch_bounds__(256) k_svgf_mod(const __grid_constant__ RtParams p,
                                                  const __grid_constant__ SvgfBuffers b, uint32_t src) {
    int x, y;
    if (!svgf_pixel(p, x, y)) return;
    const uint32_t idx = pix(p, x, y);
    const SvgfData d = b.data[src][idx];
    const float4 a = b.albedo[idx], e = b.emission[idx];
    b.out[idx] = make_float4(d.ix * a.x + e.x, d.iy * a.y + e.y, d.iz * a.z + e.z, 1.0f);
}

}  // namespace

cudaError_t upload_spectral_consts_svgf(const float *x, const float *y, const float *z, const float *d65,
                                       float y_integral) {
    return upload_spectral_consts_tu(x, y, z, d65, y_integral);
}

cudaError_t launch_svgf(const DeviceScene &s, const RtParams &p, const SvgfParams &sp, const SvgfBuffers &b,
                        uint32_t prev_d, uint32_t *final_d, cudaStream_t st, unsigned *launches) {
    const dim3 block(kSvgfTile, kSvgfTile);
    const dim3 grid((p.width + kSvgfTile - 1) / kSvgfTile, (p.height + kSvgfTile - 1) / kSvgfTile);
    const uint32_t cur_d = (prev_d + 1u) % 3u, tmp_d = (prev_d + 2u) % 3u;
    unsigned n = 0;
    k_svgf_geom<<<grid, block, 0, st>>>(s, p, b);
    k_svgf_gradient<<<grid, block, 0, st>>>(p, b);
    k_svgf_demod<<<grid, block, 0, st>>>(p, b, cur_d);
    n += 3;
    if (sp.reproject) {
        k_svgf_reproject<<<grid, block, 0, st>>>(p, sp, b, cur_d, prev_d);
        ++n;
    }
    uint32_t src = cur_d, dst = tmp_d;
    if (sp.filter_moments) {
        k_svgf_moments<<<grid, block, 0, st>>>(p, sp, b, src, dst);
        ++n;
        const uint32_t t = src;
        src = dst;
        dst = t;
    }
    for (uint32_t i = 0; i < sp.N; ++i) {
        k_svgf_atrous<<<grid, block, 0, st>>>(p, sp, b, src, dst, 1 << i);
        ++n;
        const uint32_t t = src;
        src = dst;
        dst = t;
    }
    k_svgf_mod<<<grid, block, 0, st>>>(p, b, src);
    ++n;
    *final_d = src;
    if (launches) *launches += n;
    return cudaGetLastError();
}

}  // namespace vs

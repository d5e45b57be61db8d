// Device side of the wavefront path tracer: the per-slot path state and the
// bodies of the bounce kernels (closest hit, shading, shadow rays), shared by
// the single-scene renderer (wavefront.cu) and the job server (server.cu).
// `Scenes` maps a slot's scene id to its DeviceScene (one scene for vs_render,
// a table of resident scenes for the server); the scene id of a slot lives in
// st.w, that of a shadow query in sh_c.w.
#pragma once

#include "vs_integrator.cuh"
#include "vs_wavefront.h"

namespace vs {
namespace wf {

__device__ __forceinline__ float comp(const float4 &v, int i) {
    return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w;
}

template <int N>
__device__ __forceinline__ float4 pack4(const float *a) {
    return make_float4(a[0], N > 1 ? a[1] : 0.0f, N > 2 ? a[2] : 0.0f, N > 3 ? a[3] : 0.0f);
}

template <int N>
__device__ __forceinline__ void store(const WfBuffers &b, uint32_t slot, const PathState<N> &ps, uint32_t scene) {
    b.o[slot] = make_float4(ps.ro.x, ps.ro.y, ps.ro.z, ps.scatter_pdf);
    b.d[slot] = make_float4(ps.rd.x, ps.rd.y, ps.rd.z, ps.eta_scale);
    b.tp[slot] = pack4<N>(ps.throughput.v);
    b.lam[slot] = pack4<N>(ps.wl.lambda);
    b.pdf[slot] = pack4<N>(ps.wl.pdf);
    b.L[slot] = make_float4(ps.L.x, ps.L.y, ps.L.z, 0.0f);
    b.st[slot] = make_uint4(static_cast<uint32_t>(ps.smp.state), static_cast<uint32_t>(ps.smp.state >> 32),
                            ps.bounce, scene);
}

// Loads slot `slot`; returns its scene id.
template <int N, class Scenes>
__device__ __forceinline__ uint32_t load(const Scenes &scenes, const WfBuffers &b, uint32_t slot, PathState<N> &ps) {
    const uint4 st = b.st[slot];
    const DeviceScene &s = scenes(st.w);
    const float4 o = b.o[slot], d = b.d[slot], tp = b.tp[slot], lam = b.lam[slot], pdf = b.pdf[slot],
                 L = b.L[slot];
    ps.ro = make3(o.x, o.y, o.z);
    ps.scatter_pdf = o.w;
    ps.rd = make3(d.x, d.y, d.z);
    ps.eta_scale = d.w;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        ps.throughput.v[i] = comp(tp, i);
        ps.wl.lambda[i] = comp(lam, i);
        ps.wl.pdf[i] = comp(pdf, i);
    }
    ps.L = make3(L.x, L.y, L.z);
    ps.smp.state = static_cast<uint64_t>(st.x) | (static_cast<uint64_t>(st.y) << 32);
    ps.smp.kind = s.ip.sampler;
    ps.smp.seed = s.ip.seed;
    ps.bounce = st.z;
    return st.w;
}

// Appends one entry per calling lane to a device queue: one atomicAdd per
// converged group of lanes, positions in lane order.
__device__ __forceinline__ uint32_t queue_push(uint32_t *counter) {
    const unsigned mask = __activemask();
    const int lane = static_cast<int>(threadIdx.x & 31u);
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, static_cast<uint32_t>(__popc(mask)));
    base = __shfl_sync(mask, base, leader);
    return base + static_cast<uint32_t>(__popc(mask & ((1u << lane) - 1u)));
}

// Appends the calling lane's slot to the queue of its shading class: one
// atomicAdd per class present among the converged lanes.
__device__ __forceinline__ uint32_t class_push(uint32_t *counts, uint32_t cls) {
    const unsigned active = __activemask();
    const unsigned group = __match_any_sync(active, cls);
    const int lane = static_cast<int>(threadIdx.x & 31u);
    const int leader = __ffs(group) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counts + cls, static_cast<uint32_t>(__popc(group)));
    base = __shfl_sync(active, base, leader);
    return base + static_cast<uint32_t>(__popc(group & ((1u << lane) - 1u)));
}

// Closest hits of queue `cur`, sorted into the shading-class queues.  Also
// clears the other path queue and the shadow queue for the shading pass that
// follows (their previous users have finished: kernels of one stream run in
// order; the class counters were cleared by the previous shadow pass or by
// the wave's generate kernel).
template <class Scenes>
__device__ __forceinline__ void extend(const Scenes &scenes, const WfBuffers &b, uint32_t cur) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        b.count[cur ^ 1u] = 0u;
        b.count[2] = 0u;
    }
    const uint32_t n = b.count[cur];
    const uint32_t *q = b.queue[cur];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t slot = q[i];
        const float4 o = b.o[slot], d = b.d[slot];
        const DeviceScene &s = scenes(b.st[slot].w);
        RayPre rp = precompute_ray(make3(o.x, o.y, o.z), make3(d.x, d.y, d.z));
        Hit h;
        float t;
        uint32_t cls = 0u;
        if (trace_closest(s, rp, 3.402823466e+38f, h, t)) {
            cls = 1u + s.materials[s.instances[h.inst_id].mat_id].type;
        } else {
            h = Hit{kInvalid, kInvalid, 0.0f, 0.0f};
        }
        b.hit[slot] = h;
        b.tq[static_cast<size_t>(cls) * b.capacity + class_push(b.count + 3, cls)] = slot;
    }
}

// The shading-class mask of path_shade for class C.
template <uint32_t C>
struct ClassMask {
    static constexpr uint32_t value = C == 0u ? 0u : (1u << (C - 1u));
};

// One bounce (path_shade) of every path of shading class C after its closest
// hit: survivors go to path queue cur ^ 1, next-event estimates to the shadow
// queue; a path that ends without a pending shadow query writes its radiance
// to radiance[base + slot].
template <int N, uint32_t C, class Scenes>
__device__ __forceinline__ void shade(const Scenes &scenes, const WfBuffers &b, uint32_t cur, uint64_t base,
                                      float4 *radiance) {
    const uint32_t n = b.count[3 + C];
    const uint32_t *q = b.tq + static_cast<size_t>(C) * b.capacity;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t slot = q[i];
        PathState<N> ps;
        const uint32_t scene = load<N>(scenes, b, slot, ps);
        const DeviceScene &s = scenes(scene);
        const Hit h = b.hit[slot];
        ShadowQuery sq;
        bool more = path_shade<N, false, ClassMask<C>::value>(s, ps, C != 0u, h, nullptr, sq);
        if (more) more = ++ps.bounce < s.ip.max_depth;
        if (more) {
            store<N>(b, slot, ps, scene);
            b.queue[cur ^ 1u][queue_push(&b.count[cur ^ 1u])] = slot;
        } else {
            b.L[slot] = make_float4(ps.L.x, ps.L.y, ps.L.z, 0.0f);
        }
        if (sq.valid) {
            const uint32_t k = queue_push(&b.count[2]);
            b.sh_o[k] = make_float4(sq.o.x, sq.o.y, sq.o.z, sq.tmax);
            b.sh_d[k] = make_float4(sq.d.x, sq.d.y, sq.d.z, __uint_as_float(slot | (more ? 0u : 0x80000000u)));
            b.sh_c[k] = make_float4(sq.c.x, sq.c.y, sq.c.z, __uint_as_float(scene));
        } else if (!more) {
            radiance[base + slot] = make_float4(ps.L.x, ps.L.y, ps.L.z, 1.0f);
        }
    }
}

// Shadow queries of the bounce: add the contribution when unoccluded; write
// the radiance of paths that ended at this bounce.  Clears the class
// counters for the next bounce (every shading pass of this one has finished).
template <class Scenes>
__device__ __forceinline__ void shadow(const Scenes &scenes, const WfBuffers &b, uint64_t base, float4 *radiance) {
    if (blockIdx.x == 0 && threadIdx.x < kWfClasses) b.count[3 + threadIdx.x] = 0u;
    const uint32_t n = b.count[2];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 o = b.sh_o[i], d = b.sh_d[i], c = b.sh_c[i];
        const uint32_t tag = __float_as_uint(d.w);
        const uint32_t slot = tag & 0x7fffffffu;
        const DeviceScene &s = scenes(__float_as_uint(c.w));
        const bool occluded = trace_any(s, precompute_ray(make3(o.x, o.y, o.z), make3(d.x, d.y, d.z)), o.w);
        float4 L = b.L[slot];
        if (!occluded) {
            f3 l = make3(L.x, L.y, L.z);
            l += make3(c.x, c.y, c.z);
            L = make_float4(l.x, l.y, l.z, 0.0f);
            b.L[slot] = L;
        }
        if (tag & 0x80000000u) radiance[base + slot] = make_float4(L.x, L.y, L.z, 1.0f);
    }
}

}  // namespace wf
}  // namespace vs

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
    b.L[slot] = make_float4(ps.L.x, ps.L.y, ps.L.z, ps.filter_w);
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
    ps.filter_w = L.w;
    ps.smp.state = static_cast<uint64_t>(st.x) | (static_cast<uint64_t>(st.y) << 32);
    ps.smp.kind = s.ip.sampler;
    ps.smp.seed = s.ip.seed;
    ps.bounce = st.z;
    return st.w;
}

// Camera paths of a wave: slot i holds path base + i of `cam` (frame-major
// over frames frame_begin, ...), queued for the first bounce; clears every
// counter of the wave.  A scene of max_depth 0 writes each path's (zero)
// radiance directly.
template <int N>
__device__ __forceinline__ void generate(const DeviceScene &s, const Camera &cam, const WfBuffers &b,
                                         uint32_t frame_begin, uint64_t base, uint32_t n, float4 *radiance) {
    const uint32_t npix = cam.width * cam.height;
    if (blockIdx.x == 0 && threadIdx.x < kWfCounters) b.count[threadIdx.x] = threadIdx.x == 0 ? n : 0u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint64_t p = base + i;
        const uint32_t frame = frame_begin + static_cast<uint32_t>(p / npix);
        const uint32_t pix = static_cast<uint32_t>(p % npix);
        PathState<N> ps;
        path_start<N>(s, cam, pix % cam.width, pix / cam.width, frame, ps);
        if (s.ip.max_depth == 0u) {
            radiance[p] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
            continue;
        }
        store<N>(b, i, ps, 0u);
        b.queue[0][i] = i;
    }
}

// The calling thread's lane in its warp (any block shape: a 16 x 8 block's
// warps hold two rows of threadIdx.x, so threadIdx.x % 32 is not the lane).
__device__ __forceinline__ int lane_id() {
    unsigned lane;
    asm volatile("mov.u32 %0, %%laneid;" : "=r"(lane));
    return static_cast<int>(lane);
}

// Appends one entry per calling lane to a device queue: one atomicAdd per
// converged group of lanes, positions in lane order.
__device__ __forceinline__ uint32_t queue_push(uint32_t *counter) {
    const unsigned mask = __activemask();
    const int lane = lane_id();
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
    const int lane = lane_id();
    const int leader = __ffs(group) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counts + cls, static_cast<uint32_t>(__popc(group)));
    base = __shfl_sync(active, base, leader);
    return base + static_cast<uint32_t>(__popc(group & ((1u << lane) - 1u)));
}

// Lanes of a warp that must be idle before the warp takes new rays.
#ifndef VS_REFILL_LANES
#define VS_REFILL_LANES 8
#endif

// Ray replacement for the traversal kernels: the idle lanes of a warp (at
// least VS_REFILL_LANES of them, or all) claim the next rays of a queue of `n`
// with one atomicAdd on `fetch`; returns the claimed index of the calling
// lane (>= n: none) and sets `drained` once the queue is exhausted.  Called by
// all 32 lanes.
__device__ __forceinline__ uint32_t refill(uint32_t *fetch, uint32_t n, bool active, bool &drained) {
    const unsigned idle = __ballot_sync(0xffffffffu, !active);
    const uint32_t k = static_cast<uint32_t>(__popc(idle));
    if (k < VS_REFILL_LANES && k != 32u) return n;
    const int lane = lane_id();
    const int leader = __ffs(idle) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(fetch, k);
    base = __shfl_sync(0xffffffffu, base, leader);
    if (base + k >= n) drained = true;
    if (active) return n;
    return base + static_cast<uint32_t>(__popc(idle & ((1u << lane) - 1u)));
}

// Closest hits of queue `cur`, sorted into the shading-class queues.  Each
// warp keeps 32 rays in flight and refills finished lanes from the queue.
// Also clears the other path queue, the shadow queue and the shadow fetch
// counter for the passes that follow (their previous users have finished:
// kernels of one stream run in order; the class counters and this kernel's
// fetch counter were cleared by the previous shadow pass or by the wave's
// generate kernel).
template <int Levels, class Scenes>
__device__ __forceinline__ void extend(const Scenes &scenes, const WfBuffers &b, uint32_t cur) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        b.count[cur ^ 1u] = 0u;
        b.count[2] = 0u;
        b.count[kWfFetchShadow] = 0u;
    }
    const uint32_t n = b.count[cur];
    const uint32_t *q = b.queue[cur];
    uint2 stack[kStackSize];
    bool active = false, drained = false;
    uint32_t slot = 0;
    const DeviceScene *s = nullptr;
    RayPre r;
    TravState t;
    for (;;) {
        if (!drained) {
            const uint32_t i = refill(b.count + kWfFetchExtend, n, active, drained);
            if (i < n) {
                slot = q[i];
                const float4 o = b.o[slot], d = b.d[slot];
                s = &scenes(b.st[slot].w);
                r = precompute_ray(make3(o.x, o.y, o.z), make3(d.x, d.y, d.z));
                trav_init(t, r, 3.402823466e+38f);
                active = true;
            }
        }
        if (!__any_sync(0xffffffffu, active)) break;
        if (active && closest_step<Levels>(*s, r, t, stack)) {
            const Hit h = trav_hit(*s, t);
            const uint32_t cls = h.inst_id == kInvalid ? 0u : 1u + s->materials[s->instances[h.inst_id].mat_id].type;
            b.hit[slot] = h;
            b.tq[static_cast<size_t>(cls) * b.capacity + class_push(b.count + 3, cls)] = slot;
            active = false;
        }
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
            b.L[slot] = make_float4(ps.L.x, ps.L.y, ps.L.z, ps.filter_w);
        }
        if (sq.valid) {
            const uint32_t k = queue_push(&b.count[2]);
            b.sh_o[k] = make_float4(sq.o.x, sq.o.y, sq.o.z, sq.tmax);
            b.sh_d[k] = make_float4(sq.d.x, sq.d.y, sq.d.z, __uint_as_float(slot | (more ? 0u : 0x80000000u)));
            b.sh_c[k] = make_float4(sq.c.x, sq.c.y, sq.c.z, __uint_as_float(scene));
        } else if (!more) {
            const f3 Lw = ps.L * ps.filter_w;
            radiance[base + slot] = make_float4(Lw.x, Lw.y, Lw.z, 1.0f);
        }
    }
}

// Shadow queries of the bounce (with ray replacement, as extend): add the
// contribution when unoccluded; write the radiance of paths that ended at
// this bounce.  Clears the class counters and the extend fetch counter for
// the next bounce (every shading pass of this one has finished).
template <int Levels, class Scenes>
__device__ __forceinline__ void shadow(const Scenes &scenes, const WfBuffers &b, uint64_t base, float4 *radiance) {
    if (blockIdx.x == 0 && threadIdx.x < kWfClasses) b.count[3 + threadIdx.x] = 0u;
    if (blockIdx.x == 0 && threadIdx.x == 32) b.count[kWfFetchExtend] = 0u;
    const uint32_t n = b.count[2];
    uint2 stack[kStackSize];
    bool active = false, drained = false;
    uint32_t i = 0;
    const DeviceScene *s = nullptr;
    RayPre r;
    TravState t;
    for (;;) {
        if (!drained) {
            const uint32_t k = refill(b.count + kWfFetchShadow, n, active, drained);
            if (k < n) {
                i = b.sh_perm ? b.sh_perm[k] : k;
                const float4 o = b.sh_o[i], d = b.sh_d[i];
                s = &scenes(__float_as_uint(b.sh_c[i].w));
                r = precompute_ray(make3(o.x, o.y, o.z), make3(d.x, d.y, d.z));
                trav_init(t, r, o.w);
                active = true;
            }
        }
        if (!__any_sync(0xffffffffu, active)) break;
        bool occluded = false;
        if (active && any_step<Levels>(*s, r, t, stack, occluded)) {
            const uint32_t tag = __float_as_uint(b.sh_d[i].w);
            const uint32_t slot = tag & 0x7fffffffu;
            float4 L = b.L[slot];
            if (!occluded) {
                const float4 c = b.sh_c[i];
                f3 l = make3(L.x, L.y, L.z);
                l += make3(c.x, c.y, c.z);
                L = make_float4(l.x, l.y, l.z, L.w);
                b.L[slot] = L;
            }
            if (tag & 0x80000000u) {
                const f3 Lw = make3(L.x, L.y, L.z) * L.w;
                radiance[base + slot] = make_float4(Lw.x, Lw.y, Lw.z, 1.0f);
            }
            active = false;
        }
    }
}

}  // namespace wf
}  // namespace vs

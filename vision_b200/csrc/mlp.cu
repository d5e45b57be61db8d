// Radiance-cache MLP on the tcgen05 tensor cores (sm_100a).
//
// Network: 64 BF16 inputs -> 4 hidden layers of 64 (ReLU) -> 3 outputs, no
// biases.  Every layer is a tcgen05.mma.kind::f16 with BF16 operands in
// shared memory and the FP32 accumulator in tensor memory:
//   inference  (k_mlp_infer): one CTA per SM holding the forward weights once
//     and running kInferGroups independent 4-warp pipelines, each with its
//     own 64 tensor-memory columns and two tile buffers; while a pipeline runs
//     the five layers of one 128-row tile, the TMA engine loads its next tile
//     into the other buffer (128-byte swizzle, rows past n zero-filled).
//     M=128 x N=64 (N=16 for the padded output layer), K=64 as four K=16
//     steps.  Thread t of a pipeline owns tile row t: after each layer it
//     reads its accumulator row with tcgen05.ld (32x32b), applies ReLU, rounds
//     to BF16 and writes the next layer's operand row in the no-swizzle
//     layout, over the consumed feature tile.
//   training   (k_mlp_train): the same forward pass keeping every layer's
//     BF16 input; the relative-L2 loss gradient; the backward data products
//     dX = dZ W^T (M=128) masked by ReLU'; and the weight gradients
//     dW = X^T dZ as M=64 MMAs whose operands are the same shared-memory
//     tiles read MN-major, accumulated in tensor memory over all tiles of the
//     CTA and added to the global FP32 gradient once per CTA.
//   k_mlp_adam updates the FP32 master weights; k_mlp_pack rewrites the BF16
//   operand images (forward: W as [out][in]; backward: W as [in][out]).
// Shared-memory operands use the canonical no-swizzle layout: 8-row x 16-byte
// core matrices, rows of a core matrix 16 B apart; for a K-major operand with
// R rows, core matrices along M/N are 128 B apart (SBO) and along K R*16 B
// apart (LBO); the same 128-row activation tile read MN-major has LBO = 128 B
// (next 8 batch rows) and SBO = 2048 B (next 8 features).
// Every wait on the MMA-completion mbarrier is bounded; on timeout the kernel
// records the error, skips the rest of its work, frees its tensor memory and
// returns.
#include "vs_mlp.h"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cstdint>

namespace vs {

namespace {

constexpr int kTile = 128;
constexpr uint32_t kTileBytes = kTile * 64 * 2;       // 16 KB activation tile
constexpr uint32_t kPackFwdBytes = kMlpPackFwd * 2;   // 34,816 B
constexpr long long kWaitCycles = 4000000000ll;       // ~2 s at 1.9 GHz

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, no swizzle, Blackwell version field.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor: BF16 x BF16 -> FP32, dense.
__host__ __device__ constexpr uint32_t idesc(int M, int N, int a_mn, int b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(a_mn) << 15) |
           (static_cast<uint32_t>(b_mn) << 16) | (static_cast<uint32_t>(N >> 3) << 17) |
           (static_cast<uint32_t>(M >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t id, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(id), "r"(accumulate));
}

__device__ __forceinline__ void commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

// Bounded wait on the phase parity of an mbarrier.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    long long t0 = clock64();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > kWaitCycles) return false;
    }
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Issues the loads of 64 accumulator columns (four 32x32b.x16) and waits for
// them once.
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float *v) {
    uint32_t r[64];
#pragma unroll
    for (int q = 0; q < 4; ++q)
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(r[16 * q + 0]), "=r"(r[16 * q + 1]), "=r"(r[16 * q + 2]), "=r"(r[16 * q + 3]),
              "=r"(r[16 * q + 4]), "=r"(r[16 * q + 5]), "=r"(r[16 * q + 6]), "=r"(r[16 * q + 7]),
              "=r"(r[16 * q + 8]), "=r"(r[16 * q + 9]), "=r"(r[16 * q + 10]), "=r"(r[16 * q + 11]),
              "=r"(r[16 * q + 12]), "=r"(r[16 * q + 13]), "=r"(r[16 * q + 14]), "=r"(r[16 * q + 15])
            : "r"(taddr + 16u * q));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 64; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack2(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t *>(&h);
}
__device__ __forceinline__ float bf_lo(uint32_t u) { return __uint_as_float(u << 16); }
__device__ __forceinline__ float bf_hi(uint32_t u) { return __uint_as_float(u & 0xFFFF0000u); }

// Byte offset of 16-byte chunk kc (elements 8kc..8kc+7) of row r in a
// 128-row K-major tile.
__device__ __forceinline__ uint32_t tile_chunk(uint32_t r, uint32_t kc) {
    return kc * 2048u + (r >> 3) * 128u + (r & 7u) * 16u;
}

// Reads the 64 accumulator columns [col, col + 64) of this thread's row.
__device__ __forceinline__ void ld_row64(uint32_t tmem, uint32_t col, float *v) {
    uint32_t lane = (threadIdx.x & ~31u) << 16;
#pragma unroll
    for (int q = 0; q < 4; ++q) tmem_ld16(tmem + lane + col + 16u * q, v + 16 * q);
}

// Writes 64 values as BF16 into row r of a 128-row tile.
__device__ __forceinline__ void st_row64(uint8_t *tile, uint32_t r, const float *v) {
#pragma unroll
    for (int kc = 0; kc < 8; ++kc) {
        uint4 u = make_uint4(pack2(v[8 * kc], v[8 * kc + 1]), pack2(v[8 * kc + 2], v[8 * kc + 3]),
                             pack2(v[8 * kc + 4], v[8 * kc + 5]), pack2(v[8 * kc + 6], v[8 * kc + 7]));
        *reinterpret_cast<uint4 *>(tile + tile_chunk(r, kc)) = u;
    }
}

__device__ __forceinline__ void ld_row64_bf(const uint8_t *tile, uint32_t r, float *v) {
#pragma unroll
    for (int kc = 0; kc < 8; ++kc) {
        uint4 u = *reinterpret_cast<const uint4 *>(tile + tile_chunk(r, kc));
        v[8 * kc + 0] = bf_lo(u.x);
        v[8 * kc + 1] = bf_hi(u.x);
        v[8 * kc + 2] = bf_lo(u.y);
        v[8 * kc + 3] = bf_hi(u.y);
        v[8 * kc + 4] = bf_lo(u.z);
        v[8 * kc + 5] = bf_hi(u.z);
        v[8 * kc + 6] = bf_lo(u.w);
        v[8 * kc + 7] = bf_hi(u.w);
    }
}

// Loads row `row` of the global feature matrix (zeros past n) into tile row r.
__device__ __forceinline__ void load_features(uint8_t *tile, uint32_t r, const uint16_t *feat, uint64_t row,
                                              uint32_t n) {
    const uint4 *src = reinterpret_cast<const uint4 *>(feat + row * 64u);
#pragma unroll
    for (int kc = 0; kc < 8; ++kc) {
        uint4 u = row < n ? __ldg(src + kc) : make_uint4(0, 0, 0, 0);
        *reinterpret_cast<uint4 *>(tile + tile_chunk(r, kc)) = u;
    }
}

__device__ __forceinline__ void copy_to_smem(uint8_t *dst, const uint4 *src, uint32_t bytes) {
    for (uint32_t i = threadIdx.x; i < bytes / 16u; i += blockDim.x) reinterpret_cast<uint4 *>(dst)[i] = __ldg(src + i);
}

// Forward weight descriptors: layer l < 4 is [64 out][64 in] (LBO 1024), the
// output layer [16 out][64 in] (LBO 256); K step s advances 2 K-chunks.
__device__ __forceinline__ uint64_t w_fwd_desc(uint32_t wbase, int l, int s) {
    if (l < 4) return sdesc(wbase + l * 8192u + s * 2048u, 1024u, 128u);
    return sdesc(wbase + 4u * 8192u + s * 512u, 256u, 128u);
}
// Backward weight descriptors: layer l < 4 is [64 in][64 out] (LBO 1024);
// the output layer [64 in][16 out], one K step.
__device__ __forceinline__ uint64_t w_bwd_desc(uint32_t wbase, int l, int s) {
    if (l < 4) return sdesc(wbase + l * 8192u + s * 2048u, 1024u, 128u);
    return sdesc(wbase + 4u * 8192u, 1024u, 128u);
}
// A 128-row activation tile as a K-major operand, K step s.
__device__ __forceinline__ uint64_t tile_kdesc(uint32_t base, int s) { return sdesc(base + s * 4096u, 2048u, 128u); }
// The same tile read MN-major (features along M/N, batch rows along K), K step s.
__device__ __forceinline__ uint64_t tile_mndesc(uint32_t base, int s) { return sdesc(base + s * 256u, 128u, 2048u); }

struct TmemSlot {
    uint32_t addr;
};

__device__ __forceinline__ void tmem_alloc(uint32_t slot_saddr, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot_saddr), "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

// A 128-row feature tile written by TMA with the 128-byte swizzle (row r at
// 128 r, its 16-byte chunk c at (c ^ (r & 7)) * 16, 1024-byte aligned) as a
// K-major operand, K step s: SBO 1024 B between 8-row groups, the K=16 step
// 32 B further inside the swizzle atom, layout type SWIZZLE_128B.
__device__ __forceinline__ uint64_t tile_sw128_desc(uint32_t base, int s) {
    return sdesc(base + s * 32u, 16u, 1024u) | (2ull << 61);
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

// One 2D tile of the feature tensor map into shared memory (no multicast),
// completing on `mbar` with its byte count.
__device__ __forceinline__ void tma_load_tile(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t mbar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            dst),
        "l"(map), "r"(x), "r"(y), "r"(mbar)
        : "memory");
}

// Named barrier over the 128 threads of pipeline g (barrier 1 + g), returning
// whether every thread passed true.
__device__ __forceinline__ bool group_sync_and(uint32_t g, bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.b32 p, %1, 0;\n\tbarrier.cta.red.and.pred q, %2, 128, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"(static_cast<uint32_t>(v)), "r"(1u + g)
        : "memory");
    return r != 0u;
}

constexpr uint32_t kInferGroups = 5;
constexpr uint32_t kInferThreads = 128u * kInferGroups;
constexpr uint32_t kInferBars = 3u * kInferGroups;  // per pipeline: two tile loads, one MMA
constexpr uint32_t kInferSmem = 1024u + kPackFwdBytes + kInferGroups * 2u * kTileBytes + 8u * kInferBars + 16u;
static_assert(kInferSmem <= 232448u, "inference shared memory above the per-CTA limit");

__global__ void __launch_bounds__(kInferThreads, 1) k_mlp_infer(const __grid_constant__ CUtensorMap fmap, uint32_t n,
                                                                const uint4 *__restrict__ wpack,
                                                                float4 *__restrict__ out, int *err) {
    extern __shared__ uint8_t smem_raw[];
    // 1024-byte alignment for the swizzled TMA destinations.
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t *smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    uint8_t *w = smem;
    uint8_t *bufs = smem + kPackFwdBytes;
    uint64_t *bars = reinterpret_cast<uint64_t *>(bufs + kInferGroups * 2u * kTileBytes);
    uint32_t *slot = reinterpret_cast<uint32_t *>(bars + kInferBars);
    const uint32_t tid = threadIdx.x, g = tid >> 7, gt = tid & 127u;
    if (tid < 32) tmem_alloc(smem_u32(slot), 512);
    if (tid == 0) {
        for (uint32_t i = 0; i < kInferBars; ++i) mbar_init(smem_u32(bars + i), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    copy_to_smem(w, wpack, kPackFwdBytes);
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    // Pipeline g: accumulator columns [64 g, 64 g + 64), tile buffers
    // buf0 + {0, kTileBytes}, barriers load[0], load[1], mma.
    const uint32_t tmem = *slot + 64u * g;
    const uint32_t lane = (gt & ~31u) << 16;
    const uint32_t wbase = smem_u32(w);
    uint8_t *tile0 = bufs + g * 2u * kTileBytes;
    const uint32_t buf0 = smem_u32(tile0);
    const uint32_t mb_load = smem_u32(bars + 3u * g), mb_mma = mb_load + 16u;
    const uint32_t tiles = (n + kTile - 1) / kTile;
    const uint32_t stride = gridDim.x * kInferGroups;
    uint32_t tt = blockIdx.x * kInferGroups + g;
    uint32_t ph_load = 0u, ph_mma = 0u;  // parity bits (bit b: buffer b)
    bool pending[2] = {false, false};
    if (gt == 0 && tt < tiles) {
        mbar_expect_tx(mb_load, kTileBytes);
        tma_load_tile(buf0, &fmap, 0, static_cast<int>(tt * kTile), mb_load);
    }
    pending[0] = tt < tiles;
    bool ok = true;
    for (uint32_t k = 0; tt < tiles && ok; tt += stride, ++k) {
        const uint32_t cur = k & 1u, nxt = cur ^ 1u;
        const uint32_t buf = buf0 + cur * kTileBytes;
        uint8_t *tile = tile0 + cur * kTileBytes;
        // The other buffer held the previous tile, whose last MMA has
        // completed: load the next tile into it now.
        if (tt + stride < tiles) {
            if (gt == 0) {
                mbar_expect_tx(mb_load + 8u * nxt, kTileBytes);
                tma_load_tile(buf0 + nxt * kTileBytes, &fmap, 0, static_cast<int>((tt + stride) * kTile),
                              mb_load + 8u * nxt);
            }
            pending[nxt] = true;
        }
        bool done = mbar_wait(mb_load + 8u * cur, (ph_load >> cur) & 1u);
        ph_load ^= 1u << cur;
        pending[cur] = !done;
        ok = group_sync_and(g, done);
        if (!ok) break;
        const uint64_t row = static_cast<uint64_t>(tt) * kTile + gt;
        for (int l = 0; l < 5; ++l) {
            if (gt == 0) {
                const uint32_t id = l < 4 ? idesc(128, 64, 0, 0) : idesc(128, 16, 0, 0);
#pragma unroll
                for (int s = 0; s < 4; ++s)
                    mma(tmem, l == 0 ? tile_sw128_desc(buf, s) : tile_kdesc(buf, s), w_fwd_desc(wbase, l, s), id,
                        s > 0);
                commit(mb_mma);
            }
            done = mbar_wait(mb_mma, ph_mma);
            ph_mma ^= 1u;
            fence_after();
            // The epilogue of a thread whose wait ran out is skipped; the
            // barrier that follows makes the pipeline agree to stop.
            if (done && l < 4) {
                float v[64];
                tmem_ld64(tmem + lane, v);
#pragma unroll
                for (int i = 0; i < 64; ++i) v[i] = fmaxf(v[i], 0.0f);
                st_row64(tile, gt, v);
                fence_async_smem();
            } else if (done) {
                float v[16];
                tmem_ld16(tmem + lane, v);
                if (row < n) out[row] = make_float4(v[0], v[1], v[2], 0.0f);
            }
            fence_before();
            ok = group_sync_and(g, done);
            fence_after();
            if (!ok) break;
        }
    }
    // A pipeline that stopped early waits (bounded) for the loads it still
    // has in flight before the CTA releases its shared memory.
    for (uint32_t b = 0; b < 2; ++b)
        if (pending[b]) (void)mbar_wait(mb_load + 8u * b, (ph_load >> b) & 1u);
    if (!ok && gt == 0) atomicExch(err, 1);
    fence_before();
    __syncthreads();
    fence_after();
    if (tid < 32) tmem_free(*slot, 512);
}

// Training shared memory: forward and backward weight images, the input tile
// X0, hidden activations H1..H4, the gradient tile G, the output-gradient
// tile DO (128 x 16), barrier and slots.
constexpr uint32_t kOffWf = 0;
constexpr uint32_t kOffWb = kPackFwdBytes;
constexpr uint32_t kOffX = 2 * kPackFwdBytes;
constexpr uint32_t kOffG = kOffX + 5 * kTileBytes;
constexpr uint32_t kOffDO = kOffG + kTileBytes;
constexpr uint32_t kOffBar = kOffDO + 4096;
constexpr uint32_t kTrainSmem = kOffBar + 64;
constexpr uint32_t kTrainCols = 512;   // D: 0..63; dW0..dW3: 64 + 64 l; dW4: 320..335

__global__ void __launch_bounds__(128, 1) k_mlp_train(const uint16_t *__restrict__ feat,
                                                      const float4 *__restrict__ target, uint32_t n,
                                                      const uint4 *__restrict__ wpack, float loss_scale,
                                                      float *__restrict__ grad, double *loss, int *err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *act[5];
#pragma unroll
    for (int l = 0; l < 5; ++l) act[l] = smem + kOffX + l * kTileBytes;  // X0, H1, H2, H3, H4
    uint8_t *G = smem + kOffG;
    uint8_t *DO = smem + kOffDO;
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + kOffBar);
    uint32_t *slot = reinterpret_cast<uint32_t *>(smem + kOffBar + 8);
    float *red = reinterpret_cast<float *>(smem + kOffBar + 16);
    const uint32_t tid = threadIdx.x;
    const uint32_t mbar_s = smem_u32(mbar);
    if (tid < 32) tmem_alloc(smem_u32(slot), kTrainCols);
    if (tid == 0) {
        mbar_init(mbar_s, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    copy_to_smem(smem + kOffWf, wpack, 2 * kPackFwdBytes);
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *slot;
    const uint32_t wf = smem_u32(smem + kOffWf), wb = smem_u32(smem + kOffWb);
    uint32_t abase[5];
#pragma unroll
    for (int l = 0; l < 5; ++l) abase[l] = smem_u32(act[l]);
    const uint32_t gbase = smem_u32(G), dobase = smem_u32(DO);
    const uint32_t lane = (tid & ~31u) << 16;
    uint32_t phase = 0;
    bool ok = true;
    bool first = true;
    float loss_acc = 0.0f;
    const uint32_t tiles = (n + kTile - 1) / kTile;
    auto sync_all = [&]() {
        fence_before();
        __syncthreads();
        fence_after();
    };
    auto wait_mma = [&]() {
        const bool done = ok && mbar_wait(mbar_s, phase);
        phase ^= 1u;
        ok = __syncthreads_and(done) != 0;
        fence_after();
    };
    for (uint32_t tt = blockIdx.x; tt < tiles && ok; tt += gridDim.x) {
        const uint64_t row = static_cast<uint64_t>(tt) * kTile + tid;
        const bool valid = row < n;
        load_features(act[0], tid, feat, row, n);
        fence_async_smem();
        sync_all();
        // Forward: layers 0..3 into H1..H4, output layer into registers.
        float y[3] = {0.0f, 0.0f, 0.0f};
        for (int l = 0; l < 5 && ok; ++l) {
            if (tid == 0) {
                const uint32_t id = l < 4 ? idesc(128, 64, 0, 0) : idesc(128, 16, 0, 0);
#pragma unroll
                for (int s = 0; s < 4; ++s) mma(tmem, tile_kdesc(abase[l], s), w_fwd_desc(wf, l, s), id, s > 0);
                commit(mbar_s);
            }
            wait_mma();
            if (!ok) break;
            if (l < 4) {
                float v[64];
                ld_row64(tmem, 0, v);
#pragma unroll
                for (int i = 0; i < 64; ++i) v[i] = fmaxf(v[i], 0.0f);
                st_row64(act[l + 1], tid, v);
                fence_async_smem();
            } else {
                float v[16];
                tmem_ld16(tmem + lane, v);
                y[0] = v[0];
                y[1] = v[1];
                y[2] = v[2];
            }
            sync_all();
        }
        if (!ok) break;
        // Relative L2 loss (denominator without gradient) and its gradient.
        float go[3] = {0.0f, 0.0f, 0.0f};
        if (valid) {
            float4 t = target[row];
            const float tv[3] = {t.x, t.y, t.z};
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                float e = y[c] - tv[c];
                float den = y[c] * y[c] + 0.01f;
                loss_acc += e * e / den;
                go[c] = 2.0f * e / den * loss_scale;
            }
        }
        {
            uint4 u0 = make_uint4(pack2(go[0], go[1]), pack2(go[2], 0.0f), 0u, 0u);
            *reinterpret_cast<uint4 *>(DO + tile_chunk(tid, 0)) = u0;
            *reinterpret_cast<uint4 *>(DO + tile_chunk(tid, 1)) = make_uint4(0u, 0u, 0u, 0u);
        }
        fence_async_smem();
        sync_all();
        // Backward, layer by layer: dW_l += X_l^T dZ_l, dX_l = dZ_l W_l^T, dZ_{l-1} = dX_l * (X_l > 0).
        for (int l = 4; l >= 0 && ok; --l) {
            if (tid == 0) {
                const uint32_t dz = l == 4 ? dobase : gbase;
                const uint32_t dw_col = l == 4 ? 320u : 64u + 64u * l;
                const uint32_t id_w = l == 4 ? idesc(64, 16, 1, 1) : idesc(64, 64, 1, 1);
#pragma unroll
                for (int s = 0; s < 8; ++s)
                    mma(tmem + dw_col, tile_mndesc(abase[l], s), tile_mndesc(dz, s), id_w, (!first || s > 0) ? 1u : 0u);
                if (l > 0) {
                    if (l == 4) {
                        mma(tmem, sdesc(dobase, 2048u, 128u), w_bwd_desc(wb, 4, 0), idesc(128, 64, 0, 0), 0u);
                    } else {
#pragma unroll
                        for (int s = 0; s < 4; ++s)
                            mma(tmem, tile_kdesc(gbase, s), w_bwd_desc(wb, l, s), idesc(128, 64, 0, 0), s > 0);
                    }
                }
                commit(mbar_s);
            }
            wait_mma();
            if (!ok) break;
            if (l > 0) {
                float v[64], h[64];
                ld_row64(tmem, 0, v);
                ld_row64_bf(act[l], tid, h);
#pragma unroll
                for (int i = 0; i < 64; ++i) v[i] = h[i] > 0.0f ? v[i] : 0.0f;
                st_row64(G, tid, v);
                fence_async_smem();
            }
            sync_all();
        }
        first = false;
    }
    // Weight gradients: rows of an M=64 accumulator live in lanes 16w..16w+15
    // of warp w's quarter (row 16w + t in lane 32w + t, t < 16).
    if (ok && !first) {
        const uint32_t r = 16u * (tid >> 5) + (tid & 31u);
        const bool holder = (tid & 31u) < 16u;
        for (int l = 0; l < 4; ++l) {
            float v[64];
            ld_row64(tmem, 64u + 64u * l, v);
            if (holder)
                for (int c = 0; c < 64; ++c) atomicAdd(grad + l * 4096 + r * 64 + c, v[c]);
        }
        float v[16];
        tmem_ld16(tmem + lane + 320u, v);
        if (holder)
            for (int c = 0; c < 3; ++c) atomicAdd(grad + 4 * 4096 + r * 3 + c, v[c]);
    }
    // Loss reduction.
    for (int o = 16; o > 0; o >>= 1) loss_acc += __shfl_xor_sync(0xffffffffu, loss_acc, o);
    if ((tid & 31u) == 0) red[tid >> 5] = loss_acc;
    fence_before();
    __syncthreads();
    fence_after();
    if (tid == 0) {
        double s = static_cast<double>(red[0]) + red[1] + red[2] + red[3];
        atomicAdd(loss, s * loss_scale);
        if (!ok) atomicExch(err, 1);
    }
    if (tid < 32) tmem_free(tmem, kTrainCols);
}

// Packed-image offsets (elements) of weight (l, in, out).
__device__ __forceinline__ uint32_t off_fwd(int l, uint32_t in, uint32_t out) {
    if (l < 4) return l * 4096u + (in >> 3) * 512u + (out >> 3) * 64u + (out & 7u) * 8u + (in & 7u);
    return 4u * 4096u + (in >> 3) * 128u + (out & 7u) * 8u + (in & 7u);
}
__device__ __forceinline__ uint32_t off_bwd(int l, uint32_t in, uint32_t out) {
    const uint32_t b = static_cast<uint32_t>(kMlpPackFwd);
    if (l < 4) return b + l * 4096u + (out >> 3) * 512u + (in >> 3) * 64u + (in & 7u) * 8u + (out & 7u);
    return b + 4u * 4096u + (in >> 3) * 64u + (in & 7u) * 8u + (out & 7u);
}

__device__ __forceinline__ void param_coords(uint32_t i, int &l, uint32_t &in, uint32_t &out) {
    if (i < 4u * 4096u) {
        l = static_cast<int>(i / 4096u);
        in = (i % 4096u) / 64u;
        out = i % 64u;
    } else {
        l = 4;
        in = (i - 4u * 4096u) / 3u;
        out = (i - 4u * 4096u) % 3u;
    }
}

__global__ void k_mlp_pack(const float *w, uint16_t *pack) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= static_cast<uint32_t>(kMlpParams)) return;
    int l;
    uint32_t in, out;
    param_coords(i, l, in, out);
    __nv_bfloat16 h = __float2bfloat16_rn(w[i]);
    uint16_t u = *reinterpret_cast<uint16_t *>(&h);
    pack[off_fwd(l, in, out)] = u;
    pack[off_bwd(l, in, out)] = u;
}

__global__ void k_mlp_adam(float *w, float *m, float *v, const float *g, MlpAdam a, uint16_t *pack) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= static_cast<uint32_t>(kMlpParams)) return;
    float gi = g[i];
    float mi = a.beta1 * m[i] + (1.0f - a.beta1) * gi;
    float vi = a.beta2 * v[i] + (1.0f - a.beta2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    float mh = mi / (1.0f - powf(a.beta1, static_cast<float>(a.step)));
    float vh = vi / (1.0f - powf(a.beta2, static_cast<float>(a.step)));
    float wi = w[i] - a.lr * mh / (sqrtf(vh) + a.eps);
    w[i] = wi;
    int l;
    uint32_t in, out;
    param_coords(i, l, in, out);
    __nv_bfloat16 h = __float2bfloat16_rn(wi);
    uint16_t u = *reinterpret_cast<uint16_t *>(&h);
    pack[off_fwd(l, in, out)] = u;
    pack[off_bwd(l, in, out)] = u;
}

int g_sm_count = 0;

}  // namespace

cudaError_t mlp_pack(const MlpState &s, cudaStream_t st) {
    k_mlp_pack<<<(kMlpParams + 255) / 256, 256, 0, st>>>(s.w, s.pack);
    return cudaGetLastError();
}

static cudaError_t sm_count(int &n) {
    if (g_sm_count == 0) {
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
    }
    n = g_sm_count;
    return cudaSuccess;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library).
static PFN_cuTensorMapEncodeTiled_v12000 g_encode_tiled = nullptr;

static cudaError_t encode_fn() {
    if (g_encode_tiled) return cudaSuccess;
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q);
    if (e != cudaSuccess) return e;
    if (q != cudaDriverEntryPointSuccess || !fn) return cudaErrorSymbolNotFound;
    g_encode_tiled = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    return cudaSuccess;
}

// The feature matrix (n rows of 64 BF16, 128-byte rows, 16-byte aligned) as a
// TMA tensor map with 128-row x 64-column boxes and the 128-byte swizzle.
static cudaError_t feature_map(const uint16_t *feat, uint32_t n, CUtensorMap *map) {
    cudaError_t e = encode_fn();
    if (e != cudaSuccess) return e;
    if (reinterpret_cast<uintptr_t>(feat) & 15u) return cudaErrorMisalignedAddress;
    cuuint64_t dims[2] = {64u, n};
    cuuint64_t strides[1] = {128u};
    cuuint32_t box[2] = {64u, static_cast<cuuint32_t>(kTile)};
    cuuint32_t elem[2] = {1u, 1u};
    CUresult r = g_encode_tiled(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<uint16_t *>(feat), dims, strides,
                                box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t mlp_infer(const MlpState &s, const uint16_t *feat, uint32_t n, float4 *out, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, kInferSmem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    CUtensorMap map;
    cudaError_t e = feature_map(feat, n, &map);
    if (e != cudaSuccess) return e;
    int sms = 0;
    e = sm_count(sms);
    if (e != cudaSuccess) return e;
    const uint32_t tiles = (n + kTile - 1) / kTile;
    uint32_t grid = static_cast<uint32_t>(sms);
    const uint32_t need = (tiles + kInferGroups - 1) / kInferGroups;
    if (grid > need) grid = need;
    k_mlp_infer<<<grid, kInferThreads, kInferSmem, st>>>(map, n, reinterpret_cast<const uint4 *>(s.pack), out, s.err);
    return cudaGetLastError();
}

cudaError_t mlp_train_step(const MlpState &s, const uint16_t *feat, const float4 *target, uint32_t n, MlpAdam adam,
                           bool update, cudaStream_t st) {
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrainSmem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    cudaError_t e = cudaMemsetAsync(s.grad, 0, sizeof(float) * kMlpParams, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(s.loss, 0, sizeof(double), st);
    if (e != cudaSuccess) return e;
    if (n > 0) {
        int sms = 0;
        e = sm_count(sms);
        if (e != cudaSuccess) return e;
        uint32_t tiles = (n + kTile - 1) / kTile;
        uint32_t grid = static_cast<uint32_t>(sms);
        if (grid > tiles) grid = tiles;
        k_mlp_train<<<grid, 128, kTrainSmem, st>>>(feat, target, n, reinterpret_cast<const uint4 *>(s.pack),
                                                   adam.loss_scale, s.grad, s.loss, s.err);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (update) {
        k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, st>>>(s.w, s.m, s.v, s.grad, adam, s.pack);
        e = cudaGetLastError();
    }
    return e;
}

}  // namespace vs

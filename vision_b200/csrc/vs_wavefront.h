// Wavefront form of the path tracer (wavefront.cu): the bounce loop of
// IlluminationIntegrator::Li split into kernels that pass path state through
// device memory, so that traversal runs in small kernels with high occupancy
// and the shading code runs without the traversal code beside it.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "vs_devscene.h"

namespace vs {

// Path state of `capacity` slots, structure of arrays (one 16-byte record per
// slot and field, so every kernel reads and writes whole vectors).
struct WfBuffers {
    uint32_t capacity;
    float4 *o;       // ray origin, w: pdf of the sampled direction
    float4 *d;       // ray direction, w: eta scale of Russian roulette
    float4 *tp;      // throughput at up to 4 hero wavelengths
    float4 *lam;     // hero wavelengths
    float4 *pdf;     // their pdfs (0: invalidated by dispersion)
    float4 *L;       // radiance gathered so far (linear sRGB)
    uint4 *st;       // sampler state (lo, hi), bounce, unused
    Hit *hit;        // closest hit of the slot's current ray (inst_id kInvalid: miss)
    uint32_t *queue[2];  // slots whose ray is traced next (double-buffered by bounce)
    float4 *sh_o;    // shadow queue: origin + t_max
    float4 *sh_d;    // direction + slot (bits 0..30) and a last-bounce flag (bit 31)
    float4 *sh_c;    // contribution when unoccluded (linear sRGB), w: scene id
    uint32_t *tq;    // hits sorted by shading class: class c at tq[c * capacity]
    uint32_t *count; // [0], [1]: path queue lengths; [2]: shadow queue length;
                     // [3 + c]: length of shading class c; [kWfFetchExtend],
                     // [kWfFetchShadow]: rays handed out by the traversal kernels
    // Ray binning (all null: off).  Before a traversal pass the queued rays
    // are grouped by a key of direction octant and origin cell: bin_key holds
    // each entry's key, bins 2 x kWfBins counters (sizes, then write
    // positions), binned the path queue in bin order, sh_perm the shadow
    // queue's entries in bin order.
    uint32_t *bin_key;
    uint32_t *bins;
    uint32_t *binned;
    uint32_t *sh_perm;
};

// Ray-binning keys: 3 bits of direction octant above a 9-bit Morton code of
// the ray origin's cell in an 8 x 8 x 8 grid over the scene's bounds.
constexpr uint32_t kWfBinBits = 12;
constexpr uint32_t kWfBins = 1u << kWfBinBits;

// Shading classes of a hit: 0 = miss, 1 + MaterialType otherwise.  Each class
// is shaded by its own kernel, compiled with that material's code only.
constexpr uint32_t kWfClasses = 8;
constexpr uint32_t kWfFetchExtend = 3 + kWfClasses;
constexpr uint32_t kWfFetchShadow = kWfFetchExtend + 1;
constexpr uint32_t kWfCounters = kWfFetchShadow + 1;

// Bytes of device memory per slot of WfBuffers.
constexpr size_t kWfBytesPerSlot = 6 * 16 + 16 + 16 + 2 * 4 + 3 * 16 + kWfClasses * 4;

// Renders the paths of frames [frame_begin, frame_begin + frame_count) into
// radiance[] (one float4 per path, frame-major, as launch_render) in waves of
// at most b.capacity paths.  `launches` gets the number of kernels launched.
// class_mask: bit c set when shading class c can occur (bit 0, misses, is
// always launched); classes without a bit are not launched.
cudaError_t launch_render_wavefront(const DeviceScene &s, uint32_t frame_begin, uint32_t frame_count,
                                    float4 *radiance, const WfBuffers &b, uint32_t class_mask, cudaStream_t st,
                                    unsigned *launches);

}  // namespace vs

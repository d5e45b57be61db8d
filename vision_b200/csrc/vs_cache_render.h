// Cache-terminated path tracing (cache_render.cu): camera paths stop after two
// bounces and take the radiance cache's prediction for the rest; a strided
// subset of them continues two bounces further to produce the cache's
// training samples (suffix radiance plus the cache at the suffix end).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "vs_devscene.h"
#include "vs_mlp.h"
#include "vs_wavefront.h"

namespace vs {

// Per-pixel path state at the query vertex: throughput (3 hero wavelengths;
// w: the camera sample's filter weight), wavelengths, wavelength pdfs,
// radiance gathered before the query (rgb) and a validity flag (w of the last
// float4).
struct CacheQueryRec {
    float4 t, lambda, pdf, l_valid;
};

// Per training sample: suffix radiance at the 3 hero wavelengths and the
// bootstrap flag, throughput from the query vertex to the suffix end,
// wavelengths and pdfs.
struct CacheTrainRec {
    float4 suffix_valid, t, lambda, pdf;
};

struct CacheFrameParams {
    f3 bmin;             // scene bounds for the position encoding
    f3 binv;             // 1 / extent
    const float4 *mat;   // per material: albedo rgb, roughness (alpha)
    uint16_t *q_feat;    // npix x 64 BF16 features of the query vertices
    CacheQueryRec *q_rec;
    float4 *q_out;       // cache output per query
    uint32_t n_train, train_stride, train_offset;
    uint16_t *t_feat;    // n_train x 64 features of the training vertices
    uint16_t *b_feat;    // n_train x 64 features of the suffix ends
    CacheTrainRec *t_rec;
    float4 *b_out;       // cache output per suffix end
    float4 *targets;     // n_train training targets
    uint32_t frame;
    uint32_t query_depth;  // bounces before the query (2)
    uint32_t suffix_depth; // extra bounces of training paths (2)
};

cudaError_t upload_spectral_consts_cache(const float *x, const float *y, const float *z, const float *d65,
                                         float y_integral);
// One frame: path kernel, cache inference on queries and suffix ends,
// resolve (film + training targets).  The caller then trains the cache.
cudaError_t launch_cache_frame(const DeviceScene &s, const CacheFrameParams &p, const MlpState &mlp, float4 *film32,
                               double *film64, uint32_t film_index, cudaStream_t st, unsigned *launches);
// The same frame with the paths as wavefront passes over the slots of `b`
// (capacity >= the frame's pixels): `ended` (one float4 per pixel) receives
// the radiance of paths that end before their query vertex, `suffix_list`
// (n_train entries) and `suffix_count` hold the training paths.
cudaError_t launch_cache_frame_wavefront(const DeviceScene &s, const CacheFrameParams &p, const MlpState &mlp,
                                         float4 *film32, double *film64, uint32_t film_index, const WfBuffers &b,
                                         uint32_t class_mask, float4 *ended, uint32_t *suffix_list,
                                         uint32_t *suffix_count, cudaStream_t st, unsigned *launches);

}  // namespace vs

// Host-callable launch wrappers of the kernels in kernels.cu.
#pragma once

#include <cuda_runtime.h>
#include "vs_devscene.h"
#include "vs_restir.h"
#include "vs_wavefront.h"

namespace vs {

cudaError_t upload_spectral_consts(const float *x, const float *y, const float *z, const float *d65, float y_integral);
cudaError_t launch_trace_closest(const DeviceScene &s, const float *rays, uint32_t n, Hit *hits, float *t,
                                 cudaStream_t st);
cudaError_t launch_trace_any(const DeviceScene &s, const float *rays, uint32_t n, uint32_t *occ, cudaStream_t st);
// Sampler streams (kernels.cu): `count` streams started at keys (px, py,
// sample, dim), `draws` draws each, to out (device memory).
cudaError_t launch_sampler_stream(const uint4 *keys, uint32_t count, uint32_t draws, uint32_t kind, uint32_t seed,
                                  float *out, cudaStream_t st);
// path_counter: one device word; when given, the persistent regenerating
// kernel traces the paths (same output as the one-path-per-thread grid).
cudaError_t launch_render(const DeviceScene &s, uint32_t frame_begin, uint32_t frame_count, float4 *radiance,
                          cudaStream_t st, unsigned long long *path_counter = nullptr);
// film64: double4 sums per pixel; film64sq (optional): double4 sums of squares.
cudaError_t launch_film(const float4 *radiance, uint32_t npix, uint32_t frame_begin, uint32_t frame_count, float4 *film32,
                        double *film64, cudaStream_t st, double *film64sq = nullptr);
unsigned long long launch_count();
void add_launches(unsigned n);
// wavefront.cu
cudaError_t upload_spectral_consts_wf(const float *x, const float *y, const float *z, const float *d65, float y_integral);

// Albedo tables (kLutFloats floats at `out`, device memory) with strata^2
// samples per cell (lut_gen.cu).
cudaError_t launch_albedo_luts(float *out, uint32_t strata, cudaStream_t st);
// server.cu
cudaError_t upload_spectral_consts_serve(const float *x, const float *y, const float *z, const float *d65,
                                         float y_integral);
// restir.cu (every material) and restir_diffuse.cu (diffuse and black-body
// surfaces only): the same kernels in two namespaces.  In launch_rt_frame,
// wf / radiance (one slot and one float4 per pixel), when given, run the
// initial indirect samples as wavefront passes (class_mask as for the plain
// wavefront); otherwise as the one-kernel k_gi_initial.
#define VS_RT_DECLARE(ns)                                                                                          \
    namespace ns {                                                                                                 \
    cudaError_t upload_spectral_consts_rt(const float *x, const float *y, const float *z, const float *d65,       \
                                          float y_integral);                                                       \
    cudaError_t launch_rt_reset(uint32_t npix, const RtBuffers &b, cudaStream_t st);                               \
    cudaError_t launch_rt_frame(const DeviceScene &s, const RtParams &p, const RtBuffers &b, uint32_t film_index,  \
                                float4 *film, const WfBuffers *wf, float4 *radiance, uint32_t class_mask,          \
                                cudaStream_t st, unsigned *launches);                                              \
    }
VS_RT_DECLARE(rt_all)
VS_RT_DECLARE(rt_diffuse)
#undef VS_RT_DECLARE
// svgf.cu: the SVGF passes after a real-time frame (G-buffer, gradients,
// demodulation, reprojection, moment filter, N a-trous passes, modulation).
// `prev_d` is the SVGFData buffer that holds the previous frame's result;
// *final_d gets the one that holds this frame's.
cudaError_t upload_spectral_consts_svgf(const float *x, const float *y, const float *z, const float *d65,
                                       float y_integral);
cudaError_t launch_svgf(const DeviceScene &s, const RtParams &p, const SvgfParams &sp, const SvgfBuffers &b,
                        uint32_t prev_d, uint32_t *final_d, cudaStream_t st, unsigned *launches);
// Exposed and tone-mapped pictures of the linear film (k_film_picture):
// `passes` applications of the tone mapper, then the sRGB gamma if asked;
// float4 to `out`, or 8-bit RGBA to `out8` when it is not null.
cudaError_t launch_picture(const float4 *film, uint32_t npix, float exposure, uint32_t tone_mapper, uint32_t passes,
                           bool gamma, float4 *out, uchar4 *out8, cudaStream_t st);

}  // namespace vs

// Albedo tables of the energy-compensated lobes on the GPU: the estimator of
// luts.cpp (vs_lut_samples.h) with one block per table cell, so that the
// tables can be regenerated with many more samples per cell than the CPU
// affords (the reference's apps/precompute drew 2^21 per cell,
// material.h:121-163).  Compute-bound: each sample is a few hundred FP32
// operations; sums are kept in FP64.
#include <cuda_runtime.h>

#include "vs_lut_samples.h"

namespace vs {

namespace {

constexpr int kLutThreads = 256;

__global__ void __launch_bounds__(kLutThreads) k_albedo_luts(float *out, uint32_t strata) {
    __shared__ double s_acc[2][kLutThreads / 32];
    const LutCell cell = lut_cell(blockIdx.x);
    const uint32_t n = strata * strata;
    double acc[2] = {0.0, 0.0};
    for (uint32_t k = threadIdx.x; k < n; k += kLutThreads) lut_sample(cell, strata, k, acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        acc[0] += __shfl_down_sync(0xffffffffu, acc[0], o);
        acc[1] += __shfl_down_sync(0xffffffffu, acc[1], o);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        s_acc[0][warp] = acc[0];
        s_acc[1][warp] = acc[1];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t[2] = {0.0, 0.0};
        for (int w = 0; w < kLutThreads / 32; ++w) {
            t[0] += s_acc[0][w];
            t[1] += s_acc[1][w];
        }
        lut_store(cell, t, n, out);
    }
}

}  // namespace

cudaError_t launch_albedo_luts(float *out, uint32_t strata, cudaStream_t st) {
    k_albedo_luts<<<kLutCells, kLutThreads, 0, st>>>(out, strata);
    return cudaGetLastError();
}

}  // namespace vs

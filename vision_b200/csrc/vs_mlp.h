// Radiance-cache MLP: 64 inputs -> 4 hidden layers of 64 (ReLU) -> 3 outputs,
// no biases, BF16 weights and activations with FP32 accumulation on the
// tcgen05 tensor cores (mlp.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace vs {

constexpr int kMlpIn = 64;
constexpr int kMlpHidden = 64;
constexpr int kMlpOut = 3;
constexpr int kMlpOutPad = 16;     // output layer padded to the smallest M=128 MMA width
constexpr int kMlpHiddenLayers = 4;
// Weights: 4 x 64 x 64 (input + 3 hidden-to-hidden) + 64 x 3 (output) = 16,576.
constexpr int kMlpParams = kMlpHiddenLayers * kMlpIn * kMlpHidden + kMlpHidden * kMlpOut;
// Packed BF16 image of the weights as the kernels keep them in shared memory:
// forward operands (4 x 64x64 + 16x64) then backward operands (4 x 64x64 + 64x16).
constexpr int kMlpPackFwd = kMlpHiddenLayers * 4096 + kMlpOutPad * 64;
constexpr int kMlpPackElems = 2 * kMlpPackFwd;

struct MlpAdam {
    float lr, beta1, beta2, eps;
    uint32_t step;  // 1-based step of the next update
    float loss_scale;  // 1 / (3 n) of the mean relative L2 loss
};

// Master FP32 weights W[l][in][out] (row-major per layer, layers 0..4),
// packed BF16 image, Adam moments, gradient accumulator, loss accumulator,
// and a device error flag (non-zero after a timed-out tensor-core wait).
struct MlpState {
    float *w;        // kMlpParams
    uint16_t *pack;  // kMlpPackElems (BF16 bits)
    float *m, *v;    // kMlpParams
    float *grad;     // kMlpParams
    double *loss;    // 1
    int *err;        // 1
};

cudaError_t mlp_pack(const MlpState &s, cudaStream_t st);
// out[i] = (r, g, b, 0) for n feature rows (64 BF16 each, 16-byte aligned).
cudaError_t mlp_infer(const MlpState &s, const uint16_t *feat, uint32_t n, float4 *out, cudaStream_t st);
// Gradient of the mean relative L2 loss sum_c (y_c - t_c)^2 / (y_c^2 + 0.01)
// over n samples (targets as float4), accumulated into s.grad (zeroed here),
// and the loss into s.loss; then one Adam update of the weights and a repack.
cudaError_t mlp_train_step(const MlpState &s, const uint16_t *feat, const float4 *target, uint32_t n, MlpAdam adam,
                           bool update, cudaStream_t st);

}  // namespace vs

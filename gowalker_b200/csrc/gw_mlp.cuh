// Block-demand predictor: a 16 -> 64 -> 64 -> 1 ReLU MLP in fp32 with
// hand-written forward, backward and Adam kernels (no library GEMM: the
// network is 5,313 weights applied to at most a few thousand rows, far too
// small for tensor cores to matter; one CTA of 64 threads per row group keeps
// every weight in shared memory).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gw {

constexpr int kMlpIn = 16;
constexpr int kMlpHid = 64;
// flat parameter layout
constexpr int kOffW1 = 0;                                   // [kMlpHid][kMlpIn]
constexpr int kOffB1 = kOffW1 + kMlpHid * kMlpIn;           // [kMlpHid]
constexpr int kOffW2 = kOffB1 + kMlpHid;                    // [kMlpHid][kMlpHid]
constexpr int kOffB2 = kOffW2 + kMlpHid * kMlpHid;          // [kMlpHid]
constexpr int kOffW3 = kOffB2 + kMlpHid;                    // [kMlpHid]
constexpr int kOffB3 = kOffW3 + kMlpHid;                    // [1]
constexpr int kMlpParams = kOffB3 + 1;                      // 5313
constexpr int kMlpGradCtas = 32;                            // CTAs of the gradient kernel

cudaError_t mlp_forward(const float *params, const float *x, uint32_t n, float *y, cudaStream_t s);
// Mean-squared-error gradient over n rows into grad (kMlpParams floats) and
// loss (1 float); ws must hold kMlpGradCtas * (kMlpParams + 1) floats.
cudaError_t mlp_grad(const float *params, const float *x, const float *t, uint32_t n, float *grad, float *loss,
                     float *ws, cudaStream_t s);
cudaError_t mlp_adam(float *params, const float *grad, float *m, float *v, float lr, uint32_t step, cudaStream_t s);
// Deterministic small init (Philox from a seed), He-scaled.
cudaError_t mlp_init(float *params, uint64_t seed, cudaStream_t s);
// Full-batch Adam; ws = grad partials, grad, m, v (+ loss when loss_dev is null).
cudaError_t mlp_train(float *params, const float *x, const float *t, uint32_t n, uint32_t epochs, float lr,
                      uint64_t seed, float *ws, float *loss_dev, cudaStream_t s);

}  // namespace gw

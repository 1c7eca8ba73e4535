// Kernels of the block-demand MLP (see gw_mlp.cuh).  One CTA of 64 threads
// processes a group of rows; thread j owns hidden unit j of both layers, so
// every gradient slot has exactly one writer within a CTA and the per-CTA
// partial gradients are summed in a fixed order: training is deterministic.
#include <cuda_runtime.h>
#include <cmath>
#include "gw_mlp.cuh"
#include "gw_philox.cuh"

namespace gw {

constexpr int kW2Pitch = kMlpHid + 1;  // padded rows: column reads hit distinct banks

__device__ __forceinline__ float sum64(float v, float *red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    const float s = red[0] + red[1];
    __syncthreads();
    return s;
}

__global__ void __launch_bounds__(kMlpHid) k_mlp_forward(const float *__restrict__ P, const float *__restrict__ X,
                                                         uint32_t n, float *__restrict__ Y)
{
    __shared__ float sW2[kMlpHid * kW2Pitch];
    __shared__ float sX[kMlpIn], sH1[kMlpHid], sRed[2];
    const int j = threadIdx.x;
    for (int k = j; k < kMlpHid * kMlpHid; k += kMlpHid) sW2[(k / kMlpHid) * kW2Pitch + (k % kMlpHid)] = P[kOffW2 + k];
    float w1[kMlpIn];
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) w1[i] = P[kOffW1 + j * kMlpIn + i];
    const float b1 = P[kOffB1 + j], b2 = P[kOffB2 + j], w3 = P[kOffW3 + j], b3 = P[kOffB3];
    __syncthreads();
    for (uint32_t s = blockIdx.x; s < n; s += gridDim.x) {
        if (j < kMlpIn) sX[j] = X[(uint64_t)s * kMlpIn + j];
        __syncthreads();
        float a1 = b1;
#pragma unroll
        for (int i = 0; i < kMlpIn; ++i) a1 = fmaf(w1[i], sX[i], a1);
        sH1[j] = fmaxf(a1, 0.f);
        __syncthreads();
        float a2 = b2;
#pragma unroll 16
        for (int k = 0; k < kMlpHid; ++k) a2 = fmaf(sW2[j * kW2Pitch + k], sH1[k], a2);
        const float y = b3 + sum64(w3 * fmaxf(a2, 0.f), sRed);
        if (j == 0) Y[s] = y;
    }
}

__global__ void __launch_bounds__(kMlpHid) k_mlp_grad(const float *__restrict__ P, const float *__restrict__ X,
                                                      const float *__restrict__ T, uint32_t n, float *__restrict__ ws)
{
    __shared__ float sW2[kMlpHid * kW2Pitch];
    __shared__ float sX[kMlpIn], sH1[kMlpHid], sD2[kMlpHid], sRed[2];
    const int j = threadIdx.x;
    for (int k = j; k < kMlpHid * kMlpHid; k += kMlpHid) sW2[(k / kMlpHid) * kW2Pitch + (k % kMlpHid)] = P[kOffW2 + k];
    float w1[kMlpIn], gW1[kMlpIn], gW2[kMlpHid];
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) {
        w1[i] = P[kOffW1 + j * kMlpIn + i];
        gW1[i] = 0.f;
    }
#pragma unroll
    for (int k = 0; k < kMlpHid; ++k) gW2[k] = 0.f;
    const float b1 = P[kOffB1 + j], b2 = P[kOffB2 + j], w3 = P[kOffW3 + j], b3 = P[kOffB3];
    float gb1 = 0.f, gb2 = 0.f, gW3 = 0.f, gb3 = 0.f, loss = 0.f;
    const float inv_n = 1.0f / (float)n;
    __syncthreads();
    for (uint32_t s = blockIdx.x; s < n; s += gridDim.x) {
        if (j < kMlpIn) sX[j] = X[(uint64_t)s * kMlpIn + j];
        __syncthreads();
        float a1 = b1;
#pragma unroll
        for (int i = 0; i < kMlpIn; ++i) a1 = fmaf(w1[i], sX[i], a1);
        const float h1 = fmaxf(a1, 0.f);
        sH1[j] = h1;
        __syncthreads();
        float a2 = b2;
#pragma unroll 16
        for (int k = 0; k < kMlpHid; ++k) a2 = fmaf(sW2[j * kW2Pitch + k], sH1[k], a2);
        const float h2 = fmaxf(a2, 0.f);
        const float y = b3 + sum64(w3 * h2, sRed);
        const float e = y - T[s];
        const float dy = 2.f * e * inv_n;
        if (j == 0) {
            loss += e * e;
            gb3 += dy;
        }
        gW3 += dy * h2;
        const float d2 = (a2 > 0.f) ? dy * w3 : 0.f;
        sD2[j] = d2;
        gb2 += d2;
#pragma unroll 16
        for (int k = 0; k < kMlpHid; ++k) gW2[k] = fmaf(d2, sH1[k], gW2[k]);
        __syncthreads();
        float d1 = 0.f;
#pragma unroll 16
        for (int r = 0; r < kMlpHid; ++r) d1 = fmaf(sW2[r * kW2Pitch + j], sD2[r], d1);
        d1 = (a1 > 0.f) ? d1 : 0.f;
        gb1 += d1;
#pragma unroll
        for (int i = 0; i < kMlpIn; ++i) gW1[i] = fmaf(d1, sX[i], gW1[i]);
        __syncthreads();
    }
    float *o = ws + (uint64_t)blockIdx.x * (kMlpParams + 1);
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) o[kOffW1 + j * kMlpIn + i] = gW1[i];
    o[kOffB1 + j] = gb1;
#pragma unroll 16
    for (int k = 0; k < kMlpHid; ++k) o[kOffW2 + j * kMlpHid + k] = gW2[k];
    o[kOffB2 + j] = gb2;
    o[kOffW3 + j] = gW3;
    if (j == 0) {
        o[kOffB3] = gb3;
        o[kMlpParams] = loss;
    }
}

__global__ void k_mlp_reduce(const float *__restrict__ ws, uint32_t n, float *__restrict__ grad, float *__restrict__ loss)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > kMlpParams) return;
    float s = 0.f;
    for (int b = 0; b < kMlpGradCtas; ++b) s += ws[(uint64_t)b * (kMlpParams + 1) + p];
    if (p < kMlpParams) grad[p] = s;
    else *loss = s / (float)n;
}

__global__ void k_mlp_adam(float *__restrict__ P, const float *__restrict__ G, float *__restrict__ M,
                           float *__restrict__ V, float lr, float c1, float c2)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kMlpParams) return;
    const float g = G[p];
    const float m = 0.9f * M[p] + 0.1f * g;
    const float v = 0.999f * V[p] + 0.001f * g * g;
    M[p] = m;
    V[p] = v;
    P[p] -= lr * (m / c1) / (sqrtf(v / c2) + 1e-8f);
}

__global__ void k_mlp_init(float *P, uint32_t k0, uint32_t k1)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kMlpParams) return;
    float scale = 0.f;
    // hidden layers uniform in +-sqrt(6 / fan_in); the output layer starts at
    // zero, so an untrained network outputs 0 (the residual forecast: "no
    // change") and training moves it only where the data says so
    if (p < kOffB1) scale = 0.6123724f;              // sqrt(6 / 16)
    else if (p >= kOffW2 && p < kOffB2) scale = 0.30618622f;  // sqrt(6 / 64)
    const U4 r = philox4x32_10((uint32_t)p, 0x4D4C5031u, 0u, 0u, k0, k1);
    const float u = __uint2float_rn(r.x >> 8) * 0x1p-24f;
    P[p] = (2.f * u - 1.f) * scale;
}

cudaError_t mlp_forward(const float *params, const float *x, uint32_t n, float *y, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    const uint32_t grid = n < 1024 ? n : 1024;
    k_mlp_forward<<<grid, kMlpHid, 0, s>>>(params, x, n, y);
    return cudaGetLastError();
}

cudaError_t mlp_grad(const float *params, const float *x, const float *t, uint32_t n, float *grad, float *loss,
                     float *ws, cudaStream_t s)
{
    if (n == 0) return cudaErrorInvalidValue;
    k_mlp_grad<<<kMlpGradCtas, kMlpHid, 0, s>>>(params, x, t, n, ws);
    k_mlp_reduce<<<(kMlpParams + 1 + 255) / 256, 256, 0, s>>>(ws, n, grad, loss);
    return cudaGetLastError();
}

cudaError_t mlp_adam(float *params, const float *grad, float *m, float *v, float lr, uint32_t step, cudaStream_t s)
{
    const float c1 = 1.f - (float)std::pow(0.9, (double)step);
    const float c2 = 1.f - (float)std::pow(0.999, (double)step);
    k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, s>>>(params, grad, m, v, lr, c1, c2);
    return cudaGetLastError();
}

cudaError_t mlp_init(float *params, uint64_t seed, cudaStream_t s)
{
    k_mlp_init<<<(kMlpParams + 255) / 256, 256, 0, s>>>(params, (uint32_t)seed, (uint32_t)(seed >> 32));
    return cudaGetLastError();
}

cudaError_t mlp_train(float *params, const float *x, const float *t, uint32_t n, uint32_t epochs, float lr,
                      uint64_t seed, float *ws, float *loss_dev, cudaStream_t s)
{
    float *gws = ws;
    float *grad = gws + (uint64_t)kMlpGradCtas * (kMlpParams + 1);
    float *m = grad + kMlpParams;
    float *v = m + kMlpParams;
    float *loss = loss_dev ? loss_dev : v + kMlpParams;
    cudaError_t e = cudaSuccess;
    if (seed) e = mlp_init(params, seed, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(m, 0, sizeof(float) * 2 * kMlpParams, s);
    for (uint32_t ep = 1; ep <= epochs && e == cudaSuccess; ++ep) {
        e = mlp_grad(params, x, t, n, grad, loss, gws, s);
        if (e == cudaSuccess) e = mlp_adam(params, grad, m, v, lr, ep, s);
    }
    return e;
}

}  // namespace gw

// ------------------------------------------------------------------ C ABI (caller-owned device buffers)
#include "../../include/gowalker.h"
static_assert(gw::kMlpParams == GW_MLP_PARAMS, "parameter count matches the header");
static_assert(gw::kMlpIn == GW_MLP_INPUTS, "input width matches the header");
static_assert(gw::kMlpGradCtas * (gw::kMlpParams + 1) == GW_MLP_GRAD_WS_FLOATS, "workspace matches the header");

extern "C" int gw_mlp_forward(const float *d_params, const float *d_x, uint32_t n, float *d_y)
{
    if (!d_params || !d_x || !d_y) return GW_ERR_ARG;
    cudaError_t e = gw::mlp_forward(d_params, d_x, n, d_y, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) cudaGetLastError();
    return e == cudaSuccess ? GW_OK : GW_ERR_CUDA;
}

extern "C" int gw_mlp_grad(const float *d_params, const float *d_x, const float *d_t, uint32_t n, float *d_grad,
                           float *d_loss, float *d_ws)
{
    if (!d_params || !d_x || !d_t || !d_grad || !d_loss || !d_ws || n == 0) return GW_ERR_ARG;
    cudaError_t e = gw::mlp_grad(d_params, d_x, d_t, n, d_grad, d_loss, d_ws, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) cudaGetLastError();
    return e == cudaSuccess ? GW_OK : GW_ERR_CUDA;
}

extern "C" int gw_mlp_train(float *d_params, const float *d_x, const float *d_t, uint32_t n, uint32_t epochs,
                            float lr, uint64_t seed, float *d_ws, float *loss_out)
{
    if (!d_params || !d_x || !d_t || !d_ws || n == 0 || !(lr > 0.f)) return GW_ERR_ARG;
    float *loss_dev = d_ws + GW_MLP_GRAD_WS_FLOATS + 3 * GW_MLP_PARAMS;
    cudaError_t e = gw::mlp_train(d_params, d_x, d_t, n, epochs, lr, seed, d_ws, loss_dev, 0);
    if (e == cudaSuccess && loss_out) e = cudaMemcpy(loss_out, loss_dev, sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) cudaGetLastError();
    return e == cudaSuccess ? GW_OK : GW_ERR_CUDA;
}

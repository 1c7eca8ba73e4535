// Test-only: the warp's windowed integer bounds (rand_bounds) against the
// exhaustive binary search (rand_prefix), one step's thresholds per warp.
#include <cstdint>
#include <cuda_runtime.h>
#include "gw_step.cuh"

using namespace gw;

template <bool SOPR>
__global__ void k_bounds(const float *thr, uint32_t n, uint32_t *fast, uint32_t *slow)
{
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31u;
    if (w >= n) return;
    StepConsts c{};
    StepThr t{0.f, 0.f, 0.f};
    const float *p = thr + 5 * (uint64_t)w;
    if (SOPR) {
        t.inv_deg = p[0];
        t.sum = p[1];
        t.t_prev = p[2];
    } else {
        c.n2v_maxv = p[0];
        c.n2v_minv = p[1];
        c.inv_p = p[2];
        c.inv_q = p[3];
    }
    const uint32_t k = rand_bounds<SOPR>(c, t);
    if ((lane & 7u) == 0) fast[4 * w + (lane >> 3)] = k;
    if (lane < 4) {
        const float maxv = thr_max<SOPR>(c, t);
        const float bound = lane == 0 ? thr_min<SOPR>(c, t) : lane == 1 ? thr_prev<SOPR>(c, t)
                          : lane == 2 ? thr_found<SOPR>(c, t) : thr_notfound<SOPR>(c, t);
        slow[4 * w + lane] = rand_prefix([&](uint32_t kk) {
            const float rv = rand_val(kk << 8, maxv);
            return lane == 0 ? (rv <= bound) : (rv < bound);
        });
    }
}

extern "C" int check_bounds(int sopr, const float *h_thr, uint32_t n, uint32_t *h_fast, uint32_t *h_slow)
{
    float *thr;
    uint32_t *fast, *slow;
    if (cudaMalloc(&thr, sizeof(float) * 5 * n) || cudaMalloc(&fast, 16ull * n) || cudaMalloc(&slow, 16ull * n))
        return 1;
    cudaMemcpy(thr, h_thr, sizeof(float) * 5 * n, cudaMemcpyHostToDevice);
    const uint32_t blocks = (n * 32 + 255) / 256;
    if (sopr) k_bounds<true><<<blocks, 256>>>(thr, n, fast, slow);
    else k_bounds<false><<<blocks, 256>>>(thr, n, fast, slow);
    cudaError_t e = cudaDeviceSynchronize();
    cudaMemcpy(h_fast, fast, 16ull * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(h_slow, slow, 16ull * n, cudaMemcpyDeviceToHost);
    cudaFree(thr);
    cudaFree(fast);
    cudaFree(slow);
    return e == cudaSuccess ? 0 : 2;
}

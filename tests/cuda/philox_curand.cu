// Test-only probe: the engine's device Philox4x32-10 next to curand's
// Philox4_32_10 for the same key and counter.  curand_init(seed, subsequence,
// 0) starts at counter (0, 0, subsequence_lo, subsequence_hi) with key
// (seed_lo, seed_hi); curand4 then returns the generator output at that
// counter and advances the first counter word.
#include <curand_kernel.h>
#include <cstdint>
#include "gw_philox.cuh"

__global__ void k_probe(uint64_t seed, uint64_t sub0, int n, uint32_t *ours, uint32_t *theirs)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t sub = sub0 + (uint64_t)i;
    curandStatePhilox4_32_10_t st;
    curand_init(seed, sub, 0, &st);
    const uint4 a = curand4(&st);
    const uint4 b = curand4(&st);
    const gw::U4 x = gw::philox4x32_10(0, 0, (uint32_t)sub, (uint32_t)(sub >> 32), (uint32_t)seed,
                                       (uint32_t)(seed >> 32));
    const gw::U4 y = gw::philox4x32_10(1, 0, (uint32_t)sub, (uint32_t)(sub >> 32), (uint32_t)seed,
                                       (uint32_t)(seed >> 32));
    uint32_t *o = ours + 8 * i, *t = theirs + 8 * i;
    o[0] = x.x; o[1] = x.y; o[2] = x.z; o[3] = x.w;
    o[4] = y.x; o[5] = y.y; o[6] = y.z; o[7] = y.w;
    t[0] = a.x; t[1] = a.y; t[2] = a.z; t[3] = a.w;
    t[4] = b.x; t[5] = b.y; t[6] = b.z; t[7] = b.w;
}

extern "C" int probe_philox(uint64_t seed, uint64_t sub0, int n, uint32_t *h_ours, uint32_t *h_theirs)
{
    uint32_t *d = nullptr;
    if (cudaMalloc(&d, sizeof(uint32_t) * 16 * n) != cudaSuccess) return 1;
    k_probe<<<(n + 127) / 128, 128>>>(seed, sub0, n, d, d + 8 * n);
    int rc = 0;
    if (cudaMemcpy(h_ours, d, sizeof(uint32_t) * 8 * n, cudaMemcpyDeviceToHost) != cudaSuccess) rc = 2;
    if (cudaMemcpy(h_theirs, d + 8 * n, sizeof(uint32_t) * 8 * n, cudaMemcpyDeviceToHost) != cudaSuccess) rc = 2;
    cudaFree(d);
    return rc;
}

// Synthetic graph construction on the device (gw_rmat_csr).
//
// Stands in for the reference's text-to-CSR converter (GOWalker
// preprocess/graph_converter.hpp:286-449, which cannot run as shipped) for the
// synthetic R-MAT inputs: every edge sample is a pure function of
// (seed, sample index), so the graph is identical whichever device, chunking
// or thread count builds it, and identical to the oracle's CPU build.
//
// Pipeline: sample kernel -> u64 keys (src<<32|dst, invalid = ~0) ->
// radix sort (CUB) -> unique (CUB) -> optional even thinning to an exact edge
// count -> offsets kernel + neighbour extraction.
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>
#include <cstdint>
#include "gw_philox.cuh"
#include "../../include/gowalker.h"

namespace gw {

__global__ void k_rmat_keys(uint32_t scale, uint32_t nverts, uint64_t nsamples, uint32_t t0, uint32_t t1,
                            uint32_t t2, uint32_t k0, uint32_t k1, int symmetric, uint64_t *keys)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nsamples; e += stride) {
        uint32_t s = 0, d = 0;
        U4 r{0, 0, 0, 0};
        for (uint32_t l = 0; l < scale; ++l) {
            if ((l & 3u) == 0) r = philox4x32_10((uint32_t)e, (uint32_t)(e >> 32), l >> 2, kTagRmat, k0, k1);
            const uint32_t lanes[4] = {r.x, r.y, r.z, r.w};
            const uint32_t u = lanes[l & 3u];
            uint32_t sb, db;
            if (u < t0) { sb = 0; db = 0; }
            else if (u < t1) { sb = 0; db = 1; }
            else if (u < t2) { sb = 1; db = 0; }
            else { sb = 1; db = 1; }
            s = (s << 1) | sb;
            d = (d << 1) | db;
        }
        const bool ok = s < nverts && d < nverts && s != d;
        const uint64_t kf = ok ? (((uint64_t)s << 32) | d) : ~0ull;
        if (symmetric) {
            keys[2 * e] = kf;
            keys[2 * e + 1] = ok ? (((uint64_t)d << 32) | s) : ~0ull;
        } else {
            keys[e] = kf;
        }
    }
}

// Keep unique edge i unless floor((i+1)k/U) > floor(ik/U): exactly k of the U
// edges go, spread evenly over the sorted list.
__global__ void k_thin(const uint64_t *in, uint64_t U, uint64_t k, uint64_t *out)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < U; i += stride) {
        const unsigned __int128 a = (unsigned __int128)i * k / U;
        const unsigned __int128 b = (unsigned __int128)(i + 1) * k / U;
        if (a == b) out[i - (uint64_t)a] = in[i];
    }
}

// beg[v] = first index whose source >= v; csr[i] = low word of key i.
__global__ void k_offsets(const uint64_t *keys, uint64_t n, uint32_t nverts, uint64_t *beg, uint32_t *csr)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += stride) {
        const int64_t s_here = (i < n) ? (int64_t)(keys[i] >> 32) : (int64_t)nverts;
        const int64_t s_prev = (i > 0) ? (int64_t)(keys[i - 1] >> 32) : -1;
        for (int64_t v = s_prev + 1; v <= s_here; ++v) beg[v] = i;
        if (i < n) csr[i] = (uint32_t)keys[i];
    }
}

}  // namespace gw

using namespace gw;

#define GEN_CHECK(x)                                  \
    do {                                              \
        cudaError_t e_ = (x);                         \
        if (e_ != cudaSuccess) { rc = GW_ERR_CUDA; goto done; } \
    } while (0)

extern "C" int gw_rmat_csr(uint32_t scale, uint32_t nverts, uint64_t nsamples, const uint32_t thr[3],
                           uint64_t seed, int symmetric, uint64_t target_edges, uint64_t **d_beg,
                           uint32_t **d_csr, uint64_t *nedges)
{
    if (!thr || !d_beg || !d_csr || !nedges || scale == 0 || scale > 32 || nverts == 0) return GW_ERR_ARG;
    if (scale < 32 && (uint64_t)nverts > (1ull << scale)) return GW_ERR_ARG;
    int rc = GW_OK;
    const uint64_t nkeys = nsamples * (symmetric ? 2 : 1);
    uint64_t *keys = nullptr, *alt = nullptr, *beg = nullptr;
    uint32_t *csr = nullptr;
    void *tmp = nullptr;
    int64_t *d_nsel = nullptr;
    size_t tmp_bytes = 0, tb2 = 0;
    int64_t nsel = 0;
    uint64_t U = 0;
    const int threads = 256;
    const int blocks = 148 * 16;
    cudaStream_t s = 0;

    GEN_CHECK(cudaMalloc(&keys, nkeys * sizeof(uint64_t)));
    GEN_CHECK(cudaMalloc(&alt, nkeys * sizeof(uint64_t)));
    GEN_CHECK(cudaMalloc(&d_nsel, sizeof(int64_t)));
    k_rmat_keys<<<blocks, threads, 0, s>>>(scale, nverts, nsamples, thr[0], thr[1], thr[2], (uint32_t)seed,
                                           (uint32_t)(seed >> 32), symmetric, keys);
    GEN_CHECK(cudaGetLastError());
    GEN_CHECK(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, keys, alt, nkeys, 0, 64, s));
    GEN_CHECK(cub::DeviceSelect::Unique(nullptr, tb2, alt, keys, d_nsel, (int64_t)nkeys, s));
    if (tb2 > tmp_bytes) tmp_bytes = tb2;
    GEN_CHECK(cudaMalloc(&tmp, tmp_bytes));
    GEN_CHECK(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, keys, alt, nkeys, 0, 64, s));
    GEN_CHECK(cub::DeviceSelect::Unique(tmp, tmp_bytes, alt, keys, d_nsel, (int64_t)nkeys, s));
    GEN_CHECK(cudaMemcpyAsync(&nsel, d_nsel, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    GEN_CHECK(cudaStreamSynchronize(s));
    U = (uint64_t)nsel;
    if (U > 0) {
        uint64_t last = 0;
        GEN_CHECK(cudaMemcpy(&last, keys + (U - 1), sizeof(uint64_t), cudaMemcpyDeviceToHost));
        if (last == ~0ull) U -= 1;  // the invalid-sample marker sorts last
    }
    if (target_edges > 0) {
        if (U < target_edges) { rc = GW_ERR_ARG; goto done; }
        if (U > target_edges) {
            k_thin<<<blocks, threads, 0, s>>>(keys, U, U - target_edges, alt);
            GEN_CHECK(cudaGetLastError());
            uint64_t *t = keys;
            keys = alt;
            alt = t;
            U = target_edges;
        }
    }
    GEN_CHECK(cudaMalloc(&beg, ((uint64_t)nverts + 1) * sizeof(uint64_t)));
    GEN_CHECK(cudaMalloc(&csr, (U ? U : 1) * sizeof(uint32_t)));
    k_offsets<<<blocks, threads, 0, s>>>(keys, U, nverts, beg, csr);
    GEN_CHECK(cudaGetLastError());
    GEN_CHECK(cudaStreamSynchronize(s));
    *d_beg = beg;
    *d_csr = csr;
    *nedges = U;
    beg = nullptr;
    csr = nullptr;
done:
    cudaFree(keys);
    cudaFree(alt);
    cudaFree(tmp);
    cudaFree(d_nsel);
    cudaFree(beg);
    cudaFree(csr);
    return rc;
}

extern "C" int gw_device_free(void *p)
{
    return cudaFree(p) == cudaSuccess ? GW_OK : GW_ERR_CUDA;
}

extern "C" int gw_host_alloc(uint64_t bytes, void **out)
{
    if (!out || bytes == 0) return GW_ERR_ARG;
    *out = nullptr;
    const cudaError_t e = cudaHostAlloc(out, bytes, cudaHostAllocPortable);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *out = nullptr;
        return e == cudaErrorMemoryAllocation ? GW_ERR_NOMEM : GW_ERR_CUDA;
    }
    return GW_OK;
}

extern "C" int gw_host_free(void *p)
{
    if (!p) return GW_OK;
    return cudaFreeHost(p) == cudaSuccess ? GW_OK : GW_ERR_CUDA;
}

extern "C" int gw_memcpy(void *dst, const void *src, uint64_t bytes)
{
    if ((!dst || !src) && bytes) return GW_ERR_ARG;
    if (!bytes) return GW_OK;
    return cudaMemcpy(dst, src, bytes, cudaMemcpyDefault) == cudaSuccess ? GW_OK : GW_ERR_CUDA;
}

// Synthetic graph construction on the device (gw_rmat_csr).
//
// Stands in for the reference's text-to-CSR converter (GOWalker
// preprocess/graph_converter.hpp:286-449, which cannot run as shipped) for the
// synthetic R-MAT inputs: every edge sample is a pure function of
// (seed, sample index), so the graph is identical whichever device, chunking
// or thread count builds it, and identical to the oracle's CPU build.
//
// Pipeline (sampled_csr): count the kept samples, write their packed keys
// (src << bit_length(V-1) | dst) compacted, radix sort (CUB) -> unique (CUB)
// -> optional even thinning to an exact edge count -> offsets + neighbour
// extraction (csr_from_sorted).  The web-shaped locality-ordered graph
// (gw_web_csr) draws a power-law degree per vertex, scans the degrees and
// writes each vertex's edges in place before the same sort.
//
// The same key pipeline turns a caller's edge list into a CSR
// (gw_edges_csr), and gw_split_blocks computes block split points from the
// offsets on the device.
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include "gw_fixedmath.cuh"
#include "gw_philox.cuh"
#include "../../include/gowalker.h"

namespace gw {

constexpr uint32_t kTagWeb = 0x57454230u;  // 'WEB0'

// R-MAT sample e: `scale` quadrant choices, level l from lane (l & 3) of
// Philox(e_lo, e_hi, l >> 2, 'RMAT') against the u32 thresholds a, a+b, a+b+c.
__device__ __forceinline__ void rmat_sample(uint64_t e, uint32_t scale, uint32_t t0, uint32_t t1, uint32_t t2,
                                            uint32_t k0, uint32_t k1, uint32_t &s, uint32_t &d)
{
    s = d = 0;
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
}

struct RmatSampler {
    uint32_t scale, nverts, t0, t1, t2, k0, k1;
    __device__ bool operator()(uint64_t e, uint32_t &s, uint32_t &d) const
    {
        rmat_sample(e, scale, t0, t1, t2, k0, k1, s, d);
        return s < nverts && d < nverts && s != d;
    }
};

// Web-shaped graph (locality-ordered ids).  Vertex v's out-degree is
// floor(dmin / u^(1/tail)) capped at max_degree, u = Philox(v, 0, 0, 'WDEG')
// lane x / 2^32 (x = 0 read as 1): a power law P(D >= d) = (d/dmin)^-tail,
// every vertex at least floor(dmin) edges, computed with the fixed-step log
// and exp so the oracle reproduces it.  Edge j of v draws Philox(j, v, 0,
// 'WEB0'): lane x % 1000 < local_permille makes it local, to v + o with o
// uniform over [-window, -1] u [1, window] (lane y), clipped to [0, nverts);
// otherwise its destination follows R-MAT's destination marginal over
// `scale` levels (bit 1 for quadrants b and d; level l from lane l & 3 of
// Philox(j, v, 1 + l/4, 'WEB0')), rejected when >= nverts.
constexpr uint32_t kTagWebDeg = 0x57444547u;  // 'WDEG'

struct WebParams {
    uint32_t nverts, scale, t0, t1, t2, k0, k1, local_permille, window, max_degree;
    double dmin, tail;
};

__device__ __forceinline__ uint32_t web_degree(const WebParams &p, uint32_t v)
{
    const U4 r = philox4x32_10(v, 0u, 0u, kTagWebDeg, p.k0, p.k1);
    const uint32_t z = r.x ? r.x : 1u;
    const double pw = fm_exp_nonpos(__ddiv_rn(fm_log_u32(z), p.tail));  // u^(1/tail), in (0, 1]
    const double d = __ddiv_rn(p.dmin, pw);
    return d >= (double)p.max_degree ? p.max_degree : (uint32_t)d;
}

// false when the edge is dropped (self loop after clipping, or a remote
// destination >= nverts)
__device__ __forceinline__ bool web_edge(const WebParams &p, uint32_t v, uint32_t j, uint32_t &dst)
{
    const U4 r = philox4x32_10(j, v, 0u, kTagWeb, p.k0, p.k1);
    if (r.x % 1000u < p.local_permille) {
        int64_t o = (int64_t)(r.y % (2u * p.window)) - (int64_t)p.window;
        if (o >= 0) o += 1;
        int64_t t = (int64_t)v + o;
        t = t < 0 ? 0 : (t >= (int64_t)p.nverts ? (int64_t)p.nverts - 1 : t);
        dst = (uint32_t)t;
    } else {
        uint32_t d = 0;
        U4 q{0, 0, 0, 0};
        for (uint32_t l = 0; l < p.scale; ++l) {
            if ((l & 3u) == 0) q = philox4x32_10(j, v, 1u + (l >> 2), kTagWeb, p.k0, p.k1);
            const uint32_t lanes[4] = {q.x, q.y, q.z, q.w};
            const uint32_t u = lanes[l & 3u];
            d = (d << 1) | (((u >= p.t0 && u < p.t1) || u >= p.t2) ? 1u : 0u);
        }
        dst = d;
    }
    return dst < p.nverts && dst != v;
}

__global__ void k_web_degrees(WebParams p, unsigned long long *deg)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v <= p.nverts; v += stride)
        deg[v] = v < p.nverts ? web_degree(p, (uint32_t)v) : 0ull;
}

// Thread per vertex: edge j of v at estart[v] + j, key v << sh | dst, or the
// marker ~0 for a dropped edge (it sorts after every kept key).
__global__ void k_web_edges(WebParams p, const unsigned long long *__restrict__ estart, uint32_t sh,
                            uint64_t *__restrict__ keys)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < p.nverts; v += stride) {
        const uint64_t e0 = estart[v], n = estart[v + 1] - e0;
        for (uint32_t j = 0; j < n; ++j) {
            uint32_t d;
            keys[e0 + j] = web_edge(p, (uint32_t)v, j, d) ? ((v << sh) | d) : ~0ull;
        }
    }
}

// Sampled edges -> packed keys src << sh | dst of the kept samples (and their
// reverses when symmetric), compacted: a block claims its output range with
// one atomic per 1024 samples.  COUNT: only count the kept keys.
template <class Sampler, bool COUNT>
__global__ void __launch_bounds__(256)
    k_sample_keys(Sampler smp, uint64_t nsamples, uint32_t sh, int symmetric, uint64_t *__restrict__ keys,
                  unsigned long long *cursor)
{
    __shared__ unsigned int s_cnt;
    __shared__ unsigned long long s_base;
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t per = symmetric ? 2 : 1;
    const uint64_t span = 256ull * 4;
    unsigned long long total = 0;
    for (uint64_t b0 = (uint64_t)blockIdx.x * span; b0 < nsamples; b0 += (uint64_t)gridDim.x * span) {
        uint32_t sv[4], dv[4];
        bool ok[4];
        uint32_t c = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint64_t e = b0 + (uint64_t)k * 256 + threadIdx.x;
            ok[k] = e < nsamples && smp(e, sv[k], dv[k]);
            c += ok[k] ? 1u : 0u;
        }
        if (COUNT) {
            total += c;
            continue;
        }
        if (threadIdx.x == 0) s_cnt = 0;
        __syncthreads();
        uint32_t x = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= (uint32_t)o) x += y;
        }
        uint32_t wbase = 0;
        if (lane == 31) wbase = atomicAdd(&s_cnt, x);
        wbase = __shfl_sync(0xFFFFFFFFu, wbase, 31);
        __syncthreads();
        if (threadIdx.x == 0) s_base = atomicAdd(cursor, (unsigned long long)s_cnt * per);
        __syncthreads();
        uint64_t pos = s_base + (uint64_t)(wbase + x - c) * per;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (!ok[k]) continue;
            keys[pos] = ((uint64_t)sv[k] << sh) | dv[k];
            if (symmetric) keys[pos + 1] = ((uint64_t)dv[k] << sh) | sv[k];
            pos += per;
        }
        __syncthreads();
    }
    if (COUNT) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) total += __shfl_xor_sync(0xFFFFFFFFu, total, o);
        if (lane == 0 && total) atomicAdd(cursor, total * per);
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

// Degrees from the runs of a source-sorted key list (key = src << sh | dst):
// the first key of a run adds -i and the last adds i+1 to cnt[src] (mod 2^64),
// so cnt[v] ends as the run length; two uncontended atomics per vertex
// whatever the gaps between sources.  csr[i] = dst of key i.
__global__ void k_runs(const uint64_t *__restrict__ keys, uint64_t n, uint32_t sh, unsigned long long *cnt,
                       uint32_t *__restrict__ csr)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t mask = (1ull << sh) - 1;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t k = keys[i];
        const uint64_t s = k >> sh;
        if (i == 0 || (keys[i - 1] >> sh) != s) atomicAdd(cnt + s, 0ull - (unsigned long long)i);
        if (i + 1 == n || (keys[i + 1] >> sh) != s) atomicAdd(cnt + s, (unsigned long long)(i + 1));
        csr[i] = (uint32_t)(k & mask);
    }
}

// key = src << 32 | dst  ->  src << sh | dst (dst < 2^sh), in place.
__global__ void k_repack(uint64_t *keys, uint64_t n, uint32_t sh)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t k = keys[i];
        keys[i] = ((k >> 32) << sh) | (k & 0xFFFFFFFFull);
    }
}

constexpr int kKeyThreads = 256, kKeyItems = 4;

// Edge list -> sort keys src << sh | dst (edge i and, when symmetric, its
// reverse).  Self loops and out-of-range ids are dropped.
//   COMPACT  kept keys go to a dense prefix of `keys` (a block claims its
//            range with one atomic per 1024 edges; order inside is arbitrary,
//            which a sort over the whole key makes irrelevant).
//   !COMPACT edge i at position i (2i and 2i+1 when symmetric), dropped ones
//            as the marker ~0, so a stable sort by source keeps input order;
//            with sh = 32 the marker sorts after every kept key for any sort
//            covering bit 32 + bit_length(nverts) - 1 (no kept source
//            reaches 2^b - 1).
// Per-thread maximum id and kept count are folded with one atomic per warp.
template <bool COMPACT>
__global__ void __launch_bounds__(kKeyThreads)
    k_edge_keys(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst, uint64_t n, uint64_t first,
                uint32_t lim, uint32_t sh, int symmetric, uint64_t *__restrict__ keys,
                unsigned long long *cursor, unsigned int *max_id, unsigned long long *nkept,
                unsigned int *range_err)
{
    __shared__ unsigned int s_cnt;
    __shared__ unsigned long long s_base;
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t per = symmetric ? 2 : 1;
    const uint64_t span = (uint64_t)kKeyThreads * kKeyItems;
    uint32_t mx = 0, bad = 0;
    uint64_t kept = 0;
    for (uint64_t b0 = (uint64_t)blockIdx.x * span; b0 < n; b0 += (uint64_t)gridDim.x * span) {
        uint32_t sv[kKeyItems], dv[kKeyItems];
        bool ok[kKeyItems];
        uint32_t c = 0;
#pragma unroll
        for (int k = 0; k < kKeyItems; ++k) {
            const uint64_t i = b0 + (uint64_t)k * kKeyThreads + threadIdx.x;
            sv[k] = dv[k] = 0;
            ok[k] = false;
            if (i < n) {
                sv[k] = __ldg(src + i);
                dv[k] = __ldg(dst + i);
                const bool in_range = sv[k] < lim && dv[k] < lim;
                ok[k] = in_range && sv[k] != dv[k];
                bad |= in_range ? 0u : 1u;
                if (ok[k]) mx = max(mx, max(sv[k], dv[k]));
            }
            c += ok[k] ? 1u : 0u;
        }
        kept += c;
        if (COMPACT) {
            if (threadIdx.x == 0) s_cnt = 0;
            __syncthreads();
            uint32_t x = c;  // inclusive warp scan of the per-thread counts
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
                if (lane >= (uint32_t)o) x += y;
            }
            uint32_t wbase = 0;
            if (lane == 31) wbase = atomicAdd(&s_cnt, x);
            wbase = __shfl_sync(0xFFFFFFFFu, wbase, 31);
            __syncthreads();
            if (threadIdx.x == 0) s_base = atomicAdd(cursor, (unsigned long long)s_cnt * per);
            __syncthreads();
            uint64_t pos = s_base + (uint64_t)(wbase + x - c) * per;
#pragma unroll
            for (int k = 0; k < kKeyItems; ++k) {
                if (!ok[k]) continue;
                keys[pos] = ((uint64_t)sv[k] << sh) | dv[k];
                if (symmetric) keys[pos + 1] = ((uint64_t)dv[k] << sh) | sv[k];
                pos += per;
            }
            __syncthreads();  // s_cnt / s_base are reused by the next round
        } else {
#pragma unroll
            for (int k = 0; k < kKeyItems; ++k) {
                const uint64_t i = b0 + (uint64_t)k * kKeyThreads + threadIdx.x;
                if (i >= n) continue;
                const uint64_t j = (first + i) * per;
                keys[j] = ok[k] ? (((uint64_t)sv[k] << sh) | dv[k]) : ~0ull;
                if (symmetric) keys[j + 1] = ok[k] ? (((uint64_t)dv[k] << sh) | sv[k]) : ~0ull;
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mx = max(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
        bad |= __shfl_xor_sync(0xFFFFFFFFu, bad, o);
        kept += __shfl_xor_sync(0xFFFFFFFFu, kept, o);
    }
    if (lane == 0) {
        if (kept) {
            atomicMax(max_id, mx);
            atomicAdd(nkept, (unsigned long long)kept);
        }
        if (bad) atomicOr(range_err, 1u);
    }
}

// First index in [lo, hi) with beg[idx] > t (hi if none), found by one warp
// with 32 probes per round.  Every lane returns the same value.
__device__ uint64_t warp_upper_bound(const uint64_t *beg, uint64_t lo, uint64_t hi, uint64_t t)
{
    const uint32_t lane = threadIdx.x & 31u;
    while (hi - lo > 32) {
        const uint64_t len = hi - lo;
        const uint64_t q = lo + len * (lane + 1) / 33;  // strictly increasing, all < hi
        const unsigned m = __ballot_sync(0xFFFFFFFFu, beg[q] > t);
        const uint64_t qprev = __shfl_up_sync(0xFFFFFFFFu, q, 1);
        if (m == 0) {
            lo = __shfl_sync(0xFFFFFFFFu, q, 31) + 1;
        } else {
            const int f = __ffs(m) - 1;
            const uint64_t qf = __shfl_sync(0xFFFFFFFFu, q, f);
            const uint64_t qb = __shfl_sync(0xFFFFFFFFu, qprev, f);
            hi = qf;
            lo = f == 0 ? lo : qb + 1;
        }
    }
    const uint64_t q = lo + lane;
    const unsigned m = __ballot_sync(0xFFFFFFFFu, q < hi && beg[q] > t);
    return m ? lo + (uint64_t)(__ffs(m) - 1) : hi;
}

// The reference splitter (preprocess/split.hpp:15-87) over nv = nverts + 1
// offsets, one warp.  The reference checks every v in order; here each
// round finds the next v that meets either rule by search: the edge rule
// first holds at the first v with beg[v] > rd_edges + max_nedges, the vertex
// rule at max(v, cur_pos + max_nverts); the edge rule wins a tie, as in the
// reference's if / else-if.  Writes at most cap+1 split points, counts all.
__global__ void k_split_reference(const uint64_t *beg, uint64_t nv, uint64_t max_nedges, uint64_t max_nverts,
                                  uint32_t cap, uint32_t *vb, uint64_t *eb, uint32_t *count)
{
    if (threadIdx.x >= 32) return;
    const uint32_t lane = threadIdx.x;
    uint64_t cur_pos = 0, rd_edges = 0, v = 0, nb = 0;
    if (lane == 0) {
        vb[0] = 0;
        eb[0] = 0;
    }
    while (v < nv) {
        const uint64_t ve = warp_upper_bound(beg, v, nv, rd_edges + max_nedges);
        const uint64_t vv = max(v, cur_pos + max_nverts);
        if (ve >= nv && vv >= nv) break;
        uint64_t cut;
        if (vv < ve) {
            cut = vv;
            v = vv + 1;
        } else {
            cut = ve - 1;
            v = ve + 1;
        }
        cur_pos = cut;
        rd_edges = beg[cut];
        ++nb;
        if (lane == 0 && nb <= cap) {
            vb[nb] = (uint32_t)cut;
            eb[nb] = rd_edges;
        }
    }
    ++nb;
    if (lane == 0) {
        if (nb <= cap) {
            vb[nb] = (uint32_t)(nv - 1);
            eb[nb] = beg[nv - 1];
        }
        *count = (uint32_t)min(nb, (uint64_t)0xFFFFFFFFu);
    }
}

// Equal-edge-mass split: thread k < nblocks-1 finds the first vertex
// v < V with beg[v] >= floor((k+1)*E/nblocks) (V if none), clipped to
// [1, V-1]; thread 0 then makes the cut list non-decreasing.
__global__ void k_split_equal(const uint64_t *beg, uint32_t V, uint32_t nblocks, uint32_t *vb, uint64_t *eb)
{
    const uint64_t E = beg[V];
    const uint32_t hi_clip = V > 1 ? V - 1 : 1;
    for (uint32_t k = threadIdx.x; k + 1 < nblocks; k += blockDim.x) {
        const uint64_t t = (uint64_t)((unsigned __int128)(k + 1) * E / nblocks);
        uint64_t lo = 0, hi = V;  // lower bound over beg[0, V)
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (beg[mid] < t) lo = mid + 1;
            else hi = mid;
        }
        vb[k + 1] = (uint32_t)(lo < 1 ? 1 : (lo > hi_clip ? hi_clip : lo));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        vb[0] = 0;
        vb[nblocks] = V;
        uint32_t run = 0;
        for (uint32_t k = 0; k <= nblocks; ++k) {
            run = max(run, vb[k]);
            vb[k] = run;
            eb[k] = beg[run];
        }
    }
}

// offsets + neighbour ids from n sorted keys src << sh | dst (sources <
// nverts).  Allocates *beg_out and *csr_out; s is synchronised before return.
static cudaError_t csr_from_sorted(const uint64_t *keys, uint64_t n, uint32_t sh, uint32_t nverts, cudaStream_t s,
                                   uint64_t **beg_out, uint32_t **csr_out)
{
    unsigned long long *cnt = nullptr;
    uint64_t *beg = nullptr;
    uint32_t *csr = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    const uint64_t nb = (uint64_t)nverts + 1;
    cudaError_t e;
    do {
        if ((e = cudaMalloc(&cnt, nb * sizeof(uint64_t))) != cudaSuccess) break;
        if ((e = cudaMalloc(&beg, nb * sizeof(uint64_t))) != cudaSuccess) break;
        if ((e = cudaMalloc(&csr, (n ? n : 1) * sizeof(uint32_t))) != cudaSuccess) break;
        if ((e = cudaMemsetAsync(cnt, 0, nb * sizeof(uint64_t), s)) != cudaSuccess) break;
        if (n) {
            k_runs<<<148 * 16, 256, 0, s>>>(keys, n, sh, cnt, csr);
            if ((e = cudaGetLastError()) != cudaSuccess) break;
        }
        if ((e = cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, (const uint64_t *)cnt, beg, nb, s)) != cudaSuccess)
            break;
        if ((e = cudaMalloc(&tmp, tmp_bytes)) != cudaSuccess) break;
        if ((e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, (const uint64_t *)cnt, beg, nb, s)) != cudaSuccess)
            break;
        e = cudaStreamSynchronize(s);
    } while (0);
    cudaFree(cnt);
    cudaFree(tmp);
    if (e != cudaSuccess) {
        cudaFree(beg);
        cudaFree(csr);
        return e;
    }
    *beg_out = beg;
    *csr_out = csr;
    return cudaSuccess;
}

static inline uint32_t bit_length32(uint32_t x) { return x ? 32u - (uint32_t)__builtin_clz(x) : 0u; }

static bool device_accessible(const void *p)
{
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Phase times of a conversion on stderr when GOWALKER_TRACE is set (each mark
// synchronises the stream, so tracing slows the call down).
struct PhaseTrace {
    bool on;
    cudaStream_t s;
    std::chrono::steady_clock::time_point t0;
    explicit PhaseTrace(cudaStream_t st) : s(st)
    {
        const char *e = getenv("GOWALKER_TRACE");
        on = e && *e && *e != '0';
        t0 = std::chrono::steady_clock::now();
    }
    void mark(const char *what)
    {
        if (!on) return;
        cudaStreamSynchronize(s);
        const auto t = std::chrono::steady_clock::now();
        fprintf(stderr, "[gowalker] gw_edges_csr %-10s %9.3f ms\n", what,
                std::chrono::duration<double, std::milli>(t - t0).count());
        t0 = t;
    }
};

// Sampled edge list -> CSR: count the kept keys, write them compacted and
// packed (src << bit_length(nverts-1) | dst), radix-sort, drop repeats, thin
// evenly to target_edges when given, then offsets and neighbour ids.
template <class Sampler>
static int sampled_csr(const Sampler &smp, uint64_t nsamples, uint32_t nverts, bool symmetric, uint64_t target_edges,
                       uint64_t **d_beg, uint32_t **d_csr, uint64_t *nedges)
{
    cudaStream_t s = 0;
    const uint32_t sh = bit_length32(nverts - 1);
    const int blocks = 148 * 8;
    uint64_t *keys = nullptr, *alt = nullptr, *beg = nullptr;
    uint32_t *csr = nullptr;
    unsigned long long *d_cur = nullptr, h_cur = 0;
    int64_t *d_nsel = nullptr, nsel = 0;
    void *tmp = nullptr;
    size_t tmp_bytes = 0, tb2 = 0;
    uint64_t U = 0;
    int rc = GW_OK;
    cudaError_t e = cudaSuccess;
#define SC_CHECK(x)                       \
    do {                                  \
        if ((e = (x)) != cudaSuccess) {   \
            rc = GW_ERR_CUDA;             \
            goto out;                     \
        }                                 \
    } while (0)
    SC_CHECK(cudaMalloc(&d_cur, sizeof(unsigned long long)));
    SC_CHECK(cudaMalloc(&d_nsel, sizeof(int64_t)));
    SC_CHECK(cudaMemsetAsync(d_cur, 0, sizeof(unsigned long long), s));
    k_sample_keys<Sampler, true><<<blocks, 256, 0, s>>>(smp, nsamples, sh, symmetric ? 1 : 0, nullptr, d_cur);
    SC_CHECK(cudaGetLastError());
    SC_CHECK(cudaMemcpyAsync(&h_cur, d_cur, sizeof(h_cur), cudaMemcpyDeviceToHost, s));
    SC_CHECK(cudaStreamSynchronize(s));
    U = h_cur;
    SC_CHECK(cudaMalloc(&keys, (U ? U : 1) * sizeof(uint64_t)));
    SC_CHECK(cudaMalloc(&alt, (U ? U : 1) * sizeof(uint64_t)));
    SC_CHECK(cudaMemsetAsync(d_cur, 0, sizeof(unsigned long long), s));
    k_sample_keys<Sampler, false><<<blocks, 256, 0, s>>>(smp, nsamples, sh, symmetric ? 1 : 0, keys, d_cur);
    SC_CHECK(cudaGetLastError());
    if (U) {
        cub::DoubleBuffer<uint64_t> db(keys, alt);
        const int b1 = (int)(2 * sh);
        SC_CHECK(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, db, U, 0, b1, s));
        SC_CHECK(cub::DeviceSelect::Unique(nullptr, tb2, keys, alt, d_nsel, (int64_t)U, s));
        tmp_bytes = std::max(tmp_bytes, tb2);
        SC_CHECK(cudaMalloc(&tmp, tmp_bytes));
        SC_CHECK(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, db, U, 0, b1, s));
        keys = db.Current();
        alt = db.Alternate();
        SC_CHECK(cub::DeviceSelect::Unique(tmp, tmp_bytes, keys, alt, d_nsel, (int64_t)U, s));
        SC_CHECK(cudaMemcpyAsync(&nsel, d_nsel, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        SC_CHECK(cudaStreamSynchronize(s));
        std::swap(keys, alt);
        U = (uint64_t)nsel;
    }
    if (target_edges > 0) {
        if (U < target_edges) {
            rc = GW_ERR_ARG;  // too few unique edges: sample more
            goto out;
        }
        if (U > target_edges) {
            k_thin<<<blocks * 2, 256, 0, s>>>(keys, U, U - target_edges, alt);
            SC_CHECK(cudaGetLastError());
            std::swap(keys, alt);
            U = target_edges;
        }
    }
    SC_CHECK(csr_from_sorted(keys, U, sh, nverts, s, &beg, &csr));
    *d_beg = beg;
    *d_csr = csr;
    *nedges = U;
    beg = nullptr;
    csr = nullptr;
out:
#undef SC_CHECK
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (e == cudaErrorMemoryAllocation) rc = GW_ERR_NOMEM;
    }
    cudaFree(keys);
    cudaFree(alt);
    cudaFree(tmp);
    cudaFree(d_cur);
    cudaFree(d_nsel);
    cudaFree(beg);
    cudaFree(csr);
    return rc;
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
    const RmatSampler smp{scale, nverts, thr[0], thr[1], thr[2], (uint32_t)seed, (uint32_t)(seed >> 32)};
    return sampled_csr(smp, nsamples, nverts, symmetric != 0, target_edges, d_beg, d_csr, nedges);
}

extern "C" int gw_web_csr(uint32_t scale, uint32_t nverts, const uint32_t thr[3], double dmin, double tail,
                          uint32_t max_degree, uint32_t local_permille, uint32_t window, uint64_t seed,
                          uint64_t target_edges, uint64_t **d_beg, uint32_t **d_csr, uint64_t *nedges)
{
    if (!thr || !d_beg || !d_csr || !nedges || scale == 0 || scale > 32 || nverts < 2) return GW_ERR_ARG;
    if (local_permille > 1000 || window == 0 || window > (1u << 30) || max_degree == 0) return GW_ERR_ARG;
    if (!(dmin >= 1.0 && dmin <= 1e9) || !(tail >= 0.05 && tail <= 100.0)) return GW_ERR_ARG;
    const WebParams p{nverts, scale, thr[0], thr[1], thr[2], (uint32_t)seed, (uint32_t)(seed >> 32),
                      local_permille, window, max_degree, dmin, tail};
    cudaStream_t s = 0;
    const uint64_t nb = (uint64_t)nverts + 1;
    const uint32_t sh = bit_length32(nverts - 1), bsrc = bit_length32(nverts);
    unsigned long long *deg = nullptr, *estart = nullptr;
    uint64_t *keys = nullptr, *alt = nullptr, *beg = nullptr;
    uint32_t *csr = nullptr;
    int64_t *d_nsel = nullptr, nsel = 0;
    void *tmp = nullptr;
    size_t tmp_bytes = 0, tb2 = 0;
    uint64_t M = 0, U = 0;
    int rc = GW_OK;
    cudaError_t e = cudaSuccess;
#define WB_CHECK(x)                       \
    do {                                  \
        if ((e = (x)) != cudaSuccess) {   \
            rc = GW_ERR_CUDA;             \
            goto out;                     \
        }                                 \
    } while (0)
    WB_CHECK(cudaMalloc(&deg, nb * sizeof(unsigned long long)));
    WB_CHECK(cudaMalloc(&estart, nb * sizeof(unsigned long long)));
    WB_CHECK(cudaMalloc(&d_nsel, sizeof(int64_t)));
    k_web_degrees<<<148 * 8, 256, 0, s>>>(p, deg);
    WB_CHECK(cudaGetLastError());
    WB_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, deg, estart, nb, s));
    WB_CHECK(cudaMalloc(&tmp, tmp_bytes));
    WB_CHECK(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, deg, estart, nb, s));
    WB_CHECK(cudaMemcpyAsync(&M, estart + nverts, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    WB_CHECK(cudaStreamSynchronize(s));
    cudaFree(tmp);
    tmp = nullptr;
    cudaFree(deg);
    deg = nullptr;
    WB_CHECK(cudaMalloc(&keys, (M ? M : 1) * sizeof(uint64_t)));
    WB_CHECK(cudaMalloc(&alt, (M ? M : 1) * sizeof(uint64_t)));
    k_web_edges<<<148 * 16, 128, 0, s>>>(p, estart, sh, keys);
    WB_CHECK(cudaGetLastError());
    if (M) {
        cub::DoubleBuffer<uint64_t> db(keys, alt);
        const int b1 = (int)(sh + bsrc);  // the marker's bits there are all ones: it sorts last
        WB_CHECK(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, db, M, 0, b1, s));
        WB_CHECK(cub::DeviceSelect::Unique(nullptr, tb2, keys, alt, d_nsel, (int64_t)M, s));
        tmp_bytes = std::max(tmp_bytes, tb2);
        WB_CHECK(cudaMalloc(&tmp, tmp_bytes));
        WB_CHECK(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, db, M, 0, b1, s));
        keys = db.Current();
        alt = db.Alternate();
        WB_CHECK(cub::DeviceSelect::Unique(tmp, tmp_bytes, keys, alt, d_nsel, (int64_t)M, s));
        WB_CHECK(cudaMemcpyAsync(&nsel, d_nsel, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        WB_CHECK(cudaStreamSynchronize(s));
        std::swap(keys, alt);
        U = (uint64_t)nsel;
        if (U) {
            uint64_t last = 0;
            WB_CHECK(cudaMemcpy(&last, keys + (U - 1), sizeof(uint64_t), cudaMemcpyDeviceToHost));
            if (last == ~0ull) U -= 1;
        }
    }
    if (target_edges > 0) {
        if (U < target_edges) {
            rc = GW_ERR_ARG;
            goto out;
        }
        if (U > target_edges) {
            k_thin<<<148 * 16, 256, 0, s>>>(keys, U, U - target_edges, alt);
            WB_CHECK(cudaGetLastError());
            std::swap(keys, alt);
            U = target_edges;
        }
    }
    WB_CHECK(csr_from_sorted(keys, U, sh, nverts, s, &beg, &csr));
    *d_beg = beg;
    *d_csr = csr;
    *nedges = U;
    beg = nullptr;
    csr = nullptr;
out:
#undef WB_CHECK
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (e == cudaErrorMemoryAllocation) rc = GW_ERR_NOMEM;
    }
    cudaFree(deg);
    cudaFree(estart);
    cudaFree(keys);
    cudaFree(alt);
    cudaFree(tmp);
    cudaFree(d_nsel);
    cudaFree(beg);
    cudaFree(csr);
    return rc;
}

extern "C" int gw_edges_csr(const uint32_t *src, const uint32_t *dst, uint64_t n, uint32_t nverts, uint32_t flags,
                            uint64_t **d_beg, uint32_t **d_csr, uint64_t *nedges, uint32_t *nverts_out)
{
    if (!d_beg || !d_csr || !nedges || (n && (!src || !dst))) return GW_ERR_ARG;
    if (flags & ~(GW_EDGES_SYMMETRIC | GW_EDGES_SORT | GW_EDGES_DEDUP)) return GW_ERR_ARG;
    const bool symmetric = flags & GW_EDGES_SYMMETRIC;
    const bool dedup = flags & GW_EDGES_DEDUP;
    const bool sorted = dedup || (flags & GW_EDGES_SORT);
    if (n > (symmetric ? (1ull << 62) : (1ull << 63)) / sizeof(uint64_t)) return GW_ERR_ARG;
    const uint64_t m = n * (symmetric ? 2 : 1);
    int rc = GW_OK;
    cudaStream_t s = 0;
    PhaseTrace trace(s);
    uint64_t *keys = nullptr, *alt = nullptr, *beg = nullptr;
    uint32_t *csr = nullptr, *stage = nullptr;
    unsigned int *d_max = nullptr, *d_err = nullptr;
    unsigned long long *d_cnt = nullptr;  // [0] kept edges, [1] compaction cursor
    int64_t *d_nsel = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0, tb2 = 0;
    unsigned int h_max = 0, h_err = 0;
    unsigned long long h_kept = 0;
    uint64_t U = 0;
    uint32_t V = nverts, sh = 32;
    const uint32_t lim = nverts ? nverts : 0xFFFFFFFFu;
    const int threads = kKeyThreads;
    int blocks = 148 * 8;
    // Host inputs are staged in chunks; device (or managed) inputs are read in place.
    const bool in_place = n == 0 || (device_accessible(src) && device_accessible(dst));
    const uint64_t chunk = in_place ? (n ? n : 1) : std::min<uint64_t>(n, 1ull << 26);
    // Sorted output: compacted keys, packed as src << bit_length(nverts-1) | dst
    // when nverts is given (otherwise repacked once the largest id is known).
    if (sorted && nverts) sh = bit_length32(nverts - 1);

    GEN_CHECK(cudaMalloc(&keys, (m ? m : 1) * sizeof(uint64_t)));
    GEN_CHECK(cudaMalloc(&alt, (m ? m : 1) * sizeof(uint64_t)));
    GEN_CHECK(cudaMalloc(&d_max, 2 * sizeof(unsigned int)));
    GEN_CHECK(cudaMalloc(&d_cnt, 2 * sizeof(unsigned long long)));
    GEN_CHECK(cudaMalloc(&d_nsel, sizeof(int64_t)));
    d_err = d_max + 1;
    GEN_CHECK(cudaMemsetAsync(d_max, 0, 2 * sizeof(unsigned int), s));
    GEN_CHECK(cudaMemsetAsync(d_cnt, 0, 2 * sizeof(unsigned long long), s));
    if (!in_place) GEN_CHECK(cudaMalloc(&stage, 2 * chunk * sizeof(uint32_t)));
    trace.mark("alloc");
    for (uint64_t i0 = 0; i0 < n; i0 += chunk) {
        const uint64_t k = std::min(chunk, n - i0);
        const uint32_t *ps = src + i0, *pd = dst + i0;
        if (!in_place) {
            GEN_CHECK(cudaMemcpyAsync(stage, src + i0, k * sizeof(uint32_t), cudaMemcpyDefault, s));
            GEN_CHECK(cudaMemcpyAsync(stage + chunk, dst + i0, k * sizeof(uint32_t), cudaMemcpyDefault, s));
            ps = stage;
            pd = stage + chunk;
        }
        const uint64_t need = (k + (uint64_t)kKeyThreads * kKeyItems - 1) / ((uint64_t)kKeyThreads * kKeyItems);
        blocks = (int)std::min<uint64_t>(need ? need : 1, 148 * 8);
        if (sorted)
            k_edge_keys<true><<<blocks, threads, 0, s>>>(ps, pd, k, i0, lim, sh, symmetric ? 1 : 0, keys, d_cnt + 1,
                                                         d_max, d_cnt, d_err);
        else
            k_edge_keys<false><<<blocks, threads, 0, s>>>(ps, pd, k, i0, lim, sh, symmetric ? 1 : 0, keys, d_cnt + 1,
                                                          d_max, d_cnt, d_err);
        GEN_CHECK(cudaGetLastError());
    }
    GEN_CHECK(cudaMemcpyAsync(&h_max, d_max, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
    GEN_CHECK(cudaMemcpyAsync(&h_err, d_err, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
    GEN_CHECK(cudaMemcpyAsync(&h_kept, d_cnt, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    GEN_CHECK(cudaStreamSynchronize(s));
    trace.mark("keys");
    if (h_err) {
        rc = GW_ERR_ARG;
        goto done;
    }
    if (!nverts) V = h_kept ? h_max + 1 : 0;
    U = h_kept * (symmetric ? 2 : 1);
    if (U) {
        int b0, b1;
        if (sorted) {
            // compacted: U keys, no markers; sort the packed source and destination bits
            const uint32_t bv = bit_length32(V - 1);
            if (sh != bv) {
                k_repack<<<148 * 8, 256, 0, s>>>(keys, U, bv);
                GEN_CHECK(cudaGetLastError());
                sh = bv;
            }
            b0 = 0;
            b1 = (int)(sh + bv);
        } else {
            // fixed positions: sort m keys by source only; markers end up last
            b0 = 32;
            b1 = 32 + (int)bit_length32(V);
        }
        const uint64_t nsort = sorted ? U : m;
        cub::DoubleBuffer<uint64_t> db(keys, alt);
        GEN_CHECK(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, db, nsort, b0, b1, s));
        if (dedup) {
            GEN_CHECK(cub::DeviceSelect::Unique(nullptr, tb2, keys, alt, d_nsel, (int64_t)U, s));
            tmp_bytes = std::max(tmp_bytes, tb2);
        }
        GEN_CHECK(cudaMalloc(&tmp, tmp_bytes));
        GEN_CHECK(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, db, nsort, b0, b1, s));
        keys = db.Current();
        alt = db.Alternate();
        trace.mark("sort");
        if (dedup) {
            int64_t nsel = 0;
            GEN_CHECK(cub::DeviceSelect::Unique(tmp, tmp_bytes, keys, alt, d_nsel, (int64_t)U, s));
            GEN_CHECK(cudaMemcpyAsync(&nsel, d_nsel, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
            GEN_CHECK(cudaStreamSynchronize(s));
            std::swap(keys, alt);
            U = (uint64_t)nsel;
            trace.mark("unique");
        }
    }
    GEN_CHECK(csr_from_sorted(keys, U, sh, V, s, &beg, &csr));
    trace.mark("csr");
    *d_beg = beg;
    *d_csr = csr;
    *nedges = U;
    if (nverts_out) *nverts_out = V;
    beg = nullptr;
    csr = nullptr;
done:
    cudaFree(keys);
    cudaFree(alt);
    cudaFree(stage);
    cudaFree(tmp);
    cudaFree(d_max);
    cudaFree(d_cnt);
    cudaFree(d_nsel);
    cudaFree(beg);
    cudaFree(csr);
    trace.mark("free");
    return rc;
}

extern "C" int gw_split_blocks(const uint64_t *beg, uint32_t nverts, uint32_t mode, uint64_t param,
                               uint32_t *vblocks, uint64_t *eblocks, uint32_t cap, uint32_t *nblocks)
{
    if (!beg || !vblocks || !eblocks || !nblocks || cap == 0xFFFFFFFFu) return GW_ERR_ARG;
    if (mode != GW_SPLIT_REFERENCE && mode != GW_SPLIT_EQUAL_EDGES) return GW_ERR_ARG;
    if (mode == GW_SPLIT_EQUAL_EDGES && (param < 1 || param > nverts)) return GW_ERR_ARG;
    int rc = GW_OK;
    cudaStream_t s = 0;
    const uint64_t nv = (uint64_t)nverts + 1;
    const uint64_t *d_beg = beg;
    uint64_t *own = nullptr, *d_eb = nullptr;
    uint32_t *d_vb = nullptr, *d_count = nullptr;
    uint64_t b0 = 0;
    uint32_t count = 0;
    const uint64_t slots = mode == GW_SPLIT_EQUAL_EDGES ? param + 1 : (uint64_t)cap + 1;
    if (!device_accessible(beg)) {
        GEN_CHECK(cudaMalloc(&own, nv * sizeof(uint64_t)));
        GEN_CHECK(cudaMemcpy(own, beg, nv * sizeof(uint64_t), cudaMemcpyDefault));
        d_beg = own;
    }
    GEN_CHECK(cudaMemcpy(&b0, d_beg, sizeof(uint64_t), cudaMemcpyDefault));
    if (b0 != 0) {
        rc = GW_ERR_ARG;
        goto done;
    }
    GEN_CHECK(cudaMalloc(&d_vb, slots * sizeof(uint32_t)));
    GEN_CHECK(cudaMalloc(&d_eb, slots * sizeof(uint64_t)));
    GEN_CHECK(cudaMalloc(&d_count, sizeof(uint32_t)));
    if (mode == GW_SPLIT_REFERENCE) {
        k_split_reference<<<1, 32, 0, s>>>(d_beg, nv, param / sizeof(uint32_t), param / sizeof(uint64_t), cap, d_vb,
                                           d_eb, d_count);
        GEN_CHECK(cudaGetLastError());
        GEN_CHECK(cudaMemcpyAsync(&count, d_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        GEN_CHECK(cudaStreamSynchronize(s));
    } else {
        count = (uint32_t)param;
        k_split_equal<<<1, 1024, 0, s>>>(d_beg, nverts, count, d_vb, d_eb);
        GEN_CHECK(cudaGetLastError());
        GEN_CHECK(cudaStreamSynchronize(s));
    }
    *nblocks = count;
    if (count > cap) {
        rc = GW_ERR_ARG;
        goto done;
    }
    GEN_CHECK(cudaMemcpy(vblocks, d_vb, ((uint64_t)count + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    GEN_CHECK(cudaMemcpy(eblocks, d_eb, ((uint64_t)count + 1) * sizeof(uint64_t), cudaMemcpyDeviceToHost));
done:
    cudaFree(own);
    cudaFree(d_vb);
    cudaFree(d_eb);
    cudaFree(d_count);
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

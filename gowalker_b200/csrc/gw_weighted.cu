// Weighted Node2vec walks, in-core (GW has no counterpart: the reference loads
// edge weights, engine/cache.hpp:71, gpu/memory.hpp:134-137, and never samples
// with them).
//
// Semantics: from cur (with prev), candidate x is drawn in proportion to the
// weight of cur -> x, then accepted by the unweighted rule (1/p if x == prev,
// 1 if x is a neighbour of prev, 1/q otherwise, with the reference's
// thresholds and precision, engine/engine.hpp:209-258): P(x) is proportional
// to w(cur, x) times the Node2vec bias, the usual weighted Node2vec.
// The candidate comes from Walker's alias table of cur's out-edges: column
// i = lane x % deg of the trial's draw (the unweighted rand_pos), coin =
// float(lane w >> 8) * 2^-24; the trial takes column i when coin < prob[i],
// its alias otherwise.  Lanes y (rand value) and z (termination) keep their
// meaning, so a graph whose weights are all equal walks exactly as unweighted.
//
// Alias tables (Vose's method, per vertex, one thread each): the weights are
// summed in double in index order, scaled to p_i = w_i * deg / sum, split
// into a queue of p < 1 and a queue of p >= 1 in index order; repeatedly the
// next small s takes the front large l as its alias (prob[s] = (float)p_s)
// and p_l = (p_l + p_s) - 1, l moving to the back of the small queue when it
// drops below 1; leftovers get probability 1.  Every operation is an IEEE
// double rounded to nearest, so the oracle's C restatement builds the same
// table bit for bit.
#include <cuda_runtime.h>
#include <cstdint>
#include "gw_kernels.cuh"
#include "gw_step.cuh"
#include "gw_weighted.cuh"

namespace gw {

__global__ void k_build_alias(const uint64_t *__restrict__ beg, const float *__restrict__ w, uint32_t nverts,
                              double *__restrict__ pd, uint32_t *__restrict__ qs, uint32_t *__restrict__ ql,
                              AliasEntry *__restrict__ out, uint32_t *err)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nverts; v += stride) {
        const uint64_t h = beg[v], d = beg[v + 1] - h;
        if (d == 0) continue;
        double sum = 0.0;
        bool bad = false;
        for (uint64_t i = 0; i < d; ++i) {
            const float wi = w[h + i];
            bad |= !(wi > 0.f && wi < __int_as_float(0x7F800000));
            sum = __dadd_rn(sum, (double)wi);
        }
        if (bad) {
            atomicOr(err, kErrWeight);
            for (uint64_t i = 0; i < d; ++i) out[h + i] = AliasEntry{1.f, (uint32_t)i};
            continue;
        }
        double *p = pd + h;
        uint32_t *small = qs + h, *large = ql + h;
        uint64_t ns = 0, nl = 0, hs = 0, hl = 0;
        for (uint64_t i = 0; i < d; ++i) {
            p[i] = __ddiv_rn(__dmul_rn((double)w[h + i], (double)d), sum);
            if (p[i] < 1.0) small[ns++] = (uint32_t)i;
            else large[nl++] = (uint32_t)i;
        }
        while (hs < ns && hl < nl) {
            const uint32_t sidx = small[hs++], lidx = large[hl];
            out[h + sidx] = AliasEntry{__double2float_rn(p[sidx]), lidx};
            p[lidx] = __dsub_rn(__dadd_rn(p[lidx], p[sidx]), 1.0);
            if (p[lidx] < 1.0) {
                ++hl;
                small[ns++] = lidx;
            }
        }
        while (hl < nl) {
            const uint32_t lidx = large[hl++];
            out[h + lidx] = AliasEntry{1.f, lidx};
        }
        while (hs < ns) {
            const uint32_t sidx = small[hs++];
            out[h + sidx] = AliasEntry{1.f, sidx};
        }
    }
}

// One walker per thread, grid-stride over the walker ids; the oracle's step
// loop (oracle/gw_oracle.c walk_from) with the alias draw.
template <bool PATHS>
__global__ void __launch_bounds__(256) k_walk_weighted(const __grid_constant__ IncoreArgs a,
                                                       const AliasEntry *__restrict__ al)
{
    const uint64_t *__restrict__ beg = a.beg;
    const uint32_t *__restrict__ csr = a.ix.csr;
    const uint32_t maxhops = a.c.maxhops;
    const StepThr t{0.f, 0.f, 0.f};
    const float maxv = a.c.n2v_maxv;
    unsigned long long steps = 0, trials = 0, done = 0, hsum = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.nwalkers; i += stride) {
        const uint32_t wid = a.wid_base + (uint32_t)i * a.wid_stride;
        const uint32_t src = walker_source(a.init, wid);
        uint32_t prev = src, cur = src, hop = 0, moves = 0;
        uint64_t h = hash_init(src);
        if (PATHS) a.paths[(uint64_t)wid * a.stride] = src;
        if (src >= a.nverts) {
            atomicOr(a.err, kErrSource);
            hop = maxhops;
        }
        while (hop < maxhops) {
            if (hop > 0 && a.c.term_prob > 0.f && terminates(a.c, draw(a.c, wid, hop, 0).z)) break;
            const uint64_t head = __ldg(beg + cur), deg = __ldg(beg + cur + 1) - head;
            if (deg == 0) break;  // dead end (engine/engine.hpp:196-199)
            const uint64_t phead = __ldg(beg + prev);
            const uint32_t pdeg = (uint32_t)(__ldg(beg + prev + 1) - phead);
            uint32_t attempt = 0, x = 0;
            bool ok = false;
            while (attempt < kMaxAttempts) {
                const U4 r = draw(a.c, wid, hop, attempt);
                ++attempt;
                const uint64_t pos = (uint64_t)r.x % deg;
                const uint2 e = __ldg(reinterpret_cast<const uint2 *>(al + head + pos));
                const float coin = __uint2float_rn(r.w >> 8) * 0x1p-24f;
                const uint64_t col = coin < __uint_as_float(e.x) ? pos : (uint64_t)e.y;
                x = __ldg(csr + head + col);
                if (accept_candidate<false>(a.c, t, rand_val(r.y, maxv), x, prev, cur, a.ix, phead, pdeg)) {
                    ok = true;
                    break;
                }
            }
            trials += attempt;
            if (!ok) {
                atomicOr(a.err, kErrTrials);
                break;
            }
            if (x >= a.nverts) {
                atomicOr(a.err, kErrVertexRange);
                break;
            }
            prev = cur;
            cur = x;
            ++hop;
            ++moves;
            h = hash_step(h, x);
            if (PATHS) a.paths[(uint64_t)wid * a.stride + moves] = x;
        }
        a.hashes[wid] = h;
        a.lens[wid] = moves + 1;
        steps += moves;
        done += 1;
        hsum += h;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        steps += __shfl_xor_sync(0xFFFFFFFFu, steps, o);
        trials += __shfl_xor_sync(0xFFFFFFFFu, trials, o);
        done += __shfl_xor_sync(0xFFFFFFFFu, done, o);
        hsum += __shfl_xor_sync(0xFFFFFFFFu, hsum, o);
    }
    if ((threadIdx.x & 31u) == 0 && done) {
        atomicAdd(&a.ctr[kCtrSteps], steps);
        atomicAdd(&a.ctr[kCtrTrials], trials);
        atomicAdd(&a.ctr[kCtrDone], done);
        atomicAdd(&a.ctr[kCtrHashSum], hsum);
    }
}

cudaError_t launch_build_alias(const uint64_t *beg, const float *w, uint32_t nverts, double *pd, uint32_t *qs,
                               uint32_t *ql, AliasEntry *out, uint32_t *err, int num_sms, cudaStream_t s)
{
    k_build_alias<<<num_sms * 8, 128, 0, s>>>(beg, w, nverts, pd, qs, ql, out, err);
    return cudaGetLastError();
}

cudaError_t launch_walk_weighted(const IncoreArgs &a, const AliasEntry *al, int num_sms, cudaStream_t s)
{
    const int grid = num_sms * 8;
    if (a.paths) k_walk_weighted<true><<<grid, 256, 0, s>>>(a, al);
    else k_walk_weighted<false><<<grid, 256, 0, s>>>(a, al);
    return cudaGetLastError();
}

}  // namespace gw

// Weighted Node2vec walks, in-core (the reference has no counterpart: it loads
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
// The walk itself is the in-core kernel (gw_walk.cu) with its W flag; this
// file builds the alias tables.
//
// Alias tables (Vose's method, per vertex: one thread each, a CTA for each
// vertex above 256 neighbours, below): the weights are
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
#include "gw_weighted.cuh"

namespace gw {

constexpr uint64_t kHubDeg = 256;  // vertices above this degree get a CTA each

// Vose's loop for one vertex whose probabilities p[0, d) are scaled; the
// queues hold indices in the order they are pushed.  p and the queues may be
// shared or global memory.
__device__ void vose_loop(uint64_t d, double *p, uint32_t *small, uint32_t *large, AliasEntry *out)
{
    uint64_t ns = 0, nl = 0, hs = 0, hl = 0;
    for (uint64_t i = 0; i < d; ++i) {
        if (p[i] < 1.0) small[ns++] = (uint32_t)i;
        else large[nl++] = (uint32_t)i;
    }
    while (hs < ns && hl < nl) {
        const uint32_t sidx = small[hs++], lidx = large[hl];
        out[sidx] = AliasEntry{__double2float_rn(p[sidx]), lidx};
        p[lidx] = __dsub_rn(__dadd_rn(p[lidx], p[sidx]), 1.0);
        if (p[lidx] < 1.0) {
            ++hl;
            small[ns++] = lidx;
        }
    }
    while (hl < nl) {
        const uint32_t lidx = large[hl++];
        out[lidx] = AliasEntry{1.f, lidx};
    }
    while (hs < ns) {
        const uint32_t sidx = small[hs++];
        out[sidx] = AliasEntry{1.f, sidx};
    }
}

// Vertices of degree at most kHubDeg: one thread each.
__global__ void k_build_alias(const uint64_t *__restrict__ beg, const float *__restrict__ w, uint32_t nverts,
                              double *__restrict__ pd, uint32_t *__restrict__ qs, uint32_t *__restrict__ ql,
                              AliasEntry *__restrict__ out, uint32_t *err)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nverts; v += stride) {
        const uint64_t h = beg[v], d = beg[v + 1] - h;
        if (d == 0 || d > kHubDeg) continue;
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
        for (uint64_t i = 0; i < d; ++i) pd[h + i] = __ddiv_rn(__dmul_rn((double)w[h + i], (double)d), sum);
        vose_loop(d, pd + h, qs + h, ql + h, out + h);
    }
}

// Vertices of degree above kHubDeg: one CTA each, with every memory access
// of Vose's serial loop sequential so that a warp can fetch it 32 entries
// ahead.  Vose's small queue is the initial smalls (index order) followed by
// the larges that dropped below 1, in the order they dropped; the large queue
// is the initial larges (index order), each one's probability untouched
// until it becomes the current large.  So the loop reads three streams in
// order -- initial smalls, initial larges, and the dropped larges (written
// behind the consumed larges in the same array, each with its residual) --
// and keeps the current large's residual in a register.  The warp runs the
// loop in lockstep (every lane holds the same values; lane 0 writes), so the
// sequence of double operations is exactly Vose's, as in the one-thread path
// and the oracle.  The weight sum is the same in-order chain, fed 32 weights
// at a time; the scaling and the split into the two queues run on the CTA.
// The vertices of degree in (lo, hi], appended to the list work[2 + i]
// (work[0] counts it) that the CTAs of k_build_alias_hubs take one vertex at
// a time from (work[1]): R-MAT hubs sit at ids with many zero bits, so a
// fixed stride would give a few CTAs most of the work.  Listing the largest
// first lets their serial loops start first.
__global__ void k_list_hubs(const uint64_t *__restrict__ beg, uint32_t nverts, uint64_t lo, uint64_t hi,
                            uint32_t *__restrict__ work)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x; b < nverts; b += stride) {
        const uint64_t v = b + threadIdx.x;
        const bool hub = v < nverts && beg[v + 1] - beg[v] > lo && beg[v + 1] - beg[v] <= hi;
        const unsigned m = __ballot_sync(0xFFFFFFFFu, hub);
        uint32_t base = 0;
        if (lane == 0 && m) base = atomicAdd(work, (uint32_t)__popc(m));
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (hub) work[2 + base + __popc(m & ((1u << lane) - 1u))] = (uint32_t)v;
    }
}

__global__ void __launch_bounds__(128)
    k_build_alias_hubs(const uint64_t *__restrict__ beg, const float *__restrict__ w, uint32_t *__restrict__ work,
                       double *__restrict__ pd, uint32_t *__restrict__ qs, uint32_t *__restrict__ ql,
                       AliasEntry *__restrict__ out, uint32_t *err)
{
    __shared__ uint32_t s_next;
    __shared__ double s_sum;
    __shared__ int s_bad;
    __shared__ uint32_t s_cnt[2][4];  // per warp: smalls, larges of the current 128 indices
    __shared__ uint32_t s_tot[2];     // smalls, larges so far
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    constexpr uint32_t kNone = 0xFFFFFFFFu;
    const uint32_t nhubs = work[0];
    for (;;) {
        __syncthreads();  // the previous vertex is done with s_next and the shared sums
        if (threadIdx.x == 0) s_next = atomicAdd(work + 1, 1u);
        __syncthreads();
        if (s_next >= nhubs) break;
        const uint64_t v = work[2 + s_next];
        const uint64_t h = beg[v], d = beg[v + 1] - h;
        if (warp == 0) {
            // the weight sum, one in-order chain of double additions
            double sum = 0.0;
            bool bad = false;
            float wn = lane < d ? w[h + lane] : 1.f;
            for (uint64_t b = 0; b < d; b += 32) {
                const float wc = wn;
                wn = (b + 32 + lane < d) ? w[h + b + 32 + lane] : 1.f;  // the next 32, in flight meanwhile
                bad |= !(wc > 0.f && wc < __int_as_float(0x7F800000));
                const uint32_t n = (uint32_t)min((uint64_t)32, d - b);
                for (uint32_t j = 0; j < n; ++j) sum = __dadd_rn(sum, (double)__shfl_sync(0xFFFFFFFFu, wc, j));
            }
            bad = __any_sync(0xFFFFFFFFu, bad);
            if (lane == 0) {
                s_sum = sum;
                s_bad = bad ? 1 : 0;
                s_tot[0] = s_tot[1] = 0;
            }
        }
        __syncthreads();
        if (s_bad) {
            if (threadIdx.x == 0) atomicOr(err, kErrWeight);
            for (uint64_t i = threadIdx.x; i < d; i += blockDim.x) out[h + i] = AliasEntry{1.f, (uint32_t)i};
            __syncthreads();
            continue;
        }
        // scale, and split the indices into the two queues in index order
        const double sum = s_sum;
        for (uint64_t b = 0; b < d; b += blockDim.x) {
            const uint64_t i = b + threadIdx.x;
            double p = 0.0;
            if (i < d) {
                p = __ddiv_rn(__dmul_rn((double)w[h + i], (double)d), sum);
                pd[h + i] = p;
            }
            const bool sm = i < d && p < 1.0, lg = i < d && !(p < 1.0);
            const unsigned bs = __ballot_sync(0xFFFFFFFFu, sm), bl = __ballot_sync(0xFFFFFFFFu, lg);
            if (lane == 0) {
                s_cnt[0][warp] = __popc(bs);
                s_cnt[1][warp] = __popc(bl);
            }
            __syncthreads();
            uint32_t os = s_tot[0], ol = s_tot[1];
            for (uint32_t k = 0; k < warp; ++k) {
                os += s_cnt[0][k];
                ol += s_cnt[1][k];
            }
            const unsigned lt = (1u << lane) - 1u;
            if (sm) qs[h + os + __popc(bs & lt)] = (uint32_t)i;
            if (lg) ql[h + ol + __popc(bl & lt)] = (uint32_t)i;
            __syncthreads();
            if (threadIdx.x == 0)
                for (uint32_t k = 0; k < blockDim.x / 32; ++k) {
                    s_tot[0] += s_cnt[0][k];
                    s_tot[1] += s_cnt[1][k];
                }
            __syncthreads();
        }
        const uint32_t ns0 = s_tot[0], nl = s_tot[1];
        if (warp == 0) {
            // Vose's loop.  The two initial queues are read in order, 32
            // entries at a time, the next 32 fetched ahead: their indices when
            // a chunk is entered, their probabilities 16 entries later (the
            // indices have landed by then).
            uint32_t sb_i = 0, lb_i = 0, ab_i = 0, sn_i = 0, ln_i = 0;
            double sb_p = 0.0, lb_p = 0.0, ab_p = 0.0, sn_p = 0.0, ln_p = 0.0;
            uint32_t sbase = kNone, lbase = kNone, abase = kNone;
            auto get_s = [&](uint32_t k, uint32_t &idx, double &p) {  // initial small k < ns0, k = 0, 1, 2, ...
                if (sbase == kNone) {
                    sbase = k;
                    sb_i = k + lane < ns0 ? qs[h + k + lane] : 0u;
                    sb_p = k + lane < ns0 ? pd[h + sb_i] : 0.0;
                    sn_i = k + 32 + lane < ns0 ? qs[h + k + 32 + lane] : 0u;
                } else if (k == sbase + 32) {
                    sbase = k;
                    sb_i = sn_i;
                    sb_p = sn_p;
                    sn_i = k + 32 + lane < ns0 ? qs[h + k + 32 + lane] : 0u;
                }
                if (k == sbase + 16) sn_p = sbase + 32 + lane < ns0 ? pd[h + sn_i] : 0.0;
                idx = __shfl_sync(0xFFFFFFFFu, sb_i, k - sbase);
                p = __shfl_sync(0xFFFFFFFFu, sb_p, k - sbase);
            };
            auto get_l = [&](uint32_t k, uint32_t &idx, double &p) {  // initial large k < nl, k = 0, 1, 2, ...
                if (lbase == kNone) {
                    lbase = k;
                    lb_i = k + lane < nl ? ql[h + k + lane] : 0u;
                    lb_p = k + lane < nl ? pd[h + lb_i] : 0.0;
                    ln_i = k + 32 + lane < nl ? ql[h + k + 32 + lane] : 0u;
                } else if (k == lbase + 32) {
                    lbase = k;
                    lb_i = ln_i;
                    lb_p = ln_p;
                    ln_i = k + 32 + lane < nl ? ql[h + k + 32 + lane] : 0u;
                }
                if (k == lbase + 16) ln_p = lbase + 32 + lane < nl ? pd[h + ln_i] : 0.0;
                idx = __shfl_sync(0xFFFFFFFFu, lb_i, k - lbase);
                p = __shfl_sync(0xFFFFFFFFu, lb_p, k - lbase);
            };
            // dropped larges: the last 32 in a register ring (entry j in lane
            // j % 32), older ones from memory, 32 at a time
            uint32_t na = 0;  // dropped larges so far (== larges consumed)
            uint32_t ring_i = 0;
            double ring_p = 0.0;
            auto get_a = [&](uint32_t k, uint32_t &idx, double &p) {  // dropped large k < na
                if (na - k <= 32u) {
                    idx = __shfl_sync(0xFFFFFFFFu, ring_i, k & 31u);
                    p = __shfl_sync(0xFFFFFFFFu, ring_p, k & 31u);
                    return;
                }
                if (abase == kNone || k < abase || k >= abase + 32u) {
                    __syncwarp();  // lane 0's writes of the entries are visible
                    abase = k;     // k + 32 < na: all 32 are written
                    ab_i = ql[h + k + lane];
                    ab_p = pd[h + ab_i];
                }
                idx = __shfl_sync(0xFFFFFFFFu, ab_i, k - abase);
                p = __shfl_sync(0xFFFFFFFFu, ab_p, k - abase);
            };
            uint32_t hs = 0, hl = 0, lidx = 0;
            double r = 0.0;
            if (nl) get_l(0, lidx, r);
            while (hs < ns0 + na && hl < nl) {
                uint32_t sidx;
                double ps;
                if (hs < ns0) get_s(hs, sidx, ps);
                else get_a(hs - ns0, sidx, ps);
                ++hs;
                if (lane == 0) out[h + sidx] = AliasEntry{__double2float_rn(ps), lidx};
                r = __dsub_rn(__dadd_rn(r, ps), 1.0);
                if (r < 1.0) {
                    // the large drops into the small queue, behind the consumed larges
                    if (lane == 0) {
                        pd[h + lidx] = r;
                        ql[h + na] = lidx;
                    }
                    if (lane == (na & 31u)) {
                        ring_i = lidx;
                        ring_p = r;
                    }
                    ++na;
                    if (++hl < nl) get_l(hl, lidx, r);
                }
            }
            __syncwarp();
            // what is left keeps its own column: the larges from the current
            // one on, and the smalls not consumed
            for (uint32_t k = hl + lane; k < nl; k += 32) {
                const uint32_t i = ql[h + k];
                out[h + i] = AliasEntry{1.f, i};
            }
            for (uint32_t k = hs + lane; k < ns0 + na; k += 32) {
                const uint32_t i = k < ns0 ? qs[h + k] : ql[h + (k - ns0)];
                out[h + i] = AliasEntry{1.f, i};
            }
        }
        __syncthreads();
    }
}

cudaError_t launch_build_alias(const uint64_t *beg, const float *w, uint32_t nverts, double *pd, uint32_t *qs,
                               uint32_t *ql, uint32_t *work, AliasEntry *out, uint32_t *err, int num_sms, cudaStream_t s)
{
    k_build_alias<<<num_sms * 8, 128, 0, s>>>(beg, w, nverts, pd, qs, ql, out, err);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(work, 0, 2 * sizeof(uint32_t), s)) != cudaSuccess) return e;
    k_list_hubs<<<num_sms * 4, 256, 0, s>>>(beg, nverts, 16 * kHubDeg, ~0ull, work);
    k_list_hubs<<<num_sms * 4, 256, 0, s>>>(beg, nverts, kHubDeg, 16 * kHubDeg, work);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_build_alias_hubs<<<num_sms * 4, 128, 0, s>>>(beg, w, work, pd, qs, ql, out, err);
    return cudaGetLastError();
}


}  // namespace gw

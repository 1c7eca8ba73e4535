// Out-of-core kernels (replace GOWalker gpu/gpuwalk.hpp:87-372 and the host
// block choice of engine/schedule.hpp:70-138).
//
//  k_init_walkers  walker records from ids (engine/walk.hpp:32-95)
//  k_count         walkers per (prev block, cur block) bucket, warp-aggregated
//                  atomics (one atomic per distinct bucket per warp instead of
//                  one per walker, gpu/gpuwalk.hpp:179)
//  k_scan          exclusive scan of the bucket counts in one CTA (coalesced warp segments)
//                  (the reference scans them on one thread, gpu/gpuwalk.hpp:321-338)
//  k_scatter       walkers into bucket order, finished walkers dropped
//                  (gpu/gpuwalk.hpp:340-360 + the spill of engine/walk.hpp:484-525)
//  k_runnable      ranges of the buckets whose two blocks are resident
//  k_schedule      GOwalker_scheduler_t::max_choose_blocks on the device
//  k_walk_ooc      the step kernel over runnable walkers; a walker stops when
//                  its next vertex lies in a block that is not resident
#include <cuda_runtime.h>
#include <cstdint>
#include "gw_ooc_kernels.cuh"

namespace gw {


__device__ __forceinline__ uint32_t block_of(const uint32_t *vs, uint32_t nb, uint32_t v)
{
    // largest b with vs[b] <= v (vs[nb] = nverts > v)
    uint32_t lo = 0, hi = nb;  // invariant vs[lo] <= v < vs[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (vs[mid] <= v) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ uint32_t bucket_of(const WalkerRec &r, uint32_t nb)
{
    if (r.prev_blk == kFinished) return kNoBucket;
    return ((r.cur_blk & kNeedPrev) ? nb * nb : 0u) + r.prev_blk * nb + (r.cur_blk & ~kNeedPrev);
}

__global__ void k_init_walkers(WalkerInit in, const uint32_t *__restrict__ vstart, uint32_t nb, uint32_t wid0,
                               uint64_t n, WalkerRec *__restrict__ out, uint32_t *__restrict__ order,
                               uint32_t *__restrict__ keys, uint32_t *__restrict__ paths, uint32_t stride)
{
    __shared__ uint32_t s_vs[kMaxBlocks + 1];
    for (uint32_t i = threadIdx.x; i <= nb; i += blockDim.x) s_vs[i] = vstart[i];
    __syncthreads();
    const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += step) {
        const uint32_t wid = wid0 + (uint32_t)i;
        const uint32_t src = walker_source(in, wid);
        const uint32_t b = block_of(s_vs, nb, src);
        const uint64_t h = hash_init(src);
        WalkerRec r;
        r.wid = wid;
        r.prev = src;
        r.cur = src;
        r.hop = 0;
        r.prev_blk = b;
        r.cur_blk = b;
        r.hash_lo = (uint32_t)h;
        r.hash_hi = (uint32_t)(h >> 32);
        out[i] = r;
        order[i] = (uint32_t)i;
        keys[i] = bucket_of(r, nb);
        if (paths) paths[i * stride] = src;
    }
}

__global__ void k_count(const uint32_t *__restrict__ keys, const uint32_t *__restrict__ n_ptr, uint32_t *__restrict__ counts)
{
    const uint64_t n = *n_ptr;
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) & ~31ull; base < n; base += step) {
        const uint64_t i = base + lane;
        const uint32_t b = (i < n) ? keys[i] : kNoBucket;
        const unsigned grp = __match_any_sync(0xFFFFFFFFu, b);
        if (b != kNoBucket && lane == (uint32_t)(__ffs(grp) - 1)) atomicAdd(&counts[b], (uint32_t)__popc(grp));
    }
}

__global__ void k_scatter(const uint32_t *__restrict__ keys_in, const uint32_t *__restrict__ order_in,
                          const uint32_t *__restrict__ n_ptr, const uint32_t *__restrict__ offsets,
                          uint32_t *__restrict__ cursor, uint32_t *__restrict__ keys_out,
                          uint32_t *__restrict__ order_out)
{
    const uint64_t n = *n_ptr;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt = (1u << lane) - 1u;
    const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) & ~31ull; base < n; base += step) {
        const uint64_t i = base + lane;
        uint32_t r = 0, b = kNoBucket;
        if (i < n) {
            b = keys_in[i];
            r = order_in[i];
        }
        const unsigned grp = __match_any_sync(0xFFFFFFFFu, b);
        if (b != kNoBucket) {
            const uint32_t leader = (uint32_t)(__ffs(grp) - 1);
            uint32_t pos = 0;
            if (lane == leader) pos = atomicAdd(&cursor[b], (uint32_t)__popc(grp));
            pos = __shfl_sync(grp, pos, leader) + (uint32_t)__popc(grp & lt);
            keys_out[offsets[b] + pos] = b;
            order_out[offsets[b] + pos] = r;
        }
    }
}

// One-CTA scans over at most 2^20 entries (nblocks <= 1024).
constexpr int kScanThreads = 1024;


// Warp w of the CTA owns entries [w * seg, (w + 1) * seg) and walks them 32
// at a time, so every load and store of a round is one coalesced line; the
// warps' totals are scanned once through shared memory.
__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x, uint32_t lane)
{
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    return x;
}

__device__ __forceinline__ uint32_t warp_sum(uint32_t x)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xFFFFFFFFu, x, o);
    return x;
}

// Exclusive scan of the warps' totals: warp w gets the sum of warps < w.
__device__ __forceinline__ uint32_t cta_warp_base(uint32_t wtotal, uint32_t *total)
{
    __shared__ uint32_t s_t[32];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (lane == 0) s_t[warp] = wtotal;
    __syncthreads();
    if (warp == 0) {
        const uint32_t v = lane < (blockDim.x >> 5) ? s_t[lane] : 0u;
        const uint32_t inc = warp_incl_scan(v, lane);
        s_t[lane] = inc - v;
        if (lane == 31 && total) *total = inc;
    }
    __syncthreads();
    const uint32_t b = s_t[warp];
    __syncthreads();
    return b;
}

__global__ void __launch_bounds__(kScanThreads) k_scan(const uint32_t *__restrict__ in, uint32_t n,
                                                       uint32_t *__restrict__ out)
{
    __shared__ uint32_t s_total;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint32_t seg = ((n + nw - 1) / nw + 31u) & ~31u;
    const uint32_t lo = min(warp * seg, n), hi = min(lo + seg, n);
    uint32_t part = 0;
#pragma unroll 4
    for (uint32_t i = lo + lane; i < hi; i += 32) part += in[i];
    uint32_t base = cta_warp_base(warp_sum(part), &s_total);
#pragma unroll 4
    for (uint32_t i0 = lo; i0 < hi; i0 += 32) {
        const uint32_t i = i0 + lane;
        const uint32_t v = i < hi ? in[i] : 0u;
        const uint32_t inc = warp_incl_scan(v, lane);
        if (i < hi) out[i] = base + inc - v;
        base += __shfl_sync(0xFFFFFFFFu, inc, 31);
    }
    __syncthreads();
    if (threadIdx.x == 0) out[n] = s_total;
}

__global__ void __launch_bounds__(kScanThreads) k_runnable(const uint32_t *__restrict__ counts,
                                                           const uint32_t *__restrict__ offsets,
                                                           const uint32_t *const *__restrict__ blk_csr, uint32_t nb,
                                                           uint32_t lazy, uint32_t *__restrict__ run_pre,
                                                           uint32_t *__restrict__ run_off, uint32_t *__restrict__ nrun)
{
    __shared__ uint8_t s_res[kMaxBlocks];
    __shared__ uint32_t s_cnt, s_sum;
    for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) s_res[i] = blk_csr[i] != nullptr;
    __syncthreads();
    const uint32_t nn = nb * nb, n = 2 * nn;
    // unflagged walkers need their current block (and, unless lazy, the
    // previous one); flagged walkers need both
    auto runnable = [&](uint32_t b) {
        const uint32_t pc = b < nn ? b : b - nn;
        const bool cur_ok = s_res[pc % nb] != 0, prev_ok = s_res[pc / nb] != 0;
        return cur_ok && (prev_ok || (lazy && b < nn));
    };
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t seg = ((n + nw - 1) / nw + 31u) & ~31u;
    const uint32_t lo = min(warp * seg, n), hi = min(lo + seg, n);
    uint32_t pc = 0, ps = 0;
#pragma unroll 4
    for (uint32_t b = lo + lane; b < hi; b += 32) {
        const uint32_t c = counts[b];
        if (c && runnable(b)) {
            pc++;
            ps += c;
        }
    }
    uint32_t kb = cta_warp_base(warp_sum(pc), &s_cnt);
    uint32_t sb = cta_warp_base(warp_sum(ps), &s_sum);
#pragma unroll 4
    for (uint32_t b0 = lo; b0 < hi; b0 += 32) {
        const uint32_t b = b0 + lane;
        const uint32_t c = b < hi ? counts[b] : 0u;
        const bool f = c && runnable(b);
        const unsigned fm = __ballot_sync(0xFFFFFFFFu, f);
        const uint32_t v = f ? c : 0u;
        const uint32_t inc = warp_incl_scan(v, lane);
        if (f) {
            const uint32_t k = kb + (uint32_t)__popc(fm & lt);
            run_off[k] = offsets[b];
            run_pre[k] = sb + inc - v;
        }
        kb += (uint32_t)__popc(fm);
        sb += __shfl_sync(0xFFFFFFFFu, inc, 31);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        *nrun = s_cnt;
        run_pre[s_cnt] = s_sum;
    }
}

// Block choice, GOwalker_scheduler_t::max_choose_blocks (engine/schedule.hpp:70-138):
//  cache not full: for every uncached block i, score = sum over cached c of
//    walkers(i,c) + walkers(c,i), plus walkers(i,i); the best block is added.
//  cache full: for every uncached i, s_j = walkers(i,c_j) + walkers(c_j,i);
//    score = sum_j s_j - min_j s_j and i replaces the cached block with the
//    smallest s_j (first such j).
//  A block is taken only if its score is > 0 and > zero_threshold; ties go to
//  the lowest block id (the reference's std::sort leaves their order open).
// Rescue choice, for runs without the zero-copy tail (where the reference
// would switch to it): the fullest bucket with an absent block; load its first
// absent block, evicting the cached block with the fewest incident walkers
// outside that bucket -- after at most two rescues the bucket runs, so every
// run ends.  `pred` (optional, the learned policy): each block's forecast of
// log1p(incident walkers over the next iterations); with a full cache the
// chosen block then replaces the cached block with the lowest forecast
// instead of the one with the smallest link (pred_weight is unused).
__global__ void __launch_bounds__(1024) k_schedule(const uint32_t *__restrict__ counts,
                                                   const uint32_t *__restrict__ live, uint32_t nb,
                                                   const uint32_t *__restrict__ cached, uint32_t ncached,
                                                   uint32_t nslots, uint32_t zero_threshold,
                                                   const float *__restrict__ pred, float pred_weight,
                                                   Decision *__restrict__ out)
{
    __shared__ uint8_t s_cached[kMaxBlocks];
    __shared__ uint32_t s_list[kMaxBlocks];
    __shared__ uint32_t s_pos[kMaxBlocks];
    __shared__ unsigned long long s_inc[kMaxBlocks];
    __shared__ unsigned long long s_best, s_bucket;
    for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) s_cached[i] = 0;
    if (threadIdx.x == 0) {
        s_best = 0;
        s_bucket = 0;
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < ncached; j += blockDim.x) {
        s_list[j] = cached[j];
        s_cached[cached[j]] = 1;
    }
    __syncthreads();
    const bool full = ncached >= nslots;
    // one warp per block i: lanes split the row / column and the cached list
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (uint32_t i = warp; i < nb; i += nw) {
        unsigned long long incident = 0;  // walkers in buckets touching i (row + column, diagonal once)
        for (uint32_t c = lane; c < nb; c += 32)
            incident += (unsigned long long)counts[i * nb + c] + (c != i ? counts[c * nb + i] : 0u);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) incident += __shfl_xor_sync(0xFFFFFFFFu, incident, o);
        if (lane == 0) s_inc[i] = incident;
        if (s_cached[i]) continue;  // warp-uniform
        unsigned long long score = 0;
        uint32_t pos = 0;
        if (!full) {
            for (uint32_t j = lane; j < ncached; j += 32) {
                const uint32_t c = s_list[j];
                score += (unsigned long long)counts[i * nb + c] + counts[c * nb + i];
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) score += __shfl_xor_sync(0xFFFFFFFFu, score, o);
            score += counts[i * nb + i];
        } else {
            // all minus the smallest link; the first position on ties
            unsigned long long all = 0, key = ~0ull;  // (value << 32) | position
            for (uint32_t j = lane; j < ncached; j += 32) {
                const uint32_t c = s_list[j];
                const unsigned long long v = (unsigned long long)counts[i * nb + c] + counts[c * nb + i];
                all += v;
                const unsigned long long kv = (v << 32) | j;
                key = kv < key ? kv : key;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                all += __shfl_xor_sync(0xFFFFFFFFu, all, o);
                const unsigned long long ko = __shfl_xor_sync(0xFFFFFFFFu, key, o);
                key = ko < key ? ko : key;
            }
            score = all - (key >> 32);
            pos = (uint32_t)key;
        }
        if (lane == 0) {
            s_pos[i] = pos;
            atomicMax(&s_best, (score << 11) | (2047u - i));
        }
    }
    // fullest bucket with an absent block
    const uint32_t nbk = nb * nb;
    for (uint32_t b = threadIdx.x; b < nbk; b += blockDim.x) {
        const uint32_t c = counts[b];
        if (c && !(s_cached[b / nb] && s_cached[b % nb]))
            atomicMax(&s_bucket, ((unsigned long long)c << 21) | (0x1FFFFFu - b));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        Decision d{};
        const uint64_t best = s_best >> 11;
        const int32_t bi = (int32_t)(2047u - (uint32_t)(s_best & 2047u));
        d.score = best;
        d.live = *live;
        if (s_best != 0 && best > 0 && best > zero_threshold) {
            d.action = full ? 2 : 1;
            d.block = bi;
            d.position = full ? (int32_t)s_pos[bi] : (int32_t)ncached;
            if (full && pred) {
                // learned eviction: the cached block with the lowest forecast
                // of incident walkers over the next iterations (first on ties)
                float mn = 3.0e38f;
                for (uint32_t j = 0; j < ncached; ++j)
                    if (pred[s_list[j]] < mn) {
                        mn = pred[s_list[j]];
                        d.position = (int32_t)j;
                    }
            }
        } else {
            d.action = 0;
            d.block = -1;
            d.position = -1;
        }
        d.rescue_block = -1;
        d.rescue_position = -1;
        if (s_bucket) {
            const uint32_t b = 0x1FFFFFu - (uint32_t)(s_bucket & 0x1FFFFFu);
            const uint32_t p = b / nb, c = b % nb;
            d.rescue_block = (int32_t)(s_cached[c] ? p : c);  // the current block first: lazy walkers need only it
            if (full) {
                unsigned long long mn = ~0ull;
                for (uint32_t j = 0; j < ncached; ++j) {
                    const uint32_t blk = s_list[j];
                    if (blk == p || blk == c) continue;
                    if (s_inc[blk] < mn) {
                        mn = s_inc[blk];
                        d.rescue_position = (int32_t)j;
                    }
                }
            }
        }
        *out = d;
        __threadfence_system();  // `out` may be mapped host memory
    }
}

// W: weighted Node2vec -- the candidate is alias column r.x % deg, kept when
// float(r.w >> 8) * 2^-24 < its probability, else its alias (the block's
// alias tables sit behind its neighbour list), as in the in-core kernel.
// ZC: the zero-copy tail -- the blocks marked in a.mapped are read through
// mapped host memory; every read of one is counted as a 32-byte sector in
// kCtrZcSectors (an upper bound of the host-link bytes: each probe of a
// binary search counts as its own sector).  Without ZC the same count is
// taken as if every block were mapped (kCtrModelSectors): what these steps
// would cost in the zero-copy tail, the learned policy's switch estimate.
template <bool SOPR, bool PATHS, bool COOP, bool W = false, bool ZC = false>
__global__ void __launch_bounds__(kWalkThreads) k_walk_ooc(const __grid_constant__ OocStepArgs a)
{
    __shared__ uint32_t s_vs[kMaxBlocks + 1];
    __shared__ uint8_t s_mapped[ZC ? kMaxBlocks : 1];
    if constexpr (ZC)
        for (uint32_t i = threadIdx.x; i < a.nb; i += blockDim.x) s_mapped[i] = a.mapped[i];
    uint32_t zc_sectors = 0;
    // sectors of a plain binary search over n ids plus the final read: at most
    // bit_length(n) + 1
    auto search_sectors = [](uint32_t n) { return 33u - (uint32_t)__clz(n); };
    __shared__ uint32_t s_iv[kWalkThreads / 32][kCoopScratchWords];
    __shared__ unsigned long long s_ws[kWalkThreads / 32][kWsCount];  // per-warp statistics
    for (uint32_t i = threadIdx.x; i <= a.nb; i += blockDim.x) s_vs[i] = a.vstart[i];
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    if (lane < kWsCount) s_ws[warp][lane] = 0;
    __syncthreads();

    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint32_t nrun = *a.nrun;
    const uint32_t total = a.run_pre[nrun];
    const uint32_t maxhops = a.c.maxhops;
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&a.ctr[kCtrRunnable], (unsigned long long)total);

    uint32_t q_next = 0, q_end = 0;
    bool exhausted = false;
    bool active = false;

    uint32_t wid = 0, prev = 0, cur = 0, hop = 0, hop0 = 0, attempt = 0, pb = 0, cb = 0, deg = 0, pdeg = 0;
    uint64_t idx = 0, head = 0, phead = 0, h = 0;
    const uint32_t *ccsr = nullptr, *pcsr = nullptr;
    const uint2 *calias = nullptr;  // W: the current block's alias tables
    U4 r{0, 0, 0, 0};
    StepThr t{0.f, 0.f, 0.f};
    uint32_t n_trials = 0;  // trials not yet added to s_ws

    // Statistics of the walker leaving this lane (finished or parked): its
    // steps in this launch are the hops it made since it was loaded.
    auto flush = [&]() {
        atomicAdd(&s_ws[warp][kWsSteps], (unsigned long long)(hop - hop0));
        atomicAdd(&s_ws[warp][kWsTrials], (unsigned long long)n_trials);
        n_trials = 0;
    };
    auto finish = [&]() {
        a.hashes[wid - a.out_base] = h;
        a.lens[wid - a.out_base] = hop + 1;
        a.keys[idx] = kNoBucket;
        atomicAdd(&s_ws[warp][kWsHash], (unsigned long long)h);
        atomicAdd(&s_ws[warp][kWsDone], 1ull);
        flush();
        active = false;
    };
    // Enter a step at vertex cur (block cb), prev adjacency already set:
    // termination draw, then cur's offsets (the order of the in-core kernel).
    auto enter = [&]() {
        r = draw(a.c, wid, hop, 0);
        attempt = 1;
        if (hop > 0 && terminates(a.c, r.z)) {
            finish();
            return;
        }
        ccsr = a.blk_csr[cb];
        if constexpr (W) calias = a.blk_alias[cb];
        const uint64_t b0 = __ldg(a.beg + cur), b1 = __ldg(a.beg + cur + 1);
        head = b0 - a.estart[cb];
        deg = (uint32_t)(b1 - b0);
        if (deg == 0) {
            finish();
            return;
        }
        t = step_thresholds<SOPR>(a.c, deg, pdeg);
        active = true;
    };

    for (;;) {
        for (;;) {
            const unsigned need = __ballot_sync(0xFFFFFFFFu, !active);
            if (need == 0 || exhausted) break;
            if (q_next >= q_end) {
                uint32_t base = 0;
                if (lane == 0) base = (uint32_t)atomicAdd(&a.ctr[kCtrCursor], (unsigned long long)kChunk);
                base = __shfl_sync(0xFFFFFFFFu, base, 0);
                if (base >= total) {
                    exhausted = true;
                    break;
                }
                q_next = base;
                q_end = min(base + kChunk, total);
            }
            const uint32_t avail = q_end - q_next;
            const uint32_t rank = __popc(need & lt_mask);
            if (!active && rank < avail) {
                const uint32_t g = q_next + rank;
                uint32_t lo = 0, hi = nrun;  // run_pre[lo] <= g < run_pre[hi]
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (__ldg(a.run_pre + mid) <= g) lo = mid;
                    else hi = mid;
                }
                idx = (uint64_t)__ldg(a.run_off + lo) + (g - __ldg(a.run_pre + lo));
                const WalkerRec rec = a.recs[__ldg(a.order + idx)];
                wid = rec.wid;
                prev = rec.prev;
                cur = rec.cur;
                hop = rec.hop;
                hop0 = hop;
                pb = rec.prev_blk;
                cb = rec.cur_blk & ~kNeedPrev;
                h = ((uint64_t)rec.hash_hi << 32) | rec.hash_lo;
                // lazy mode: the previous block may be absent (pcsr null); its
                // offsets are resident, so deg(prev) is known either way
                pcsr = hop < maxhops ? a.blk_csr[pb] : nullptr;
                if (hop >= maxhops) {
                    finish();
                } else if (pcsr == nullptr && !a.lazy) {
                    atomicOr(a.err, kErrBlock);  // scheduled without its previous block
                    finish();
                } else {
                    const uint64_t p0 = __ldg(a.beg + prev), p1 = __ldg(a.beg + prev + 1);
                    phead = p0 - a.estart[pb];
                    pdeg = (uint32_t)(p1 - p0);
                    enter();
                }
            }
            q_next += min((uint32_t)__popc(need), avail);
        }
        if (!__any_sync(0xFFFFFFFFu, active)) break;

        // hard steps: the whole warp evaluates 32 attempts per round
        for (unsigned hm = COOP ? __ballot_sync(0xFFFFFFFFu, active && attempt > kHardAttempts) : 0u; hm;
             hm &= hm - 1) {
            const int L = __ffs(hm) - 1;
            const uint32_t p0 = __shfl_sync(0xFFFFFFFFu, attempt, L) - 1;
            const uint64_t hd = shfl64(head, L), ph = shfl64(phead, L);
            const uint32_t *cc = shfl_ptr(ccsr, L), *pc = shfl_ptr(pcsr, L);
            uint32_t xs;
            const CsrIndex cix{cc, {}, 0}, pix{pc, {}, 0};
            const uint32_t astar = warp_first_accept<SOPR>(
                a.c, shfl_thr<SOPR>(t, L), __shfl_sync(0xFFFFFFFFu, wid, L), __shfl_sync(0xFFFFFFFFu, hop, L), p0,
                kMaxAttempts, cix, hd, __shfl_sync(0xFFFFFFFFu, deg, L), __shfl_sync(0xFFFFFFFFu, prev, L),
                __shfl_sync(0xFFFFFFFFu, cur, L), pix, ph, __shfl_sync(0xFFFFFFFFu, pdeg, L), s_iv[warp], &xs);
            if (lane == (uint32_t)L) {
                n_trials += astar - p0;
                if constexpr (ZC)  // every attempt: a candidate and, at most, a search of N(prev)
                    zc_sectors += (astar - p0) * ((s_mapped[cb] ? 1u : 0u) + (s_mapped[pb] ? search_sectors(pdeg) : 0u));
                else
                    zc_sectors += (astar - p0) * (1u + search_sectors(pdeg));
                if (astar >= kMaxAttempts) {
                    atomicOr(a.err, kErrTrials);
                    finish();
                } else {
                    r = draw(a.c, wid, hop, astar);
                    attempt = astar + 1;
                }
            }
        }
        if (!active) continue;

        const uint32_t pos = r.x % deg;
        const float rv = rand_val(r.y, thr_max<SOPR>(a.c, t));
        uint32_t col = pos;
        if constexpr (W) {
            const uint2 e = __ldg(calias + head + pos);
            if (!(__uint2float_rn(r.w >> 8) * 0x1p-24f < __uint_as_float(e.x))) col = e.y;
        }
        const uint32_t x = __ldg(ccsr + head + col);
        n_trials++;
        {
            // accept_candidate searches N(prev) when neither the rand value
            // nor x == prev (nor prev == cur) decides the trial
            const bool cm = ZC ? s_mapped[cb] != 0 : true, pm = ZC ? s_mapped[pb] != 0 : true;
            if (cm) zc_sectors += 1u;
            if (pcsr != nullptr && pm && !(rv <= thr_min<SOPR>(a.c, t)) && x != prev && prev != cur)
                zc_sectors += search_sectors(pdeg);
        }
        const int verdict = pcsr != nullptr
                                ? (accept_candidate<SOPR>(a.c, t, rv, x, prev, cur, CsrIndex{pcsr, {}, 0}, phead, pdeg) ? 1 : 0)
                                : accept_without_prev<SOPR>(a.c, t, rv, x, prev, cur);
        if (verdict < 0) {
            // Needs N(prev), whose block is absent: park the walker flagged in
            // bucket (prev block, cur block).  The step restarts at attempt 0
            // once both blocks are resident (the draws are counter-based), so
            // its attempts so far are not counted.
            WalkerRec rec;
            rec.wid = wid;
            rec.prev = prev;
            rec.cur = cur;
            rec.hop = hop;
            rec.prev_blk = pb;
            rec.cur_blk = cb | kNeedPrev;
            rec.hash_lo = (uint32_t)h;
            rec.hash_hi = (uint32_t)(h >> 32);
            a.recs[__ldg(a.order + idx)] = rec;
            a.keys[idx] = bucket_of(rec, a.nb);
            n_trials -= attempt;
            flush();
            active = false;
        } else if (verdict > 0) {
            hop++;
            h = hash_step(h, x);
            if (PATHS) a.paths[(uint64_t)(wid - a.out_base) * a.stride + hop] = x;
            if (n_trials & 0x80000000u) {  // a step adds < 2^27: no wrap
                atomicAdd(&s_ws[warp][kWsTrials], (unsigned long long)n_trials);
                n_trials = 0;
            }
            prev = cur;
            pb = cb;
            phead = head;
            pdeg = deg;
            pcsr = ccsr;
            cur = x;
            if (hop >= maxhops) {
                finish();
            } else if (x >= a.nverts) {
                atomicOr(a.err, kErrVertexRange);
                finish();
            } else {
                const uint32_t nbx = (x >= s_vs[cb] && x < s_vs[cb + 1]) ? cb : block_of(s_vs, a.nb, x);
                if (a.blk_csr[nbx] == nullptr) {
                    // next block absent: park the walker in bucket (cb, nbx)
                    WalkerRec rec;
                    rec.wid = wid;
                    rec.prev = prev;
                    rec.cur = cur;
                    rec.hop = hop;
                    rec.prev_blk = pb;
                    rec.cur_blk = nbx;
                    rec.hash_lo = (uint32_t)h;
                    rec.hash_hi = (uint32_t)(h >> 32);
                    a.recs[__ldg(a.order + idx)] = rec;
                    a.keys[idx] = bucket_of(rec, a.nb);
                    flush();
                    active = false;
                } else {
                    cb = nbx;
                    enter();
                }
            }
        } else if (attempt >= kMaxAttempts) {
            atomicOr(a.err, kErrTrials);
            finish();
        } else {
            r = draw(a.c, wid, hop, attempt);
            attempt++;
        }
    }

    __syncwarp();
    if (lane == 0) {
        atomicAdd(&a.ctr[kCtrSteps], s_ws[warp][kWsSteps]);
        atomicAdd(&a.ctr[kCtrTrials], s_ws[warp][kWsTrials]);
        atomicAdd(&a.ctr[kCtrDone], s_ws[warp][kWsDone]);
        atomicAdd(&a.ctr[kCtrHashSum], s_ws[warp][kWsHash]);
    }
    {
        const unsigned long long zs = warp_sum((unsigned long long)zc_sectors);
        if (lane == 0 && zs) atomicAdd(&a.ctr[ZC ? kCtrZcSectors : kCtrModelSectors], zs);
    }
}

// ------------------------------------------------------------------ learned policy

// Per-block features of the demand predictor (all log1p-scaled counts):
//  0 waiting at i (cur block i)   1 leaving i (prev block i)   2 diagonal (i,i)
//  3 walkers between i and resident blocks   4 walkers that run if i is resident
//  5 resident   6 edge share   7 vertex share   8 arrival EMA   9 arrivals
// 10 live fraction  11 iteration/256  12 waiting share  13 incident
// 14 leaving, off-diagonal  15 waiting, off-diagonal
__global__ void __launch_bounds__(1024) k_features(const FeatureArgs f)
{
    __shared__ uint8_t s_res[kMaxBlocks];
    const uint32_t nb = f.nb;
    for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) s_res[i] = f.blk_csr[i] != nullptr;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) {
        uint64_t col = 0, row = 0, cross = 0, ready = 0;
        for (uint32_t p = 0; p < nb; ++p) {
            const uint32_t cpi = f.counts[p * nb + i], cip = f.counts[i * nb + p];
            col += cpi;
            row += cip;
            if (s_res[p]) cross += (uint64_t)cpi + cip;
            if (s_res[p] || p == i) ready += cpi;
        }
        const uint32_t diag = f.counts[i * nb + i];
        const float colf = (float)col;
        const float arr = fmaxf(colf - f.prev_col[i], 0.f);
        const float ema = 0.7f * f.ema_arr[i] + 0.3f * arr;
        f.prev_col[i] = colf;
        f.ema_arr[i] = ema;
        float *x = f.x + (uint64_t)i * 16;
        x[0] = log1pf(colf);
        x[1] = log1pf((float)row);
        x[2] = log1pf((float)diag);
        x[3] = log1pf((float)cross);
        x[4] = log1pf((float)ready);
        x[5] = s_res[i] ? 1.f : 0.f;
        x[6] = f.emass[i];
        x[7] = f.vfrac[i];
        x[8] = log1pf(ema);
        x[9] = log1pf(arr);
        x[10] = f.live_frac;
        x[11] = 0.f;  // (the iteration count: left out, it only grows past what training saw)
        x[12] = colf * f.inv_live * (float)nb;
        x[13] = log1pf((float)(row + col - diag));
        x[14] = log1pf((float)(row - diag));
        x[15] = log1pf((float)(col - diag));
        f.col[i] = (float)(row + col - diag);  // incident walkers: the forecast's quantity
    }
}

// Training set from the trace ring (ring slots of kMlpIn features and of
// incident walkers per block -- walkers whose current or previous block it
// is; iteration t lives in slot t % ring): samples t0 .. t0+T-1 gathered in
// order, with targets y = log1p(mean incident walkers over the next k
// iterations) - x[13] (x[13] = log1p of the incident walkers then), so the
// network learns the change of that log demand and an untrained one
// forecasts no change.
__global__ void k_gather_train(const float *ring_x, const float *ring_col, uint32_t t0, uint32_t ring, uint32_t T,
                               uint32_t k, uint32_t nb, float *train_x, float *y)
{
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= T * nb) return;
    const uint32_t j = idx / nb, i = idx % nb;
    const uint32_t t = t0 + j;
    const float *xs = ring_x + ((uint64_t)(t % ring) * nb + i) * 16;
    float *xd = train_x + (uint64_t)idx * 16;
    for (int f = 0; f < 16; ++f) xd[f] = xs[f];
    float s = 0.f;
    for (uint32_t d = 1; d <= k; ++d) s += ring_col[(uint64_t)((t + d) % ring) * nb + i];
    y[idx] = log1pf(s / (float)k) - xs[13];
}

// level[i] = res[i] + x[i][13]: the forecast change back to log incident walkers.
__global__ void k_add_level(const float *res, const float *x, float *level, uint32_t nb)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nb) level[i] = res[i] + x[(uint64_t)i * 16 + 13];
}


cudaError_t launch_features(const FeatureArgs &f, cudaStream_t s)
{
    k_features<<<1, 1024, 0, s>>>(f);
    return cudaGetLastError();
}

cudaError_t launch_gather_train(const float *ring_x, const float *ring_col, uint32_t t0, uint32_t ring, uint32_t T,
                                uint32_t k, uint32_t nb, float *train_x, float *y, cudaStream_t s)
{
    const uint32_t n = T * nb;
    k_gather_train<<<(n + 255) / 256, 256, 0, s>>>(ring_x, ring_col, t0, ring, T, k, nb, train_x, y);
    return cudaGetLastError();
}

cudaError_t launch_add_level(const float *res, const float *x, float *level, uint32_t nb, cudaStream_t s)
{
    k_add_level<<<(nb + 255) / 256, 256, 0, s>>>(res, x, level, nb);
    return cudaGetLastError();
}


// ------------------------------------------------------------------ launchers

cudaError_t launch_init_walkers(const WalkerInit &in, const uint32_t *vstart, uint32_t nb, uint32_t wid0, uint64_t n,
                                WalkerRec *recs, uint32_t *order, uint32_t *keys, uint32_t *paths, uint32_t stride,
                                int num_sms, cudaStream_t s)
{
    k_init_walkers<<<num_sms * 8, 256, 0, s>>>(in, vstart, nb, wid0, n, recs, order, keys, paths, stride);
    return cudaGetLastError();
}

cudaError_t launch_count(const uint32_t *keys, const uint32_t *n, uint32_t *counts, int num_sms, cudaStream_t s)
{
    k_count<<<num_sms * 8, 256, 0, s>>>(keys, n, counts);
    return cudaGetLastError();
}

cudaError_t launch_scan(const uint32_t *counts, uint32_t n, uint32_t *offsets, cudaStream_t s)
{
    k_scan<<<1, kScanThreads, 0, s>>>(counts, n, offsets);
    return cudaGetLastError();
}

cudaError_t launch_scatter(const uint32_t *keys_in, const uint32_t *order_in, const uint32_t *n, const uint32_t *offsets,
                           uint32_t *cursor, uint32_t *keys_out, uint32_t *order_out, int num_sms, cudaStream_t s)
{
    k_scatter<<<num_sms * 8, 256, 0, s>>>(keys_in, order_in, n, offsets, cursor, keys_out, order_out);
    return cudaGetLastError();
}

cudaError_t launch_runnable(const uint32_t *counts, const uint32_t *offsets, const uint32_t *const *blk_csr,
                            uint32_t nb, uint32_t lazy, uint32_t *run_pre, uint32_t *run_off, uint32_t *nrun,
                            cudaStream_t s)
{
    k_runnable<<<1, kScanThreads, 0, s>>>(counts, offsets, blk_csr, nb, lazy, run_pre, run_off, nrun);
    return cudaGetLastError();
}

__global__ void k_combine(const uint32_t *__restrict__ counts, uint32_t nn, uint32_t *__restrict__ combined)
{
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x)
        combined[k] = counts[k] + counts[nn + k];
}

// Counters and error word into out (mapped host memory): one thread each.
__global__ void k_snapshot(const unsigned long long *__restrict__ ctr, const uint32_t *__restrict__ err,
                           unsigned long long *out)
{
    const uint32_t i = threadIdx.x;
    if (i < kCtrCount) out[i] = ctr[i];
    else if (i == kCtrCount) out[i] = *err;
    __threadfence_system();
}

cudaError_t launch_snapshot(const unsigned long long *ctr, const uint32_t *err, unsigned long long *out,
                            cudaStream_t s)
{
    k_snapshot<<<1, 32, 0, s>>>(ctr, err, out);
    return cudaGetLastError();
}

cudaError_t launch_combine(const uint32_t *counts, uint32_t nb, uint32_t *combined, int num_sms, cudaStream_t s)
{
    k_combine<<<num_sms, 256, 0, s>>>(counts, nb * nb, combined);
    return cudaGetLastError();
}

cudaError_t launch_schedule(const uint32_t *counts, const uint32_t *live, uint32_t nb, const uint32_t *cached,
                            uint32_t ncached, uint32_t nslots, uint32_t zero_threshold, const float *pred,
                            float pred_weight, Decision *out, cudaStream_t s)
{
    k_schedule<<<1, 1024, 0, s>>>(counts, live, nb, cached, ncached, nslots, zero_threshold, pred, pred_weight, out);
    return cudaGetLastError();
}

template <bool SOPR, bool PATHS, bool COOP, bool W = false>
static int ooc_grid_for(int num_sms)
{
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_walk_ooc<SOPR, PATHS, COOP, W>, kWalkThreads, 0);
    return (per_sm < 1 ? 1 : per_sm) * num_sms;
}

template <bool SOPR, bool PATHS, bool COOP, bool W = false>
static void ooc_launch_one(const OocStepArgs &a, int grid, cudaStream_t s)
{
    if (a.mapped) k_walk_ooc<SOPR, PATHS, COOP, W, true><<<grid, kWalkThreads, 0, s>>>(a);
    else k_walk_ooc<SOPR, PATHS, COOP, W><<<grid, kWalkThreads, 0, s>>>(a);
}

int ooc_grid(bool sopr, bool paths, bool coop, int num_sms, bool weighted)
{
    if (weighted) return paths ? ooc_grid_for<false, true, false, true>(num_sms) : ooc_grid_for<false, false, false, true>(num_sms);
    const int v = (sopr ? 4 : 0) | (paths ? 2 : 0) | (coop ? 1 : 0);
    switch (v) {
    case 0: return ooc_grid_for<false, false, false>(num_sms);
    case 1: return ooc_grid_for<false, false, true>(num_sms);
    case 2: return ooc_grid_for<false, true, false>(num_sms);
    case 3: return ooc_grid_for<false, true, true>(num_sms);
    case 4: return ooc_grid_for<true, false, false>(num_sms);
    case 5: return ooc_grid_for<true, false, true>(num_sms);
    case 6: return ooc_grid_for<true, true, false>(num_sms);
    default: return ooc_grid_for<true, true, true>(num_sms);
    }
}

cudaError_t launch_walk_ooc(const OocStepArgs &a, bool sopr, bool coop, bool weighted, int grid, cudaStream_t s)
{
    if (weighted) {
        if (sopr || coop || !a.blk_alias) return cudaErrorInvalidValue;  // weighted walks are Node2vec walks
        if (a.paths) ooc_launch_one<false, true, false, true>(a, grid, s);
        else ooc_launch_one<false, false, false, true>(a, grid, s);
        return cudaGetLastError();
    }
    const int v = (sopr ? 4 : 0) | (a.paths ? 2 : 0) | (coop ? 1 : 0);
    switch (v) {
    case 0: ooc_launch_one<false, false, false>(a, grid, s); break;
    case 1: ooc_launch_one<false, false, true>(a, grid, s); break;
    case 2: ooc_launch_one<false, true, false>(a, grid, s); break;
    case 3: ooc_launch_one<false, true, true>(a, grid, s); break;
    case 4: ooc_launch_one<true, false, false>(a, grid, s); break;
    case 5: ooc_launch_one<true, false, true>(a, grid, s); break;
    case 6: ooc_launch_one<true, true, false>(a, grid, s); break;
    default: ooc_launch_one<true, true, true>(a, grid, s); break;
    }
    return cudaGetLastError();
}

}  // namespace gw

// Step kernels of the walk engine (replace GOWalker gpu/gpuwalk.hpp:87-319).
//
// In-core kernel: one persistent grid sized to fill the SMs.  Each lane owns
// one walker at a time and takes it to the end; a warp claims walker ids in
// chunks of kChunk with one atomic and hands them to its idle lanes, so lanes
// whose walks end early (SOPR termination, dead ends) pick up new walkers
// instead of idling -- the work-stealing loop that replaces the reference's
// grid-stride loop (gpu/gpuwalk.hpp:200) and its one-walker-per-thread
// imbalance.  The loop body is one rejection-sampling trial, so lanes of a
// warp stay converged at trial granularity whatever their walk lengths.
//
// Walkers of the in-core kernel are generated from their id on the fly
// (engine/walk.hpp:32-49 for per-vertex init), so no walker record is read
// or written; per walker the kernel writes its path row (optional), length
// and 64-bit path hash.
#include <cuda_runtime.h>
#include <cstdint>
#include "gw_kernels.cuh"
#include "../../include/gowalker.h"

namespace gw {

// Words of a lane's walker parked in shared memory while its warp serves hard
// steps (kPkAstar receives the accepting attempt found for it).
enum ParkWord : int {
    kPkWid = 0, kPkPrev, kPkCur, kPkHop, kPkAttempt, kPkDeg, kPkPdeg, kPkHeadLo, kPkHeadHi, kPkPheadLo,
    kPkPheadHi, kPkHashLo, kPkHashHi, kPkThr0, kPkThr1, kPkThr2, kPkRx, kPkRy, kPkTrials, kPkAstar, kPkCount
};

// W: weighted Node2vec -- the trial's candidate is alias column r.x % deg,
// kept when float(r.w >> 8) * 2^-24 < its probability, else its alias (the
// alias tables of gw_weighted.cu); everything else is the unweighted step.
template <bool SOPR, bool PATHS, bool COOP, int MINB, bool W = false>
__global__ void __launch_bounds__(kWalkThreads, MINB) k_walk_incore(const __grid_constant__ IncoreArgs a)
{
    __shared__ uint32_t s_iv[kWalkThreads / 32][kCoopScratchWords];  // per-warp scratch of warp_first_accept
    __shared__ unsigned long long s_ws[kWalkThreads / 32][kWsCount];  // per-warp statistics
    __shared__ uint32_t s_park[COOP ? kWalkThreads / 32 : 1][kPkCount][32];  // lane state during hard steps
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt_mask = (1u << lane) - 1u;
    if (lane < kWsCount) s_ws[warp][lane] = 0;
    __syncwarp();
    const uint64_t *__restrict__ beg = a.beg;
    const uint32_t *__restrict__ csr = a.ix.csr;
    const uint32_t maxhops = a.c.maxhops;
    const uint32_t chunk = a.chunk ? a.chunk : kChunk;

    uint32_t q_next = 0, q_end = 0;  // warp-uniform claimed range
    bool exhausted = false;          // warp-uniform
    bool active = false;

    // Lane state.  Statistics live in s_ws and the path row is recomputed
    // from wid, so the registers hold only what the next trial reads.
    uint32_t wid = 0, prev = 0, cur = 0, hop = 0, attempt = 0;
    uint32_t deg = 0, pdeg = 0;
    uint64_t head = 0, phead = 0, h = 0;
    U4 r{0, 0, 0, 0};
    StepThr t{0.f, 0.f, 0.f};
    uint32_t n_trials = 0;  // trials not yet added to s_ws

    auto flush_trials = [&]() {
        atomicAdd(&s_ws[warp][kWsTrials], (unsigned long long)n_trials);
        n_trials = 0;
    };
    // A walker's steps are its hops: every accepted trial moves it one hop.
    auto finish = [&]() {
        a.hashes[wid - a.out_base] = h;
        a.lens[wid - a.out_base] = hop + 1;
        atomicAdd(&s_ws[warp][kWsSteps], (unsigned long long)hop);
        atomicAdd(&s_ws[warp][kWsDone], 1ull);
        atomicAdd(&s_ws[warp][kWsHash], (unsigned long long)h);
        flush_trials();
        active = false;
    };

    for (;;) {
        // Hand walkers to idle lanes.
        for (;;) {
            const unsigned need = __ballot_sync(0xFFFFFFFFu, !active);
            if (need == 0 || exhausted) break;
            if (q_next >= q_end) {
                unsigned long long base = 0;
                if (lane == 0) base = atomicAdd(&a.ctr[kCtrCursor], (unsigned long long)chunk);
                base = __shfl_sync(0xFFFFFFFFu, base, 0);
                if (base >= a.nwalkers) {
                    exhausted = true;
                    break;
                }
                q_next = (uint32_t)base;
                q_end = (uint32_t)min(base + chunk, (unsigned long long)a.nwalkers);
            }
            const uint32_t avail = q_end - q_next;
            const uint32_t rank = __popc(need & lt_mask);
            if (!active && rank < avail) {
                wid = a.wid_base + (q_next + rank) * a.wid_stride;
                const uint32_t src = walker_source(a.init, wid);
                prev = cur = src;
                hop = 0;
                h = hash_init(src);
                if (PATHS) a.paths[(uint64_t)(wid - a.out_base) * a.stride] = src;
                if (src >= a.nverts) {
                    atomicOr(a.err, kErrSource);
                    finish();
                } else if (maxhops == 0) {
                    finish();
                } else {
                    head = __ldg(beg + src);
                    deg = (uint32_t)(__ldg(beg + src + 1) - head);
                    if (deg == 0) {
                        finish();  // dead end (engine/engine.hpp:196-199)
                    } else {
                        phead = head;
                        pdeg = deg;
                        t = step_thresholds<SOPR>(a.c, deg, pdeg);
                        r = draw(a.c, wid, 0, 0);
                        attempt = 1;
                        active = true;
                    }
                }
            }
            q_next += min((uint32_t)__popc(need), avail);
        }
        if (!__any_sync(0xFFFFFFFFu, active)) break;

        // Walkers whose step keeps rejecting (a low-degree prev next to a hub
        // under SOPR) are served one at a time by the whole warp; the lane
        // then re-takes the accepting attempt below.  Meanwhile every lane's
        // walker is parked in shared memory: the registers go to the attempt
        // loop, and lane L's fields reach all lanes as broadcast loads.
        if (COOP) {
            const unsigned hm = __ballot_sync(0xFFFFFFFFu, active && attempt > kHardAttempts);
            if (hm) {
                uint32_t(*pk)[32] = s_park[COOP ? warp : 0];
                pk[kPkWid][lane] = wid;
                pk[kPkPrev][lane] = prev;
                pk[kPkCur][lane] = cur;
                pk[kPkHop][lane] = hop;
                pk[kPkAttempt][lane] = attempt;
                pk[kPkDeg][lane] = deg;
                pk[kPkPdeg][lane] = pdeg;
                pk[kPkHeadLo][lane] = (uint32_t)head;
                pk[kPkHeadHi][lane] = (uint32_t)(head >> 32);
                pk[kPkPheadLo][lane] = (uint32_t)phead;
                pk[kPkPheadHi][lane] = (uint32_t)(phead >> 32);
                pk[kPkHashLo][lane] = (uint32_t)h;
                pk[kPkHashHi][lane] = (uint32_t)(h >> 32);
                pk[kPkThr0][lane] = __float_as_uint(t.inv_deg);
                pk[kPkThr1][lane] = __float_as_uint(t.sum);
                pk[kPkThr2][lane] = __float_as_uint(t.t_prev);
                pk[kPkRx][lane] = r.x;
                pk[kPkRy][lane] = r.y;
                pk[kPkTrials][lane] = n_trials;
                __syncwarp();
                for (unsigned m = hm; m; m &= m - 1) {
                    const int L = __ffs(m) - 1;
                    const uint32_t p0 = pk[kPkAttempt][L] - 1;
                    const uint32_t Lprev = pk[kPkPrev][L], Lcur = pk[kPkCur][L], Lpdeg = pk[kPkPdeg][L];
                    const uint64_t hd = ((uint64_t)pk[kPkHeadHi][L] << 32) | pk[kPkHeadLo][L];
                    const uint64_t ph = ((uint64_t)pk[kPkPheadHi][L] << 32) | pk[kPkPheadLo][L];
                    const StepThr tl{__uint_as_float(pk[kPkThr0][L]), __uint_as_float(pk[kPkThr1][L]),
                                     __uint_as_float(pk[kPkThr2][L])};
                    uint32_t xs;
                    const uint32_t astar = warp_first_accept<SOPR>(a.c, tl, pk[kPkWid][L], pk[kPkHop][L], p0,
                                                                   kMaxAttempts, a.ix, hd, pk[kPkDeg][L], Lprev, Lcur,
                                                                   a.ix, ph, Lpdeg, s_iv[warp], &xs);
                    if (lane == 0) {
                        pk[kPkAstar][L] = astar;
                        const bool by_pos = Lpdeg < 32 && Lprev != Lcur;
                        atomicAdd(&s_ws[warp][by_pos ? kWsCoopSmall : kWsCoopLarge], 1ull);
                        atomicAdd(&s_ws[warp][by_pos ? kWsCoopSmallAtt : kWsCoopLargeAtt],
                                  (unsigned long long)(astar - p0 + 1));
                    }
                }
                __syncwarp();
                wid = pk[kPkWid][lane];
                prev = pk[kPkPrev][lane];
                cur = pk[kPkCur][lane];
                hop = pk[kPkHop][lane];
                attempt = pk[kPkAttempt][lane];
                deg = pk[kPkDeg][lane];
                pdeg = pk[kPkPdeg][lane];
                head = ((uint64_t)pk[kPkHeadHi][lane] << 32) | pk[kPkHeadLo][lane];
                phead = ((uint64_t)pk[kPkPheadHi][lane] << 32) | pk[kPkPheadLo][lane];
                h = ((uint64_t)pk[kPkHashHi][lane] << 32) | pk[kPkHashLo][lane];
                t.inv_deg = __uint_as_float(pk[kPkThr0][lane]);
                t.sum = __uint_as_float(pk[kPkThr1][lane]);
                t.t_prev = __uint_as_float(pk[kPkThr2][lane]);
                r.x = pk[kPkRx][lane];
                r.y = pk[kPkRy][lane];
                n_trials = pk[kPkTrials][lane];
                if ((hm >> lane) & 1u) {
                    const uint32_t astar = pk[kPkAstar][lane];
                    n_trials += astar - (attempt - 1);
                    if (astar >= kMaxAttempts) {
                        atomicOr(a.err, kErrTrials);
                        finish();
                    } else {
                        r = draw(a.c, wid, hop, astar);
                        attempt = astar + 1;
                    }
                }
                __syncwarp();
            }
        }
        if (!active) continue;

        // One rejection-sampling trial.
        const uint32_t pos = r.x % deg;
        const float rv = rand_val(r.y, thr_max<SOPR>(a.c, t));
        uint32_t col = pos;
        if constexpr (W) {
            const uint2 e = __ldg(a.alias + head + pos);
            if (!(__uint2float_rn(r.w >> 8) * 0x1p-24f < __uint_as_float(e.x))) col = e.y;
        }
        const uint32_t x = __ldg(csr + head + col);
        n_trials++;
        if (accept_candidate<SOPR>(a.c, t, rv, x, prev, cur, a.ix, phead, pdeg)) {
            hop++;
            h = hash_step(h, x);
            if (PATHS) a.paths[(uint64_t)(wid - a.out_base) * a.stride + hop] = x;
            if (n_trials & 0x80000000u) flush_trials();  // a step adds < 2^27: no wrap
            prev = cur;
            phead = head;
            pdeg = deg;
            cur = x;
            if (hop >= maxhops) {
                finish();
            } else if (x >= a.nverts) {
                atomicOr(a.err, kErrVertexRange);
                finish();
            } else if (a.c.term_prob > 0.0f) {
                r = draw(a.c, wid, hop, 0);
                attempt = 1;
                if (terminates(a.c, r.z)) {
                    finish();
                } else {
                    head = __ldg(beg + x);
                    deg = (uint32_t)(__ldg(beg + x + 1) - head);
                    if (deg == 0) finish();
                    else t = step_thresholds<SOPR>(a.c, deg, pdeg);
                }
            } else {
                head = __ldg(beg + x);
                const uint64_t tail = __ldg(beg + x + 1);
                r = draw(a.c, wid, hop, 0);
                attempt = 1;
                deg = (uint32_t)(tail - head);
                if (deg == 0) finish();
                else t = step_thresholds<SOPR>(a.c, deg, pdeg);
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
        if (COOP) {
            atomicAdd(&a.ctr[kCtrCoopSmall], s_ws[warp][kWsCoopSmall]);
            atomicAdd(&a.ctr[kCtrCoopSmallAtt], s_ws[warp][kWsCoopSmallAtt]);
            atomicAdd(&a.ctr[kCtrCoopLarge], s_ws[warp][kWsCoopLarge]);
            atomicAdd(&a.ctr[kCtrCoopLargeAtt], s_ws[warp][kWsCoopLargeAtt]);
        }
    }
}

// Memory-safety check of a resident CSR before any walk reads it: offsets
// non-decreasing and within [0, nedges], every neighbour id < nverts.
// (Adjacency order is a precondition -- the reference's `sorted` option --
// and affects results, not safety.)
__global__ void k_validate_csr(const uint64_t *__restrict__ beg, const uint32_t *__restrict__ csr,
                               uint32_t nverts, uint64_t nedges, uint32_t *err)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t t0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool bad = false;
    for (uint64_t v = t0; v < nverts; v += stride) {
        const uint64_t a = beg[v], b = beg[v + 1];
        bad |= (a > b) | (b > nedges);
    }
    for (uint64_t i = t0; i < nedges; i += stride) bad |= csr[i] >= nverts;
    if (__any_sync(0xFFFFFFFFu, bad) && (threadIdx.x & 31u) == 0) atomicOr(err, kErrVertexRange);
}

__global__ void k_sample_level(const uint32_t *__restrict__ src, uint64_t n, uint32_t *__restrict__ dst)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) dst[j] = src[32 * j];
}

cudaError_t launch_sample_level(const uint32_t *src, uint64_t n, uint32_t *dst, int num_sms, cudaStream_t s)
{
    k_sample_level<<<num_sms * 8, 256, 0, s>>>(src, n, dst);
    return cudaGetLastError();
}

cudaError_t launch_validate_csr(const uint64_t *beg, const uint32_t *csr, uint32_t nverts, uint64_t nedges,
                                uint32_t *err, int num_sms, cudaStream_t s)
{
    k_validate_csr<<<num_sms * 8, 256, 0, s>>>(beg, csr, nverts, nedges, err);
    return cudaGetLastError();
}

// Register-cap variants the autotuner chooses between: at 256 threads per CTA,
// 4, 5, 6 or 8 resident CTAs per SM (<= 64, 51, 40, 32 registers per thread).
template <int V>
struct MinBlocks;
template <> struct MinBlocks<0> { static constexpr int value = 4; };
template <> struct MinBlocks<1> { static constexpr int value = 5; };
template <> struct MinBlocks<2> { static constexpr int value = 6; };
template <> struct MinBlocks<3> { static constexpr int value = 8; };

template <bool SOPR, bool PATHS, bool COOP, int V, bool W = false>
static int grid_for(int num_sms)
{
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_walk_incore<SOPR, PATHS, COOP, MinBlocks<V>::value, W>,
                                                  kWalkThreads, 0);
    if (per_sm < 1) per_sm = 1;
    return per_sm * num_sms;
}

template <bool SOPR, bool PATHS, bool COOP, int V, bool W = false>
static void launch_one(const IncoreArgs &a, int grid, cudaStream_t s)
{
    k_walk_incore<SOPR, PATHS, COOP, MinBlocks<V>::value, W><<<grid, kWalkThreads, 0, s>>>(a);
}

template <bool SOPR, bool PATHS, bool COOP, bool W = false>
static int grid_v(int variant, int num_sms)
{
    if (variant == 0) return grid_for<SOPR, PATHS, COOP, 0, W>(num_sms);
    if (variant == 1) return grid_for<SOPR, PATHS, COOP, 1, W>(num_sms);
    if (variant == 2) return grid_for<SOPR, PATHS, COOP, 2, W>(num_sms);
    return grid_for<SOPR, PATHS, COOP, 3, W>(num_sms);
}

template <bool SOPR, bool PATHS, bool COOP, bool W = false>
static void launch_v(const IncoreArgs &a, int variant, int grid, cudaStream_t s)
{
    if (variant == 0) launch_one<SOPR, PATHS, COOP, 0, W>(a, grid, s);
    else if (variant == 1) launch_one<SOPR, PATHS, COOP, 1, W>(a, grid, s);
    else if (variant == 2) launch_one<SOPR, PATHS, COOP, 2, W>(a, grid, s);
    else launch_one<SOPR, PATHS, COOP, 3, W>(a, grid, s);
}

int incore_grid_weighted(bool paths, int variant, int num_sms)
{
    return paths ? grid_v<false, true, false, true>(variant, num_sms) : grid_v<false, false, false, true>(variant, num_sms);
}

cudaError_t launch_walk_incore_weighted(const IncoreArgs &a, int variant, int grid, cudaStream_t s)
{
    if (!a.alias) return cudaErrorInvalidValue;
    if (a.paths) launch_v<false, true, false, true>(a, variant, grid, s);
    else launch_v<false, false, false, true>(a, variant, grid, s);
    return cudaGetLastError();
}

int incore_grid(bool sopr, bool paths, bool coop, int variant, int num_sms)
{
    const int v = (sopr ? 4 : 0) | (paths ? 2 : 0) | (coop ? 1 : 0);
    switch (v) {
    case 0: return grid_v<false, false, false>(variant, num_sms);
    case 1: return grid_v<false, false, true>(variant, num_sms);
    case 2: return grid_v<false, true, false>(variant, num_sms);
    case 3: return grid_v<false, true, true>(variant, num_sms);
    case 4: return grid_v<true, false, false>(variant, num_sms);
    case 5: return grid_v<true, false, true>(variant, num_sms);
    case 6: return grid_v<true, true, false>(variant, num_sms);
    default: return grid_v<true, true, true>(variant, num_sms);
    }
}

cudaError_t launch_walk_incore(const IncoreArgs &a, bool sopr, bool coop, int variant, int grid, cudaStream_t s)
{
    const int v = (sopr ? 4 : 0) | (a.paths ? 2 : 0) | (coop ? 1 : 0);
    switch (v) {
    case 0: launch_v<false, false, false>(a, variant, grid, s); break;
    case 1: launch_v<false, false, true>(a, variant, grid, s); break;
    case 2: launch_v<false, true, false>(a, variant, grid, s); break;
    case 3: launch_v<false, true, true>(a, variant, grid, s); break;
    case 4: launch_v<true, false, false>(a, variant, grid, s); break;
    case 5: launch_v<true, false, true>(a, variant, grid, s); break;
    case 6: launch_v<true, true, false>(a, variant, grid, s); break;
    default: launch_v<true, true, true>(a, variant, grid, s); break;
    }
    return cudaGetLastError();
}

}  // namespace gw

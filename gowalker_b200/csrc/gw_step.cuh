// The second-order walk step, shared by every walk kernel.
//
// Semantics follow the reference CPU step (GOWalker engine/engine.hpp:158-404)
// with every draw taken from Philox4x32-10 keyed by the walk seed and
// countered by (walker id, hop, attempt, 0):
//   lane x -> rand_pos = x % deg                                (util/util.hpp:294)
//   lane y -> rand_val = float(y >> 8) * 2^-24 * max_val        (one fp32 multiply)
//   lane z -> SOPR/SOSR termination draw at hop >= 1 (attempt 0)
// Acceptance keeps the reference's precision mix:
//   Node2vec: fp32 thresholds 1/p, 1, 1/q, min and max of the three
//             (engine/engine.hpp:169-172, 209-258)
//   SOPR/SOSR: inv_deg = (float)((1-alpha)/deg) in fp64, inv_prev_deg =
//             alpha/(float)prev_deg in fp32 (323-326); the x==prev compare is
//             fp64 (341), the others fp32 (334, 368, 373).
// Every rounding step is an explicit _rn intrinsic so no contraction or
// fast-math flag can change a bit.
#pragma once
#include <cstdint>
#include "gw_philox.cuh"

namespace gw {

// Per-run constants, computed on the host.
struct StepConsts {
    uint32_t maxhops;
    uint32_t key0, key1;
    float n2v_maxv, n2v_minv;  // max / min of {1/p, 1/q, 1}
    float inv_p, inv_q;        // 1.0f/p, 1.0f/q
    float alpha;               // SOPR/SOSR
    float term_prob;           // 0 = no termination draw
    double one_m_alpha;        // 1.0 - (double)alpha
};

// Thresholds of one step (depend on deg / prev_deg for SOPR).
struct StepThr {
    float maxv, minv;
    float t_prev;      // Node2vec: x == prev accepts below 1/p
    float t_found;     // x in N(prev)
    float t_notfound;  // otherwise
    double t_prev_d;   // SOPR: x == prev accepts below (1-alpha)/deg in fp64
};

template <bool SOPR>
__device__ __forceinline__ StepThr step_thresholds(const StepConsts &c, uint64_t deg, uint64_t pdeg)
{
    StepThr t;
    if constexpr (!SOPR) {
        t.maxv = c.n2v_maxv;
        t.minv = c.n2v_minv;
        t.t_prev = c.inv_p;
        t.t_found = 1.0f;
        t.t_notfound = c.inv_q;
        t.t_prev_d = 0.0;
    } else {
        const double tp = __ddiv_rn(c.one_m_alpha, (double)deg);
        const float inv_deg = __double2float_rn(tp);
        const float inv_prev = __fdiv_rn(c.alpha, __ull2float_rn((unsigned long long)pdeg));
        const float sum = __fadd_rn(inv_deg, inv_prev);
        t.maxv = (inv_deg < sum) ? sum : inv_deg;   // std::max(inv_deg, sum)
        t.minv = (sum < inv_deg) ? sum : inv_deg;   // std::min(inv_deg, sum)
        t.t_prev = 0.f;
        t.t_found = sum;
        t.t_notfound = inv_deg;
        t.t_prev_d = tp;
    }
    return t;
}

__device__ __forceinline__ U4 draw(const StepConsts &c, uint32_t wid, uint32_t hop, uint32_t attempt)
{
    return philox4x32_10(wid, hop, attempt, kTagWalk, c.key0, c.key1);
}

__device__ __forceinline__ float rand_val(uint32_t y, float maxv)
{
    return __fmul_rn(__uint2float_rn(y >> 8) * 0x1p-24f, maxv);
}

__device__ __forceinline__ bool terminates(const StepConsts &c, uint32_t z)
{
    return c.term_prob > 0.0f && __uint2float_rn(z >> 8) * 0x1p-24f < c.term_prob;
}

// Membership of x in the sorted run base[0, n): plain binary search.
__device__ __forceinline__ bool search_sorted(const uint32_t *__restrict__ base, uint32_t n, uint32_t x)
{
    int32_t lo = 0, hi = (int32_t)n - 1;
    while (lo <= hi) {
        const int32_t mid = lo + ((hi - lo) >> 1);
        const uint32_t v = __ldg(base + mid);
        if (v == x) return true;
        if (v < x) lo = mid + 1;
        else hi = mid - 1;
    }
    return false;
}

// Acceptance of candidate x drawn with rand value rv (engine/engine.hpp:209-258,
// 334-375).  `searched` gets the membership result when a search ran.
template <bool SOPR>
__device__ __forceinline__ bool accept_candidate(const StepThr &t, float rv, uint32_t x, uint32_t prev,
                                                 uint32_t cur, const uint32_t *__restrict__ prev_adj,
                                                 uint32_t pdeg)
{
    if (rv <= t.minv) return true;
    if (x == prev) {
        if constexpr (SOPR) return (double)rv < t.t_prev_d;
        else return rv < t.t_prev;
    }
    // x is drawn from N(cur); when prev == cur the search must succeed.
    const bool found = (prev == cur) ? true : search_sorted(prev_adj, pdeg, x);
    return found ? (rv < t.t_found) : (rv < t.t_notfound);
}

// A walker whose step has already rejected this many attempts is served by
// the whole warp (warp_first_accept).
constexpr uint32_t kHardAttempts = 4;

__device__ __forceinline__ uint64_t shfl64(uint64_t v, int src)
{
    const uint32_t lo = __shfl_sync(0xFFFFFFFFu, (uint32_t)v, src);
    const uint32_t hi = __shfl_sync(0xFFFFFFFFu, (uint32_t)(v >> 32), src);
    return ((uint64_t)hi << 32) | lo;
}

template <typename T>
__device__ __forceinline__ T *shfl_ptr(T *p, int src)
{
    return reinterpret_cast<T *>(shfl64(reinterpret_cast<uint64_t>(p), src));
}

__device__ __forceinline__ StepThr shfl_thr(const StepThr &t, int src)
{
    StepThr o;
    o.maxv = __shfl_sync(0xFFFFFFFFu, t.maxv, src);
    o.minv = __shfl_sync(0xFFFFFFFFu, t.minv, src);
    o.t_prev = __shfl_sync(0xFFFFFFFFu, t.t_prev, src);
    o.t_found = __shfl_sync(0xFFFFFFFFu, t.t_found, src);
    o.t_notfound = __shfl_sync(0xFFFFFFFFu, t.t_notfound, src);
    o.t_prev_d = __shfl_sync(0xFFFFFFFFu, t.t_prev_d, src);
    return o;
}

// First index in the sorted run a[0, n) whose value is >= y.
__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t *__restrict__ a, uint32_t n, uint32_t y)
{
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(a + mid) < y) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Per-warp shared scratch of a cooperative step, in 32-bit words: run starts
// (32), run ends (32), and a filter of 2^kFilterBits buckets, one bit each.
constexpr uint32_t kFilterBits = 12;
constexpr int kCoopScratchWords = 64 + (1 << kFilterBits) / 32;

// Smallest k in [0, 2^24] for which `pred(k)` fails, where pred holds on a
// prefix of [0, 2^24).  rand_val(k << 8, maxv) is non-decreasing in k (an
// exact scaling followed by one rounded multiply by a positive constant), so
// every "rv <= T" / "rv < T" test of a step is such a prefix, and comparing
// k = y >> 8 with its bound gives the same verdict bit for bit.
template <class Pred>
__device__ __forceinline__ uint32_t rand_prefix(Pred pred)
{
    uint32_t lo = 0, hi = 1u << 24;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (pred(mid)) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Hard steps whose prev has fewer than 32 neighbours are decided without
// touching the candidate: a trial's verdict depends on x = cand[pos] only
// through "x == prev" and "x in N(prev)", i.e. through whether pos falls in
// the run of prev, or of some y in N(prev), inside the sorted N(cur).  Those
// runs are located once per step (one lower-bound search per lane).
//
// Trials then run on integers only.  The rand-value tests become bounds on
// k = y >> 8 (rand_prefix).  pos = x mod deg is never formed on the common
// path: with Lemire's fraction f = M*x mod 2^64 (M = ceil(2^64/deg)), pos =
// floor(f*deg / 2^64), so f lies in [pos, pos+1) * 2^64/deg and its top
// kFilterBits bits name a bucket of positions.  A per-warp bitmap marks every
// bucket a run can reach; a trial whose bucket is unmarked is in no run and
// its verdict is k < max(k_min, k_notfound).  Only marked buckets take the
// exact path (pos, run lookup in `iv`).
template <bool SOPR>
__device__ __forceinline__ uint32_t warp_first_accept_runs(const StepConsts &c, const StepThr &t, uint32_t wid,
                                                           uint32_t hop, uint32_t p0, uint32_t limit,
                                                           const uint32_t *__restrict__ cand, uint32_t deg,
                                                           uint32_t prev, const uint32_t *__restrict__ prev_adj,
                                                           uint32_t pdeg, uint32_t *iv, uint32_t *x_out)
{
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t *bm = iv + 64;
    constexpr uint32_t kFilterWords = (1u << kFilterBits) / 32;
    for (uint32_t w = lane; w < kFilterWords; w += 32) bm[w] = 0;
    // lane k < pdeg: run of N(prev)[k]; lane pdeg: run of prev
    uint32_t lo = 0, hi = 0;
    if (lane <= pdeg) {
        const uint32_t y = (lane < pdeg) ? __ldg(prev_adj + lane) : prev;
        lo = lower_bound_u32(cand, deg, y);
        hi = lo;
        while (hi < deg && __ldg(cand + hi) == y) hi++;
    }
    if (lane < pdeg) {
        iv[lane] = lo;
        iv[32 + lane] = hi;
    }
    const uint64_t M = fastmod_magic(deg);
    __syncwarp();
    if (hi > lo) {
        // buckets floor(p * 2^B / deg) for p in [lo, hi], widened by one below
        // (umul64hi(M, P) exceeds floor(P / deg) by at most one); deg = 1 has
        // M = 0 and covers everything.
        uint32_t b0 = 0, b1 = (1u << kFilterBits) - 1;
        if (deg > 1) {
            const uint32_t e0 = (uint32_t)__umul64hi(M, (uint64_t)lo << kFilterBits);
            const uint32_t e1 = (uint32_t)__umul64hi(M, (uint64_t)hi << kFilterBits);
            b0 = e0 > 0 ? e0 - 1 : 0;
            b1 = min(e1, b1);
        }
        for (uint32_t w = b0 >> 5; w <= (b1 >> 5); ++w) {
            const uint32_t from = (w == (b0 >> 5)) ? (b0 & 31u) : 0u;
            const uint32_t to = (w == (b1 >> 5)) ? (b1 & 31u) : 31u;
            const uint32_t mask = (0xFFFFFFFFu >> (31u - to)) & (0xFFFFFFFFu << from);
            atomicOr(bm + w, mask);
        }
    }
    // integer bounds of the four rand-value tests, one per lane of a quad
    uint32_t kq;
    {
        const uint32_t which = lane & 3u;
        kq = rand_prefix([&](uint32_t k) {
            const float rv = rand_val(k << 8, t.maxv);
            bool prev_ok;
            if constexpr (SOPR) prev_ok = (double)rv < t.t_prev_d;
            else prev_ok = rv < t.t_prev;
            return which == 0 ? (rv <= t.minv) : which == 1 ? prev_ok : which == 2 ? (rv < t.t_found)
                                                                                    : (rv < t.t_notfound);
        });
    }
    const uint32_t k_min = __shfl_sync(0xFFFFFFFFu, kq, 0), k_prev = __shfl_sync(0xFFFFFFFFu, kq, 1);
    const uint32_t k_found = __shfl_sync(0xFFFFFFFFu, kq, 2), k_nf = __shfl_sync(0xFFFFFFFFu, kq, 3);
    const uint32_t k_fast = max(k_min, k_nf);
    const uint32_t plo = __shfl_sync(0xFFFFFFFFu, lo, (int)pdeg), phi = __shfl_sync(0xFFFFFFFFu, hi, (int)pdeg);
    const uint32_t m_lo = (uint32_t)M, m_hi = (uint32_t)(M >> 32);
    __syncwarp();

    // exact verdict of a trial whose bucket is marked
    auto exact = [&](uint32_t x, uint32_t k) -> bool {
        if (k < k_min) return true;
        const uint32_t pos = fastmod(x, M, deg);
        if (pos >= plo && pos < phi) return k < k_prev;
        // last run whose start is <= pos (runs are in N(prev) order, so sorted)
        int r = -1;
        uint32_t a = 0, b = pdeg;
        while (a < b) {
            const uint32_t m = (a + b) >> 1;
            if (iv[m] <= pos) {
                r = (int)m;
                a = m + 1;
            } else {
                b = m;
            }
        }
        const bool found = r >= 0 && pos < iv[32 + r];
        return found ? (k < k_found) : (k < k_nf);
    };
    auto judge = [&](uint32_t att, uint32_t &xr) -> bool {
        if (att >= limit) return false;
        const U4 r = draw(c, wid, hop, att);
        xr = r.x;
        const uint32_t k = r.y >> 8;
        const uint32_t b = (m_hi * r.x + __umulhi(m_lo, r.x)) >> (32 - kFilterBits);
        if ((bm[b >> 5] >> (b & 31u)) & 1u) return exact(r.x, k);
        return k < k_fast;
    };
    // 64 attempts per round, two independent Philox chains per lane
    for (uint32_t base = p0; base < limit; base += 64) {
        uint32_t x0 = 0, x1 = 0;
        const bool acc0 = judge(base + lane, x0);
        const bool acc1 = judge(base + 32 + lane, x1);
        const unsigned m0 = __ballot_sync(0xFFFFFFFFu, acc0);
        const unsigned m1 = __ballot_sync(0xFFFFFFFFu, acc1);
        if (m0 | m1) {
            const bool first_half = m0 != 0;
            const int f = __ffs(first_half ? m0 : m1) - 1;
            const uint32_t xf = __shfl_sync(0xFFFFFFFFu, first_half ? x0 : x1, f);
            *x_out = __ldg(cand + fastmod(xf, M, deg));
            __syncwarp();
            return base + (first_half ? 0u : 32u) + (uint32_t)f;
        }
    }
    *x_out = 0;
    __syncwarp();
    return limit;
}

// All 32 lanes, with identical (broadcast) arguments, evaluate attempts
// p0+lane, p0+32+lane, ... of one walker's step and return the first accepting
// attempt in attempt order -- the one a single thread evaluating them one by
// one would take -- and its candidate in *x_out.  Returns `limit` if none of
// the attempts below `limit` accepts.
template <bool SOPR>
__device__ __forceinline__ uint32_t warp_first_accept(const StepConsts &c, const StepThr &t, uint32_t wid,
                                                      uint32_t hop, uint32_t p0, uint32_t limit,
                                                      const uint32_t *__restrict__ cand, uint32_t deg,
                                                      uint32_t prev, uint32_t cur,
                                                      const uint32_t *__restrict__ prev_adj, uint32_t pdeg,
                                                      uint32_t *iv, uint32_t *x_out)
{
    if (pdeg < 32 && prev != cur)
        return warp_first_accept_runs<SOPR>(c, t, wid, hop, p0, limit, cand, deg, prev, prev_adj, pdeg, iv, x_out);
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t M = fastmod_magic(deg);
    for (uint32_t base = p0; base < limit; base += 32) {
        const uint32_t att = base + lane;
        bool acc = false;
        uint32_t x = 0;
        if (att < limit) {
            const U4 r = draw(c, wid, hop, att);
            const uint32_t pos = fastmod(r.x, M, deg);
            const float rv = rand_val(r.y, t.maxv);
            x = __ldg(cand + pos);
            acc = accept_candidate<SOPR>(t, rv, x, prev, cur, prev_adj, pdeg);
        }
        const unsigned m = __ballot_sync(0xFFFFFFFFu, acc);
        if (m) {
            const int f = __ffs(m) - 1;
            *x_out = __shfl_sync(0xFFFFFFFFu, x, f);
            return base + (uint32_t)f;
        }
    }
    *x_out = 0;
    return limit;
}

}  // namespace gw

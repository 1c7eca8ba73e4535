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
// fast-math flag can change a bit.  The fp64 compare is carried out in fp32
// without changing a verdict: for a float rv and a double T,
// (double)rv < T  <=>  rv < RU(T), RU(T) the smallest float >= T (if T is a
// float, RU(T) = T; otherwise every float below RU(T) is below T).
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
    uint32_t rk0[10], rk1[10]; // Philox key schedule: round r uses key + r * Weyl constant
};

// Per-step thresholds.  Node2vec's are run constants and live in
// StepConsts; SOPR/SOSR's depend on deg and prev_deg and take three floats.
struct StepThr {
    float inv_deg;  // (float)((1-alpha)/deg), divided in fp64
    float sum;      // inv_deg + alpha/(float)prev_deg
    float t_prev;   // RU((1-alpha)/deg): x == prev accepts iff rv < t_prev
};

template <bool SOPR>
__device__ __forceinline__ StepThr step_thresholds(const StepConsts &c, uint64_t deg, uint64_t pdeg)
{
    StepThr t{0.f, 0.f, 0.f};
    if constexpr (SOPR) {
        const double tp = __ddiv_rn(c.one_m_alpha, (double)deg);
        t.inv_deg = __double2float_rn(tp);
        const float inv_prev = __fdiv_rn(c.alpha, __ull2float_rn((unsigned long long)pdeg));
        t.sum = __fadd_rn(t.inv_deg, inv_prev);
        t.t_prev = __double2float_ru(tp);
    }
    return t;
}

// The five thresholds of a trial (engine/engine.hpp:209-258, 334-375).
template <bool SOPR>
__device__ __forceinline__ float thr_max(const StepConsts &c, const StepThr &t)
{
    if constexpr (SOPR) return (t.inv_deg < t.sum) ? t.sum : t.inv_deg;  // std::max(inv_deg, sum)
    else return c.n2v_maxv;
}
template <bool SOPR>
__device__ __forceinline__ float thr_min(const StepConsts &c, const StepThr &t)
{
    if constexpr (SOPR) return (t.sum < t.inv_deg) ? t.sum : t.inv_deg;  // std::min(inv_deg, sum)
    else return c.n2v_minv;
}
template <bool SOPR>
__device__ __forceinline__ float thr_prev(const StepConsts &c, const StepThr &t)
{
    if constexpr (SOPR) return t.t_prev;
    else return c.inv_p;
}
template <bool SOPR>
__device__ __forceinline__ float thr_found(const StepConsts &c, const StepThr &t)
{
    if constexpr (SOPR) return t.sum;
    else return 1.0f;
}
template <bool SOPR>
__device__ __forceinline__ float thr_notfound(const StepConsts &c, const StepThr &t)
{
    if constexpr (SOPR) return t.inv_deg;
    else return c.inv_q;
}

// The walk draw.  The key schedule comes precomputed in the kernel's
// parameters, so each round is two wide multiplies and two three-way xors
// with a constant operand.
__device__ __forceinline__ U4 draw(const StepConsts &c, uint32_t wid, uint32_t hop, uint32_t attempt)
{
    return philox4x32_10_sched(wid, hop, attempt, kTagWalk, c.rk0, c.rk1);
}

__device__ __forceinline__ float rand_val(uint32_t y, float maxv)
{
    return __fmul_rn(__uint2float_rn(y >> 8) * 0x1p-24f, maxv);
}

__device__ __forceinline__ bool terminates(const StepConsts &c, uint32_t z)
{
    return c.term_prob > 0.0f && __uint2float_rn(z >> 8) * 0x1p-24f < c.term_prob;
}

// Neighbour array of the graph (or of one block) with its sample levels:
// lvl[L-1][j] = csr[j * 32^L].  Inside one vertex's sorted neighbours the
// entries of level L are every 32^L-th neighbour (by global position), so a
// search walks down the levels, each a binary search over at most 65
// contiguous entries (one or two lines, then L1 hits), and ends in fewer than
// 32 neighbours: about one new line per level where a plain binary search
// takes a miss per halving.  nlvl = 0 is a plain binary search.
constexpr int kIdxLevels = 6;
struct CsrIndex {
    const uint32_t *csr;
    const uint32_t *lvl[kIdxLevels];
    uint32_t nlvl;
};

// First position p in [lo, hi) with csr[p] >= y, or hi (csr[lo, hi) sorted,
// hi - lo < 2^32).  Ranges of at most 64 go straight to the last binary
// search; longer ones start at the highest level with more than two entries
// inside (level L qualifies when hi - lo > 2 * 32^L).
__device__ __forceinline__ uint64_t csr_lower_bound(const CsrIndex &ix, uint64_t lo, uint64_t hi, uint32_t y)
{
    if (hi - lo > 64 && ix.nlvl != 0) {
        int L = min((int)ix.nlvl, (62 - __clzll((long long)(hi - lo))) / 5);  // (floor(log2 n) - 1) / 5
        for (; L >= 1; --L) {
            const uint32_t sh = 5u * (uint32_t)L;
            if (hi - lo <= (2ull << sh)) continue;
            const uint32_t *__restrict__ g = ix.lvl[L - 1];
            const uint64_t j0 = (lo + (1ull << sh) - 1) >> sh, j1 = (hi - 1) >> sh;
            uint32_t a = 0, b = (uint32_t)(j1 - j0) + 1;  // first j in [j0, j1] with csr[j << sh] >= y
            while (a < b) {
                const uint32_t m = (a + b) >> 1;
                if (__ldg(g + j0 + m) < y) a = m + 1;
                else b = m;
            }
            if (a > 0) lo = ((j0 + a - 1) << sh) + 1;
            if (j0 + a <= j1) hi = (j0 + a) << sh;
        }
    }
    const uint32_t *__restrict__ p = ix.csr + lo;
    uint32_t a = 0, b = (uint32_t)(hi - lo);
    while (a < b) {
        const uint32_t m = (a + b) >> 1;
        if (__ldg(p + m) < y) a = m + 1;
        else b = m;
    }
    return lo + a;
}

// Membership of x in the sorted csr[lo, lo + n).
__device__ __forceinline__ bool csr_contains(const CsrIndex &ix, uint64_t lo, uint32_t n, uint32_t x)
{
    const uint64_t p = csr_lower_bound(ix, lo, lo + n, x);
    return p < lo + n && __ldg(ix.csr + p) == x;
}

// Acceptance of candidate x drawn with rand value rv (engine/engine.hpp:209-258,
// 334-375); N(prev) is pix.csr[phead, phead + pdeg).
template <bool SOPR>
__device__ __forceinline__ bool accept_candidate(const StepConsts &c, const StepThr &t, float rv, uint32_t x,
                                                 uint32_t prev, uint32_t cur, const CsrIndex &pix, uint64_t phead,
                                                 uint32_t pdeg)
{
    if (rv <= thr_min<SOPR>(c, t)) return true;
    if (x == prev) return rv < thr_prev<SOPR>(c, t);
    // x is drawn from N(cur); when prev == cur the search must succeed.
    const bool found = (prev == cur) ? true : csr_contains(pix, phead, pdeg, x);
    return found ? (rv < thr_found<SOPR>(c, t)) : (rv < thr_notfound<SOPR>(c, t));
}

// The same verdict without N(prev), for a walker whose previous block is not
// resident: 1 accept, 0 reject, -1 when it depends on x in N(prev) (the
// found and not-found thresholds disagree at rv).
template <bool SOPR>
__device__ __forceinline__ int accept_without_prev(const StepConsts &c, const StepThr &t, float rv, uint32_t x,
                                                   uint32_t prev, uint32_t cur)
{
    if (rv <= thr_min<SOPR>(c, t)) return 1;
    if (x == prev) return rv < thr_prev<SOPR>(c, t) ? 1 : 0;
    const bool af = rv < thr_found<SOPR>(c, t);
    if (prev == cur) return af ? 1 : 0;
    const bool an = rv < thr_notfound<SOPR>(c, t);
    return af == an ? (af ? 1 : 0) : -1;
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

template <bool SOPR>
__device__ __forceinline__ StepThr shfl_thr(const StepThr &t, int src)
{
    StepThr o{0.f, 0.f, 0.f};
    if constexpr (SOPR) {
        o.inv_deg = __shfl_sync(0xFFFFFFFFu, t.inv_deg, src);
        o.sum = __shfl_sync(0xFFFFFFFFu, t.sum, src);
        o.t_prev = __shfl_sync(0xFFFFFFFFu, t.t_prev, src);
    }
    return o;
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

// Integer bounds of a step's four rand-value tests, found by the whole warp:
// lanes 8w..8w+7 compute bound w (0: rv <= min, 1: rv < prev, 2: rv < found,
// 3: rv < notfound) and lane 8w returns it.  Each group tests the eight k
// around the estimate bound / maxv * 2^24, within two of the true bound when
// maxv and the bound are normal floats (one rounding of k * 2^-24 * maxv moves
// it by at most half an ulp, i.e. by at most one step of k); a group whose
// window does not bracket the bound falls back to rand_prefix.
template <bool SOPR>
__device__ __forceinline__ uint32_t rand_bounds(const StepConsts &c, const StepThr &t)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t which = lane >> 3;
    const float maxv = thr_max<SOPR>(c, t);
    const float bound = which == 0 ? thr_min<SOPR>(c, t) : which == 1 ? thr_prev<SOPR>(c, t)
                      : which == 2 ? thr_found<SOPR>(c, t) : thr_notfound<SOPR>(c, t);
    auto pred = [&](uint32_t k) {
        const float rv = rand_val(k << 8, maxv);
        return which == 0 ? (rv <= bound) : (rv < bound);
    };
    const double est = __dmul_rn(__ddiv_rn((double)bound, (double)maxv), 16777216.0);
    const bool est_ok = est >= 0.0 && est <= 16777216.0;  // false for NaN
    const int64_t base = (est_ok ? (int64_t)est : 0) - 4;
    const int64_t kc = base + (int64_t)(lane & 7u);
    const bool q = kc < 0 ? true : (kc >= (1 << 24) ? false : pred((uint32_t)kc));
    const unsigned g = (__ballot_sync(0xFFFFFFFFu, q) >> (lane & 24u)) & 0xFFu;
    // a bracket: true at the first candidate, false at the last, ones then zeros
    if (est_ok && (g & 1u) && !(g & 0x80u) && g == (1u << __popc(g)) - 1u) return (uint32_t)(base + __popc(g));
    return rand_prefix(pred);
}

// Hard steps whose prev has fewer than 32 neighbours are decided without
// touching the candidate: a trial's verdict depends on x = N(cur)[pos] only
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
                                                           const CsrIndex &cix, uint64_t head, uint32_t deg,
                                                           uint32_t prev, const CsrIndex &pix, uint64_t phead,
                                                           uint32_t pdeg, uint32_t *iv, uint32_t *x_out)
{
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t *bm = iv + 64;
    constexpr uint32_t kFilterWords = (1u << kFilterBits) / 32;
    for (uint32_t w = lane; w < kFilterWords; w += 32) bm[w] = 0;
    // lane k < pdeg: run of N(prev)[k]; lane pdeg: run of prev
    uint32_t lo = 0, hi = 0;
    if (lane <= pdeg) {
        const uint32_t y = (lane < pdeg) ? __ldg(pix.csr + phead + lane) : prev;
        lo = (uint32_t)(csr_lower_bound(cix, head, head + deg, y) - head);
        hi = lo;
        while (hi < deg && __ldg(cix.csr + head + hi) == y) hi++;
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
    // integer bounds of the four rand-value tests
    const uint32_t kq = rand_bounds<SOPR>(c, t);
    const uint32_t k_min = __shfl_sync(0xFFFFFFFFu, kq, 0), k_prev = __shfl_sync(0xFFFFFFFFu, kq, 8);
    const uint32_t k_found = __shfl_sync(0xFFFFFFFFu, kq, 16), k_nf = __shfl_sync(0xFFFFFFFFu, kq, 24);
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
            *x_out = __ldg(cix.csr + head + fastmod(xf, M, deg));
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
                                                      const CsrIndex &cix, uint64_t head, uint32_t deg,
                                                      uint32_t prev, uint32_t cur, const CsrIndex &pix,
                                                      uint64_t phead, uint32_t pdeg, uint32_t *iv, uint32_t *x_out)
{
    if (pdeg < 32 && prev != cur)
        return warp_first_accept_runs<SOPR>(c, t, wid, hop, p0, limit, cix, head, deg, prev, pix, phead, pdeg, iv,
                                            x_out);
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t M = fastmod_magic(deg);
    const float maxv = thr_max<SOPR>(c, t);
    for (uint32_t base = p0; base < limit; base += 32) {
        const uint32_t att = base + lane;
        bool acc = false;
        uint32_t x = 0;
        if (att < limit) {
            const U4 r = draw(c, wid, hop, att);
            const uint32_t pos = fastmod(r.x, M, deg);
            const float rv = rand_val(r.y, maxv);
            x = __ldg(cix.csr + head + pos);
            // N(prev) serves every attempt of the step and stays in L1: a
            // plain binary search beats the sample levels here.
            acc = accept_candidate<SOPR>(c, t, rv, x, prev, cur, CsrIndex{pix.csr, {}, 0}, phead, pdeg);
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

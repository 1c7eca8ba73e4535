/*
 * gw_oracle.c -- CPU oracle for the GOWalker second-order walk step.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links or calls this file:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg and
 * `--impl reference` arm load it, and only as the checker or the timed CPU
 * baseline.
 *
 * What it restates (reference file:line, paths inside the GOWalker project):
 *   - Node2vec CPU step   engine/engine.hpp:158-287  (sidewalkupdate)
 *   - SOPR/SOSR CPU step  engine/engine.hpp:289-404  (SOPR_sidewalkupdate)
 *   - binary search of the candidate in N(prev)  engine/engine.hpp:225-243
 *   - dead-end rule (deg == 0 -> hop = maxhop-1, next vertex 0)
 *                                              engine/engine.hpp:196-199
 *   - walker init, Node2vec: id = v*wps + i     engine/walk.hpp:32-49, 294-321
 *   - walker init, SOPR (all at vertex 1) / SOSR (half at 1, half at 3)
 *                                              engine/walk.hpp:275-293, 355-384
 *
 * The reference draws from RandNum::inlineRandPair (util/util.hpp:291-301),
 * a stateful xoroshiro128+ seeded from time(NULL).  Here every draw comes from
 * Philox4x32-10 (Salmon et al., SC'11) keyed by the walk seed and countered by
 * (walker id, hop, attempt, 0):
 *   lane0 -> rand_pos = lane0 % deg                     (util/util.hpp:294)
 *   lane1 -> rand_val = float(lane1 >> 8) * 2^-24 * max_val   (one fp32 multiply)
 *   lane2 -> SOPR/SOSR geometric termination draw at hop >= 1 (not in the
 *            reference, whose walks have fixed length)
 * A second keying, (walker id, running trial index), matches the shim used
 * by oracle/ref_step_harness.cu, which drives the reference's own
 * sidewalkupdate for the differential test.
 *
 * The floating-point mix of the reference is kept exactly:
 *   Node2vec: inv_p = 1.0f/p, inv_q = 1.0f/q, all compares in fp32
 *             (engine.hpp:169-172, 209, 216, 247, 254).
 *   SOPR:     inv_deg = (float)((1.0 - alpha)/deg) in fp64, inv_prev_deg =
 *             alpha / (float)prev_deg in fp32 (engine.hpp:323-326); the x==prev
 *             compare is fp64 against (1.0-alpha)/deg (engine.hpp:341), the
 *             others fp32 (engine.hpp:334, 368, 373).
 * Build with -ffp-contract=off so no multiply-add is fused.
 *
 * Besides paths, the oracle counts the memory the step needs, in 32-byte
 * sectors: the (beg[cur], beg[cur+1]) pair, one csr sector per trial, and the
 * distinct sectors touched by the binary search of each trial.  These give the
 * algorithmic bytes per step used for the roofline.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

#define PHILOX_M0 0xD2511F53u
#define PHILOX_M1 0xCD9E8D57u
#define PHILOX_W0 0x9E3779B9u
#define PHILOX_W1 0xBB67AE85u

#define FNV_OFFSET 0xcbf29ce484222325ull
#define FNV_PRIME 0x100000001b3ull

#define RMAT_TAG 0x524D4154u /* 'RMAT' */
#define INIT_TAG 0x494E4954u /* 'INIT' */

enum { ALG_NODE2VEC = 0, ALG_SOPR = 1, ALG_SOSR = 2 };
enum { INIT_PER_VERTEX = 0, INIT_SINGLE_SOURCE = 1, INIT_RANDOM = 2 };
enum { KEY_HOP_ATTEMPT = 0, KEY_TRIAL = 1 };

/* Philox4x32-10: ten rounds of the published S-box-free bijection, key bumped
 * by the Weyl constants between rounds. */
void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)PHILOX_M0 * c0;
        uint64_t p1 = (uint64_t)PHILOX_M1 * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += PHILOX_W0;
        k1 += PHILOX_W1;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static inline void draw4(uint64_t seed, uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t out[4])
{
    uint32_t ctr[4] = {a, b, c, d};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    oracle_philox4x32_10(ctr, key, out);
}

/* ---------------------------------------------------------------- R-MAT */

/* R-MAT edge sample e at `scale` levels.  Level l uses lane (l & 3) of the
 * Philox call (e_lo, e_hi, l >> 2, 'RMAT').  thr[] are the cumulative quadrant
 * thresholds a, a+b, a+b+c scaled to 2^32 (integers, so CPU and GPU agree). */
static inline void rmat_one(uint32_t scale, uint64_t e, const uint32_t thr[3], uint64_t seed,
                            uint32_t *src, uint32_t *dst)
{
    uint32_t s = 0, d = 0, r[4];
    for (uint32_t l = 0; l < scale; ++l) {
        if ((l & 3u) == 0)
            draw4(seed, (uint32_t)e, (uint32_t)(e >> 32), l >> 2, RMAT_TAG, r);
        uint32_t u = r[l & 3u];
        uint32_t sb, db;
        if (u < thr[0]) { sb = 0; db = 0; }
        else if (u < thr[1]) { sb = 0; db = 1; }
        else if (u < thr[2]) { sb = 1; db = 0; }
        else { sb = 1; db = 1; }
        s = (s << 1) | sb;
        d = (d << 1) | db;
    }
    *src = s;
    *dst = d;
}

/* Raw samples e in [first, first+count). */
void oracle_rmat_edges(uint32_t scale, uint64_t first, uint64_t count, const uint32_t thr[3],
                       uint64_t seed, uint32_t *src, uint32_t *dst, int nthreads)
{
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)count; ++i)
        rmat_one(scale, first + (uint64_t)i, thr, seed, &src[i], &dst[i]);
}

#define WEB_TAG 0x57454230u  /* 'WEB0' */
#define WDEG_TAG 0x57444547u /* 'WDEG' */

/* Fixed-step ln(z * 2^-32) and exp(x <= 0) in IEEE double, the device's
 * fm_log_u32 / fm_exp_nonpos step for step (this file builds with
 * -ffp-contract=off, so every operation rounds to nearest on its own). */
static double fm_log_u32(uint32_t z)
{
    if (z == 0) return -INFINITY;
    int e = 31 - __builtin_clz(z);
    double m = (double)z * ldexp(1.0, -e);
    if (m >= 1.4142135623730951) {
        m = m * 0.5;
        e += 1;
    }
    const double s = (m - 1.0) / (m + 1.0);
    const double s2 = s * s;
    double q = 1.0 / 23;
    for (int j = 10; j >= 0; --j) q = 1.0 / (2 * j + 1) + s2 * q;
    const double lnm = (2.0 * s) * q;
    const double ex = (double)(e - 32);
    return (ex * 0.693145751953125 + ex * 1.4286068203094172e-06) + lnm;
}

static double fm_exp_nonpos(double x)
{
    if (!(x > -700.0)) return 0.0;
    if (x >= 0.0) return 1.0;
    const double nd = nearbyint(x * 1.4426950408889634);
    const double r = (x - nd * 0.693145751953125) - nd * 1.4286068203094172e-06;
    double q = 1.0;
    for (int k = 13; k >= 1; --k) q = 1.0 + (r * q) * (1.0 / k);
    return ldexp(q, (int)nd);
}

/* Web-shaped graph (gw_web_csr restated).  Out-degree of v:
 * floor(dmin / u^(1/tail)) capped at max_degree, u = Philox(v, 0, 0, 'WDEG')
 * lane 0 / 2^32 (0 read as 1). */
void oracle_web_degrees(uint32_t nverts, double dmin, double tail, uint32_t max_degree, uint64_t seed,
                        uint64_t *deg)
{
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < (int64_t)nverts; ++v) {
        uint32_t r[4];
        draw4(seed, (uint32_t)v, 0u, 0u, WDEG_TAG, r);
        const uint32_t z = r[0] ? r[0] : 1u;
        const double pw = fm_exp_nonpos(fm_log_u32(z) / tail);
        const double d = dmin / pw;
        deg[v] = d >= (double)max_degree ? max_degree : (uint64_t)d;
    }
}

/* Edge j of v at estart[v] + j: Philox(j, v, 0, 'WEB0') lane 0 % 1000 <
 * local_permille makes it local (v + o, o uniform over [-window, -1] u
 * [1, window] from lane 1, clipped); otherwise the destination takes `scale`
 * bits from R-MAT's destination marginal (quadrants b, d; level l from lane
 * l & 3 of Philox(j, v, 1 + l/4, 'WEB0')).  dst = 0xFFFFFFFF marks a dropped
 * edge (self loop or destination >= nverts). */
void oracle_web_edges(uint32_t scale, uint32_t nverts, const uint32_t thr[3], uint32_t local_permille,
                      uint32_t window, uint64_t seed, const uint64_t *estart, uint32_t *src, uint32_t *dst)
{
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t v = 0; v < (int64_t)nverts; ++v) {
        for (uint64_t j = 0; j < estart[v + 1] - estart[v]; ++j) {
            uint32_t r[4], d;
            draw4(seed, (uint32_t)j, (uint32_t)v, 0u, WEB_TAG, r);
            if (r[0] % 1000u < local_permille) {
                int64_t o = (int64_t)(r[1] % (2u * window)) - (int64_t)window;
                if (o >= 0) o += 1;
                int64_t t = v + o;
                t = t < 0 ? 0 : (t >= (int64_t)nverts ? (int64_t)nverts - 1 : t);
                d = (uint32_t)t;
            } else {
                uint32_t q[4] = {0, 0, 0, 0};
                d = 0;
                for (uint32_t l = 0; l < scale; ++l) {
                    if ((l & 3u) == 0) draw4(seed, (uint32_t)j, (uint32_t)v, 1u + (l >> 2), WEB_TAG, q);
                    const uint32_t u = q[l & 3u];
                    d = (d << 1) | (((u >= thr[0] && u < thr[1]) || u >= thr[2]) ? 1u : 0u);
                }
            }
            const uint64_t e = estart[v] + j;
            src[e] = (uint32_t)v;
            dst[e] = (d < nverts && d != (uint32_t)v) ? d : 0xFFFFFFFFu;
        }
    }
}

/* ---------------------------------------------------------------- walks */

typedef struct {
    uint32_t algo;       /* ALG_* (AlgorithmType order, api/types.hpp:27) */
    uint32_t maxhops;    /* walk length (the "length" option) */
    float p, q, alpha;   /* Node2vec p, q; SOPR/SOSR alpha */
    float term_prob;     /* geometric termination per step at hop >= 1; 0 = off */
    uint64_t seed;       /* walk seed (Philox key) */
    uint32_t keying;     /* KEY_* */
    uint32_t init_mode;  /* INIT_* */
    uint32_t wps;        /* walkers per source vertex (INIT_PER_VERTEX) */
    uint32_t numwalks;   /* total walkers (INIT_SINGLE_SOURCE / INIT_RANDOM) */
} oracle_cfg;

typedef struct {
    uint64_t steps;          /* real moves (path entries after the source) */
    uint64_t trials;         /* rejection-sampling attempts */
    uint64_t probes;         /* binary-search reads of N(prev) */
    uint64_t search_sectors; /* distinct 32-B sectors per trial's search, summed */
    uint64_t off_sectors;    /* sectors of (beg[cur], beg[cur+1]) per step */
    uint64_t dead_ends;      /* walks stopped by the deg==0 rule */
    uint64_t terminated;     /* walks stopped by the termination draw */
    uint64_t acc_sectors;    /* distinct sectors of the accepted trial's search of N(prev), when its
                                verdict needed one: with the offsets and the accepted candidate, the
                                bytes a step cannot avoid reading */
} oracle_stats;

/* Source vertex of walker `wid` (engine/walk.hpp init kernels). */
uint32_t oracle_walker_source(const oracle_cfg *c, uint32_t nverts, uint32_t wid)
{
    switch (c->init_mode) {
    case INIT_PER_VERTEX:
        return wid / c->wps;
    case INIT_SINGLE_SOURCE:
        if (c->algo == ALG_SOSR)
            return wid < c->numwalks / 2 ? 1u : 3u;
        return 1u;
    default: {
        uint32_t r[4];
        draw4(c->seed, wid, 0xFFFFFFFFu, 0, INIT_TAG, r);
        return r[0] % nverts;
    }
    }
}

typedef struct {
    uint32_t deg;
    uint32_t maxv_bits;
    uint32_t pos;
    uint32_t rv_bits;
} oracle_trial;

static inline uint32_t f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

/* Membership of x in the sorted run csr[lo, hi), by the reference's binary
 * search (engine/engine.hpp:225-243), counting reads and distinct sectors. */
static inline int search_sorted(const uint32_t *csr, uint64_t lo, uint64_t hi, uint32_t x,
                                uint64_t *probes, uint64_t *sectors)
{
    int64_t left = (int64_t)lo, right = (int64_t)hi - 1;
    uint64_t seen[72];
    int nseen = 0;
    while (left <= right) {
        int64_t mid = left + ((right - left) >> 1);
        uint64_t sec = ((uint64_t)mid * 4u) >> 5;
        int dup = 0;
        for (int i = 0; i < nseen; ++i)
            if (seen[i] == sec) { dup = 1; break; }
        if (!dup && nseen < 72) seen[nseen++] = sec;
        (*probes)++;
        uint32_t v = csr[mid];
        if (v == x) { *sectors += (uint64_t)nseen; return 1; }
        if (v < x) left = mid + 1;
        else right = mid - 1;
    }
    *sectors += (uint64_t)nseen;
    return 0;
}

/* One walk from an explicit state.  Returns the number of real moves.
 * path (may be NULL) receives the vertices visited after `cur`.
 * trace (may be NULL, capacity trace_cap) receives every trial. */
static uint32_t walk_from(const uint64_t *beg, const uint32_t *csr, const float *aprob, const uint32_t *aalias,
                          const oracle_cfg *c, uint32_t wid, uint32_t *pprev, uint32_t *pcur, uint32_t *phop,
                          uint64_t *phash, uint32_t *path, oracle_stats *st,
                          oracle_trial *trace, uint64_t trace_cap, uint64_t *ntrace,
                          uint64_t *trial_counter, uint8_t *needprev)
{
    uint32_t prev = *pprev, cur = *pcur, hop = *phop;
    uint64_t h = *phash;
    uint32_t moves = 0;
    const uint32_t maxhops = c->maxhops;

    /* Node2vec constants, engine/engine.hpp:169-172 */
    const float inv_p = 1.0f / c->p;
    const float inv_q = 1.0f / c->q;
    const float t_iq1 = (inv_q < 1.0f) ? 1.0f : inv_q; /* std::max(inv_q, 1.0f) */
    const float n2v_max = (inv_p < t_iq1) ? t_iq1 : inv_p;
    const float t_iq2 = (1.0f < inv_q) ? 1.0f : inv_q; /* std::min(inv_q, 1.0f) */
    const float n2v_min = (t_iq2 < inv_p) ? t_iq2 : inv_p;

    while (hop < maxhops) {
        uint32_t r[4];
        if (c->term_prob > 0.0f && hop > 0 && c->keying == KEY_HOP_ATTEMPT) {
            draw4(c->seed, wid, hop, 0, 0, r);
            float u = (float)(r[2] >> 8) * 0x1p-24f;
            if (u < c->term_prob) { st->terminated++; break; }
        }
        uint64_t head = beg[cur], tail = beg[cur + 1];
        st->off_sectors += (((uint64_t)cur * 8u) >> 5) != (((uint64_t)cur * 8u + 15u) >> 5) ? 2 : 1;
        uint64_t deg = tail - head;
        if (deg == 0) {
            /* engine/engine.hpp:196-199: hop = maxhop-1, next vertex 0, then hop++ */
            prev = cur;
            cur = 0;
            hop = maxhops;
            st->dead_ends++;
            break;
        }
        uint64_t phead = beg[prev], ptail = beg[prev + 1];
        uint64_t pdeg = ptail - phead;

        float maxv, minv, t_prev_f = 0.f, t_found, t_notfound;
        double t_prev_d = 0.0;
        if (c->algo == ALG_NODE2VEC) {
            maxv = n2v_max;
            minv = n2v_min;
            t_prev_f = inv_p;
            t_found = 1.0f;
            t_notfound = inv_q;
        } else {
            /* engine/engine.hpp:323-326, 341, 368, 373 */
            t_prev_d = (1.0 - (double)c->alpha) / (double)deg;
            float inv_deg = (float)t_prev_d;
            float inv_prev_deg = c->alpha / (float)pdeg;
            float sum = inv_deg + inv_prev_deg;
            maxv = (inv_deg < sum) ? sum : inv_deg;
            minv = (sum < inv_deg) ? sum : inv_deg;
            t_found = sum;
            t_notfound = inv_deg;
        }

        uint32_t attempt = 0, x;
        uint8_t np = 0; /* some trial of this step is decided only by x in N(prev) */
        for (;;) {
            if (c->keying == KEY_HOP_ATTEMPT)
                draw4(c->seed, wid, hop, attempt, 0, r);
            else
                draw4(c->seed, wid, (uint32_t)*trial_counter, (uint32_t)(*trial_counter >> 32), 0, r);
            attempt++;
            (*trial_counter)++;
            st->trials++;
            uint32_t pos = (uint32_t)((uint64_t)r[0] % deg);
            float rv = ((float)(r[1] >> 8) * 0x1p-24f) * maxv;
            if (trace && *ntrace < trace_cap) {
                oracle_trial *t = &trace[*ntrace];
                t->deg = (uint32_t)deg;
                t->maxv_bits = f2u(maxv);
                t->pos = pos;
                t->rv_bits = f2u(rv);
            }
            if (ntrace) (*ntrace)++;
            if (aprob) {
                /* weighted: alias column pos, kept when coin < prob, else its alias */
                const float coin = (float)(r[3] >> 8) * 0x1p-24f;
                const uint64_t col = coin < aprob[head + pos] ? pos : aalias[head + pos];
                x = csr[head + col];
            } else {
                x = csr[head + pos];
            }
            if (rv <= minv) break;
            if (x == prev) {
                int acc = (c->algo == ALG_NODE2VEC) ? (rv < t_prev_f) : ((double)rv < t_prev_d);
                if (acc) break;
                continue;
            }
            int found;
            const int decides = (rv < t_found) != (rv < t_notfound);
            if (prev != cur && decides) np = 1;
            const uint64_t sec0 = st->search_sectors;
            if (prev == cur)
                found = 1; /* x is drawn from N(cur) = N(prev): the search must succeed */
            else
                found = search_sorted(csr, phead, ptail, x, &st->probes, &st->search_sectors);
            if (found ? (rv < t_found) : (rv < t_notfound)) {
                if (decides) st->acc_sectors += st->search_sectors - sec0;
                break;
            }
        }
        (void)pdeg;
        prev = cur;
        cur = x;
        hop++;
        h = (h ^ (uint64_t)x) * FNV_PRIME;
        if (path) path[moves] = x;
        if (needprev) needprev[moves] = np;
        moves++;
        st->steps++;
    }
    *pprev = prev;
    *pcur = cur;
    *phop = hop;
    *phash = h;
    return moves;
}

uint64_t oracle_hash_init(uint32_t source)
{
    return (FNV_OFFSET ^ (uint64_t)source) * FNV_PRIME;
}

/* Walk walkers [wid_begin, wid_begin + count) from their initial state.
 *   paths:  count x (maxhops+1) u32 or NULL (source first)
 *   lens:   count u32 (vertices recorded) or NULL
 *   hashes: count u64 (FNV-1a over the path's 32-bit vertices) or NULL
 *   finals: count x 3 u32 (prev, cur, hop) after the walk, or NULL */
static int walk_many(const uint64_t *beg, const uint32_t *csr, const float *aprob, const uint32_t *aalias,
                     uint32_t nverts, const oracle_cfg *c, uint32_t wid_begin, const uint32_t *ids, uint32_t count,
                     uint32_t *paths, uint32_t *lens, uint64_t *hashes, uint32_t *finals, oracle_stats *stats,
                     int nthreads)
{
    if (c->algo > ALG_SOSR || c->maxhops == 0) return -1;
    if (c->init_mode == INIT_PER_VERTEX && c->wps == 0) return -1;
    /* every source must be a vertex */
    if (c->init_mode == INIT_PER_VERTEX && !ids && (uint64_t)wid_begin + count > (uint64_t)nverts * c->wps)
        return -1;
    if (c->init_mode == INIT_PER_VERTEX && ids)
        for (uint32_t i = 0; i < count; ++i)
            if ((uint64_t)ids[i] >= (uint64_t)nverts * c->wps) return -1;
    if (c->init_mode == INIT_SINGLE_SOURCE && nverts <= (c->algo == ALG_SOSR ? 3u : 1u)) return -1;
    if (nverts == 0) return -1;
    memset(stats, 0, sizeof(*stats));
    if (nthreads > 0) omp_set_num_threads(nthreads);
    const uint64_t stride = (uint64_t)c->maxhops + 1;
#pragma omp parallel
    {
        oracle_stats st;
        memset(&st, 0, sizeof(st));
#pragma omp for schedule(dynamic, 1024)
        for (int64_t i = 0; i < (int64_t)count; ++i) {
            uint32_t wid = ids ? ids[i] : wid_begin + (uint32_t)i;
            uint32_t src = oracle_walker_source(c, nverts, wid);
            uint32_t prev = src, cur = src, hop = 0;
            uint64_t h = oracle_hash_init(src);
            uint64_t tc = 0;
            uint32_t *path = paths ? paths + (uint64_t)i * stride : NULL;
            if (path) path[0] = src;
            uint32_t moves = walk_from(beg, csr, aprob, aalias, c, wid, &prev, &cur, &hop, &h,
                                       path ? path + 1 : NULL, &st, NULL, 0, NULL, &tc, NULL);
            if (lens) lens[i] = moves + 1;
            if (hashes) hashes[i] = h;
            if (finals) {
                finals[3 * i + 0] = prev;
                finals[3 * i + 1] = cur;
                finals[3 * i + 2] = hop;
            }
        }
#pragma omp critical
        {
            stats->steps += st.steps;
            stats->trials += st.trials;
            stats->probes += st.probes;
            stats->search_sectors += st.search_sectors;
            stats->off_sectors += st.off_sectors;
            stats->dead_ends += st.dead_ends;
            stats->terminated += st.terminated;
            stats->acc_sectors += st.acc_sectors;
        }
    }
    return 0;
}

int oracle_walk(const uint64_t *beg, const uint32_t *csr, uint32_t nverts, const oracle_cfg *c,
                uint32_t wid_begin, uint32_t count, uint32_t *paths, uint32_t *lens,
                uint64_t *hashes, uint32_t *finals, oracle_stats *stats, int nthreads)
{
    return walk_many(beg, csr, NULL, NULL, nverts, c, wid_begin, NULL, count, paths, lens, hashes, finals, stats,
                     nthreads);
}

/* The walkers whose ids are listed (any order, repeats allowed): row i of
 * the outputs is walker ids[i]. */
int oracle_walk_ids(const uint64_t *beg, const uint32_t *csr, uint32_t nverts, const oracle_cfg *c,
                    const uint32_t *ids, uint32_t count, uint32_t *paths, uint32_t *lens, uint64_t *hashes,
                    oracle_stats *stats, int nthreads)
{
    return walk_many(beg, csr, NULL, NULL, nverts, c, 0, ids, count, paths, lens, hashes, NULL, stats, nthreads);
}

/* Weighted Node2vec (the device's gw_weighted.cu): candidates by the alias
 * tables of oracle_build_alias, acceptance by the unweighted rule. */
int oracle_walk_weighted(const uint64_t *beg, const uint32_t *csr, const float *aprob, const uint32_t *aalias,
                         uint32_t nverts, const oracle_cfg *c, uint32_t wid_begin, uint32_t count, uint32_t *paths,
                         uint32_t *lens, uint64_t *hashes, uint32_t *finals, oracle_stats *stats, int nthreads)
{
    if (c->algo != ALG_NODE2VEC) return -1;
    return walk_many(beg, csr, aprob, aalias, nverts, c, wid_begin, NULL, count, paths, lens, hashes, finals, stats,
                     nthreads);
}

/* Walker's alias tables by Vose's method, per vertex (the device's
 * k_build_alias step for step): weights summed in double in index order,
 * p_i = w_i * deg / sum, small (p < 1) and large queues in index order; the
 * next small s takes the front large l (prob[s] = (float)p_s, alias[s] = l,
 * p_l = (p_l + p_s) - 1, l to the back of the small queue when below 1);
 * leftovers get probability 1.  Returns -1 on a weight that is not positive
 * and finite. */
int oracle_build_alias(const uint64_t *beg, const float *w, uint32_t nverts, float *prob, uint32_t *alias)
{
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(| : bad)
    for (int64_t v = 0; v < (int64_t)nverts; ++v) {
        const uint64_t h = beg[v], d = beg[v + 1] - h;
        if (d == 0) continue;
        double sum = 0.0;
        int b = 0;
        for (uint64_t i = 0; i < d; ++i) {
            const float wi = w[h + i];
            b |= !(wi > 0.f && wi < INFINITY);
            sum = sum + (double)wi;
        }
        if (b) {
            bad = 1;
            continue;
        }
        double *p = malloc(d * sizeof(double));
        uint32_t *small = malloc(d * sizeof(uint32_t)), *large = malloc(d * sizeof(uint32_t));
        uint64_t ns = 0, nl = 0, hs = 0, hl = 0;
        for (uint64_t i = 0; i < d; ++i) {
            p[i] = ((double)w[h + i] * (double)d) / sum;
            if (p[i] < 1.0) small[ns++] = (uint32_t)i;
            else large[nl++] = (uint32_t)i;
        }
        while (hs < ns && hl < nl) {
            const uint32_t s = small[hs++], l = large[hl];
            prob[h + s] = (float)p[s];
            alias[h + s] = l;
            p[l] = (p[l] + p[s]) - 1.0;
            if (p[l] < 1.0) {
                ++hl;
                small[ns++] = l;
            }
        }
        while (hl < nl) {
            const uint32_t l = large[hl++];
            prob[h + l] = 1.0f;
            alias[h + l] = l;
        }
        while (hs < ns) {
            const uint32_t s = small[hs++];
            prob[h + s] = 1.0f;
            alias[h + s] = s;
        }
        free(p);
        free(small);
        free(large);
    }
    return bad ? -1 : 0;
}

/* Single walker from an explicit state (prev, cur, hop) with a trial trace,
 * for the differential test against the reference's sidewalkupdate.
 * Returns the number of moves; *ntrace receives the number of trials. */
uint32_t oracle_walk_traced(const uint64_t *beg, const uint32_t *csr, const oracle_cfg *c,
                            uint32_t wid, uint32_t prev, uint32_t cur, uint32_t hop,
                            uint32_t *path, oracle_trial *trace, uint64_t trace_cap,
                            uint64_t *ntrace, uint32_t *final3)
{
    oracle_stats st;
    memset(&st, 0, sizeof(st));
    uint64_t h = 0, tc = 0;
    *ntrace = 0;
    uint32_t moves = walk_from(beg, csr, NULL, NULL, c, wid, &prev, &cur, &hop, &h, path, &st, trace, trace_cap,
                               ntrace, &tc, NULL);
    if (final3) {
        final3[0] = prev;
        final3[1] = cur;
        final3[2] = hop;
    }
    return moves;
}


/* ------------------------------------------------------------------ out-of-core schedule emulation
 *
 * A walk does not depend on the block schedule, so the blocks each walker
 * will need, in order, are fixed in advance.  oracle_walk_reqs writes them
 * per walker as u16 entries, one per "enter" (the engine's step set-up at the
 * walker's current vertex):
 *   bits 0-13  block of the current vertex
 *   bit 14     terminal: the walk ends at this enter (dead end, or the
 *              termination draw) -- it still needs the block resident
 *   bit 15     the step taken from here has a trial decided only by whether
 *              the candidate is in N(prev) (the lazy residency rule then
 *              needs the previous block resident too)
 * A walk that reaches maxhops has no terminal entry.  reqs is count x
 * (maxhops+1) u16, nent[i] the entries of walker wid_begin+i. */
int oracle_walk_reqs(const uint64_t *beg, const uint32_t *csr, uint32_t nverts, const oracle_cfg *c,
                     const uint32_t *vstart, uint32_t nb, uint32_t wid_begin, uint32_t count, uint16_t *reqs,
                     uint32_t *nent, int nthreads)
{
    if (c->algo > ALG_SOSR || c->maxhops == 0 || nb == 0 || nb > 1024 || nverts == 0) return -1;
    if (c->init_mode == INIT_PER_VERTEX && (c->wps == 0 || (uint64_t)wid_begin + count > (uint64_t)nverts * c->wps))
        return -1;
    if (nthreads > 0) omp_set_num_threads(nthreads);
    const uint64_t stride = (uint64_t)c->maxhops + 1;
    int bad = 0;
#pragma omp parallel reduction(| : bad)
    {
        oracle_stats st;
        memset(&st, 0, sizeof(st));
        uint32_t *path = (uint32_t *)malloc(sizeof(uint32_t) * c->maxhops);
        uint8_t *np = (uint8_t *)malloc(c->maxhops);
#pragma omp for schedule(dynamic, 1024)
        for (int64_t i = 0; i < (int64_t)count; ++i) {
            const uint32_t wid = wid_begin + (uint32_t)i;
            const uint32_t src = oracle_walker_source(c, nverts, wid);
            uint32_t prev = src, cur = src, hop = 0;
            uint64_t h = oracle_hash_init(src), tc = 0;
            const uint32_t moves = walk_from(beg, csr, NULL, NULL, c, wid, &prev, &cur, &hop, &h, path, &st, NULL, 0,
                                             NULL, &tc, np);
            uint16_t *r = reqs + (uint64_t)i * stride;
            for (uint32_t e = 0; e <= moves && e < c->maxhops; ++e) {
                const uint32_t v = e ? path[e - 1] : src;
                /* block of v: the last block starting at or before it */
                uint32_t lo = 0, hi = nb;
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (vstart[mid] <= v) lo = mid;
                    else hi = mid;
                }
                if (v >= vstart[nb]) bad = 1;
                uint16_t ent = (uint16_t)lo;
                if (e < moves) {
                    if (np[e]) ent |= 0x8000u;
                } else {
                    ent |= 0x4000u; /* moves < maxhops: the walk ends at this enter */
                }
                r[e] = ent;
            }
            nent[i] = moves + (moves < c->maxhops ? 1u : 0u);
        }
        free(path);
        free(np);
    }
    return bad ? -1 : 0;
}

typedef struct {
    uint64_t iterations, loads, steps, parks, rescues;
    uint64_t finished;
    uint64_t zc_steps; /* steps left to the mapped-host tail (zero mode) */
} oracle_sched_stats;

/* Plain block choice, GOwalker_scheduler_t::max_choose_blocks
 * (engine/schedule.hpp:70-138), with the engine's rescue when nothing
 * qualifies: *action 1 append, 2 replace cached[*pos], 0 none (then *rblk /
 * *rpos give the rescue: the fullest bucket with an absent block, its current
 * block first, evicting the cached block with the fewest incident walkers
 * outside that bucket).  Ties: lowest block id, first position. */
static void plain_choice(const uint64_t *pairs, uint32_t nb, const uint32_t *cached, uint32_t ncached,
                         uint32_t nslots, uint64_t zero_threshold, int *action, int *blk, int *pos, int *rblk,
                         int *rpos)
{
    uint8_t isc[1024];
    memset(isc, 0, nb);
    for (uint32_t j = 0; j < ncached; ++j) isc[cached[j]] = 1;
    const int full = ncached >= nslots;
    int64_t best = -1;
    int bi = -1, bp = -1;
    for (uint32_t i = 0; i < nb; ++i) {
        if (isc[i]) continue;
        uint64_t score = 0;
        int p = (int)ncached;
        if (!full) {
            for (uint32_t j = 0; j < ncached; ++j) score += pairs[(uint64_t)i * nb + cached[j]] + pairs[(uint64_t)cached[j] * nb + i];
            score += pairs[(uint64_t)i * nb + i];
        } else {
            uint64_t all = 0, mn = 0xFFFFFFFFull;
            p = 0;
            for (uint32_t j = 0; j < ncached; ++j) {
                const uint64_t v = pairs[(uint64_t)i * nb + cached[j]] + pairs[(uint64_t)cached[j] * nb + i];
                all += v;
                if (v < mn) {
                    mn = v;
                    p = (int)j;
                }
            }
            score = all - mn;
        }
        if ((int64_t)score > best) {
            best = (int64_t)score;
            bi = (int)i;
            bp = p;
        }
    }
    if (bi >= 0 && best > 0 && (uint64_t)best > zero_threshold) {
        *action = full ? 2 : 1;
        *blk = bi;
        *pos = bp;
    } else {
        *action = 0;
        *blk = *pos = -1;
    }
    *rblk = *rpos = -1;
    uint64_t bc = 0;
    int64_t bb = -1;
    for (uint64_t b = 0; b < (uint64_t)nb * nb; ++b)
        if (pairs[b] > bc && !(isc[b / nb] && isc[b % nb])) {
            bc = pairs[b];
            bb = (int64_t)b;
        }
    if (bb >= 0) {
        const uint32_t p = (uint32_t)(bb / nb), cc = (uint32_t)(bb % nb);
        *rblk = (int)(isc[cc] ? p : cc);
        if (full) {
            uint64_t mn = ~0ull;
            for (uint32_t j = 0; j < ncached; ++j) {
                const uint32_t b2 = cached[j];
                if (b2 == p || b2 == cc) continue;
                uint64_t inc = 0;
                for (uint32_t k = 0; k < nb; ++k)
                    inc += pairs[(uint64_t)b2 * nb + k] + (k != b2 ? pairs[(uint64_t)k * nb + b2] : 0);
                if (inc < mn) {
                    mn = inc;
                    *rpos = (int)j;
                }
            }
        }
    }
}

/* The out-of-core engine's block schedule replayed on the CPU from the
 * walkers' requirement entries (oracle_walk_reqs): per iteration, the block
 * staged in the last iteration becomes resident, the plain choice is taken
 * from the bucket counts of the last re-bucketing (prefetch: the decision
 * picks the next iteration's block), every runnable walker advances while
 * its blocks are resident, and the walkers are re-bucketed by (prev block,
 * cur block, needs-prev flag).  `lazy` is the engine's residency rule (0:
 * both blocks, the reference's).  nslots = cache slots; with prefetch one of
 * them stages the next block.  log (optional, 3 x iterations cap): per
 * iteration the loaded block, the cached position it replaced (-1 append)
 * and the steps taken.  Returns the iteration count or -1. */
int64_t oracle_sched_replay(const uint16_t *reqs, const uint32_t *nent, uint32_t count, uint32_t stride, uint32_t nb,
                            uint32_t nslots, int prefetch, int lazy, uint64_t zero_threshold, int evict_incident,
                            int zero_tail, int32_t *log, uint64_t log_cap, oracle_sched_stats *out)
{
    if (nb == 0 || nb > 1024 || nslots < (prefetch ? 3u : 2u)) return -1;
    memset(out, 0, sizeof(*out));
    const uint64_t nn = (uint64_t)nb * nb;
    uint32_t *e = (uint32_t *)calloc(count, sizeof(uint32_t));      /* next entry of each walker */
    uint8_t *flag = (uint8_t *)calloc(count, 1);                     /* parked needing its prev block */
    uint64_t *cnt = (uint64_t *)calloc(2 * nn, sizeof(uint64_t));   /* bucket counts */
    uint64_t *pairs = (uint64_t *)calloc(nn, sizeof(uint64_t));
    uint32_t *live = (uint32_t *)malloc(sizeof(uint32_t) * (count ? count : 1));
    uint8_t res[1024];
    uint32_t cached[1024], ncached = 0;
    memset(res, 0, sizeof(res));
    uint32_t nlive = 0;
    for (uint32_t w = 0; w < count; ++w)
        if (nent[w]) live[nlive++] = w;
        else out->finished++;
    const uint32_t capacity = prefetch ? nslots - 1 : nslots;
    int staged = -1, staged_pos = -1;
    int64_t it = 0;
#define BLK(w, k) ((uint32_t)(reqs[(uint64_t)(w) * stride + (k)] & 0x3FFFu))
    /* bucket counts of the live walkers (the re-bucketing) */
#define REBUCKET()                                                                 \
    do {                                                                            \
        memset(cnt, 0, sizeof(uint64_t) * 2 * nn);                                  \
        for (uint32_t k = 0; k < nlive; ++k) {                                      \
            const uint32_t w = live[k];                                             \
            const uint32_t cb = BLK(w, e[w]), pb = e[w] ? BLK(w, e[w] - 1) : cb;     \
            cnt[(flag[w] ? nn : 0) + (uint64_t)pb * nb + cb]++;                     \
        }                                                                           \
        for (uint64_t b = 0; b < nn; ++b) pairs[b] = cnt[b] + cnt[nn + b];          \
    } while (0)
    REBUCKET();
    for (;;) {
        if (++it > (1 << 22)) {
            it = -1;
            break;
        }
        if (prefetch && staged >= 0) {
            if (staged_pos >= 0) {
                res[cached[staged_pos]] = 0;
                cached[staged_pos] = (uint32_t)staged;
            } else {
                cached[ncached++] = (uint32_t)staged;
            }
            res[staged] = 1;
            staged = -1;
        }
        int action, blk, pos, rblk, rpos;
        plain_choice(pairs, nb, cached, ncached, capacity, zero_threshold, &action, &blk, &pos, &rblk, &rpos);
        if (evict_incident && action == 2) {
            /* the cached block with the fewest incident walkers (first on ties) */
            uint64_t mn = ~0ull;
            for (uint32_t j = 0; j < ncached; ++j) {
                const uint32_t c = cached[j];
                uint64_t inc = 0;
                for (uint32_t k = 0; k < nb; ++k)
                    inc += pairs[(uint64_t)c * nb + k] + (k != c ? pairs[(uint64_t)k * nb + c] : 0);
                if (inc < mn) {
                    mn = inc;
                    pos = (int)j;
                }
            }
        }
        const uint32_t live_at_decision = nlive;
        /* zero mode: nothing scores above the threshold -- the rest finishes
           through mapped host memory (with prefetch, after this iteration's step) */
        const int tail = zero_tail && !action && live_at_decision > 0;
        int load = -1, lpos = -1;
        if (tail) {
            /* no load */
        } else if (action) {
            load = blk;
            lpos = action == 2 ? pos : -1;
        } else if (rblk >= 0 && (ncached < capacity || rpos >= 0)) {
            load = rblk;
            lpos = ncached >= capacity ? rpos : -1;
            out->rescues++;
        }
        if (!prefetch && live_at_decision == 0) break;
        if (tail && !prefetch) {
            for (uint32_t k = 0; k < nlive; ++k) out->zc_steps += nent[live[k]] - e[live[k]] -
                                                                 ((reqs[(uint64_t)live[k] * stride + nent[live[k]] - 1] & 0x4000u) ? 1u : 0u);
            break;
        }
        if (!prefetch && load >= 0) {
            /* loaded before this iteration's step */
            if (lpos >= 0) {
                res[cached[lpos]] = 0;
                cached[lpos] = (uint32_t)load;
            } else {
                cached[ncached++] = (uint32_t)load;
            }
            res[load] = 1;
        }
        /* the step: every walker of a runnable bucket advances while it can */
        uint64_t steps_before = out->steps;
        uint32_t k2 = 0;
        for (uint32_t k = 0; k < nlive; ++k) {
            const uint32_t w = live[k];
            uint32_t ew = e[w];
            const uint32_t cb0 = BLK(w, ew), pb0 = ew ? BLK(w, ew - 1) : cb0;
            const int runnable = res[cb0] && (res[pb0] || (lazy && !flag[w]));
            int done = 0;
            if (runnable) {
                flag[w] = 0;
                for (;;) {
                    const uint16_t ent = reqs[(uint64_t)w * stride + ew];
                    const uint32_t cb = ent & 0x3FFFu, pb = ew ? BLK(w, ew - 1) : cb;
                    if (ent & 0x4000u) {
                        done = 1;
                        break;
                    }
                    if (!res[pb] && (!lazy || (ent & 0x8000u))) {
                        flag[w] = 1; /* parked: needs N(prev) */
                        out->parks++;
                        break;
                    }
                    (void)cb;
                    ew++;
                    out->steps++;
                    if (ew >= nent[w]) {
                        done = 1;
                        break;
                    }
                    if (!res[BLK(w, ew)]) {
                        out->parks++;
                        break;
                    }
                }
                e[w] = ew;
            }
            if (done) out->finished++;
            else live[k2++] = w;
        }
        nlive = k2;
        if (log && (uint64_t)(it - 1) < log_cap) {
            log[3 * (it - 1) + 0] = load;
            log[3 * (it - 1) + 1] = lpos;
            log[3 * (it - 1) + 2] = (int32_t)(out->steps - steps_before);
        }
        if (load >= 0) out->loads++;
        if (prefetch && tail) {
            for (uint32_t k = 0; k < nlive; ++k) out->zc_steps += nent[live[k]] - e[live[k]] -
                                                                 ((reqs[(uint64_t)live[k] * stride + nent[live[k]] - 1] & 0x4000u) ? 1u : 0u);
            break;
        }
        if (prefetch) {
            if (live_at_decision == 0) break;
            staged = load;
            staged_pos = lpos;
        }
        REBUCKET();
    }
#undef REBUCKET
#undef BLK
    out->iterations = it > 0 ? (uint64_t)it : 0;
    free(e);
    free(flag);
    free(cnt);
    free(pairs);
    free(live);
    return it;
}

/* ------------------------------------------------------------------ schedule study
 *
 * What other block policies would do on the same walks (the engine's
 * lazy-residency rule, no prefetch): how much a better block choice or
 * eviction could save, and what finishing the low-yield tail through mapped
 * host memory saves.  Analysis only (the engine runs oracle_sched_replay's
 * plain rule or its learned variant).
 *   policy 0  GOWalker's choice (max_choose_blocks) and its rescue
 *   policy 1  clairvoyant one-iteration yield: load the block (with the plain
 *             rule's victim) whose load lets the walkers take the most steps
 *             this iteration, computed exactly from the walks
 *   policy 2  GOWalker's choice, clairvoyant eviction: evict the cached block
 *             that the fewest waiting walkers need within their next 4 entries
 *   policy 3  GOWalker's choice, evicting the cached block with the fewest
 *             incident walkers (current or previous block) now
 *   policy 4  GOWalker's choice, evicting the lowest running average of steps
 *             taken in the block (weight 1/2 per iteration)
 *   policy 5  GOWalker's choice, evicting the block unused the longest
 * zt > 0: once the plain rule's best score is <= zt (the reference's zero
 * threshold, engine/schedule.hpp:101,124 and apps/Node2vec.cu:100-108), stop
 * loading; the remaining steps are counted in *zc_steps (they would run
 * through mapped host memory). */
static const uint16_t *st_reqs;
static const uint32_t *st_nent;
static uint32_t st_stride;
#define SENT(w, k) (st_reqs[(uint64_t)(w) * st_stride + (k)])
#define SBLK(w, k) ((uint32_t)(SENT(w, k) & 0x3FFFu))

static uint32_t study_run(uint32_t *e, uint8_t *flag, uint32_t w, const uint8_t *res, int lazy, int commit, int *done,
                          uint64_t *usage)
{
    uint32_t ew = e[w], steps = 0;
    *done = 0;
    const uint32_t cb0 = SBLK(w, ew), pb0 = ew ? SBLK(w, ew - 1) : cb0;
    if (!(res[cb0] && (res[pb0] || (lazy && !flag[w])))) return 0;
    uint8_t fl = 0;
    for (;;) {
        const uint16_t ent = SENT(w, ew);
        const uint32_t pb = ew ? SBLK(w, ew - 1) : (ent & 0x3FFFu);
        if (ent & 0x4000u) {
            *done = 1;
            break;
        }
        if (!res[pb] && (!lazy || (ent & 0x8000u))) {
            fl = 1;
            break;
        }
        if (usage) usage[ent & 0x3FFFu]++;
        ew++;
        steps++;
        if (ew >= st_nent[w]) {
            *done = 1;
            break;
        }
        if (!res[SBLK(w, ew)]) break;
    }
    if (commit) {
        e[w] = ew;
        flag[w] = fl;
    }
    return steps + (uint32_t)(*done && steps == 0);
}

int64_t oracle_sched_study(const uint16_t *reqs, const uint32_t *nent, uint32_t count, uint32_t stride, uint32_t nb,
                           uint32_t nslots, int lazy, int policy, uint64_t zt, uint64_t *loads, uint64_t *steps,
                           uint64_t *zc_steps)
{
    if (nb == 0 || nb > 1024 || nslots < 2 || policy < 0 || policy > 5) return -1;
    st_reqs = reqs;
    st_nent = nent;
    st_stride = stride;
    const uint64_t nn = (uint64_t)nb * nb;
    uint32_t *e = (uint32_t *)calloc(count, sizeof(uint32_t));
    uint8_t *flag = (uint8_t *)calloc(count, 1);
    uint64_t *pairs = (uint64_t *)calloc(nn, sizeof(uint64_t));
    uint64_t *need = (uint64_t *)calloc(nb, sizeof(uint64_t));
    uint64_t *usage = (uint64_t *)calloc(nb, sizeof(uint64_t));   /* steps taken in each block, this iteration */
    double *use_ema = (double *)calloc(nb, sizeof(double));        /* their running average */
    int64_t *last_use = (int64_t *)calloc(nb, sizeof(int64_t));    /* last iteration with steps in the block */
    uint32_t *live = (uint32_t *)malloc(sizeof(uint32_t) * (count ? count : 1));
    uint32_t nlive = 0;
    for (uint32_t w = 0; w < count; ++w) live[nlive++] = w;
    uint8_t res[1024];
    uint32_t cached[1024], ncached = 0;
    memset(res, 0, sizeof(res));
    *loads = *steps = *zc_steps = 0;
    int64_t it = 0;
    int stalled = 0; /* the last iteration moved no walker: the plain rule decides the next one */
    for (;;) {
        if (++it > (1 << 22)) {
            it = -1;
            break;
        }
        memset(pairs, 0, sizeof(uint64_t) * nn);
        for (uint32_t k = 0; k < nlive; ++k) {
            const uint32_t w = live[k], cb = SBLK(w, e[w]), pb = e[w] ? SBLK(w, e[w] - 1) : cb;
            pairs[(uint64_t)pb * nb + cb]++;
        }
        if (nlive == 0) break;
        const int full = ncached >= nslots;
        int action, blk, pos, rblk, rpos;
        plain_choice(pairs, nb, cached, ncached, nslots, 0, &action, &blk, &pos, &rblk, &rpos);
        uint64_t plain_score = 0;
        if (action) {
            for (uint32_t j = 0; j < ncached; ++j) {
                plain_score += pairs[(uint64_t)blk * nb + cached[j]] + pairs[(uint64_t)cached[j] * nb + blk];
            }
            if (full) {
                uint64_t mn = 0xFFFFFFFFull;
                for (uint32_t j = 0; j < ncached; ++j) {
                    const uint64_t v = pairs[(uint64_t)blk * nb + cached[j]] + pairs[(uint64_t)cached[j] * nb + blk];
                    if (v < mn) mn = v;
                }
                plain_score -= mn;
            } else {
                plain_score += pairs[(uint64_t)blk * nb + blk];
            }
        }
        if (zt && plain_score <= zt) {
            for (uint32_t k = 0; k < nlive; ++k) {
                const uint32_t w = live[k];
                *zc_steps += st_nent[w] - e[w] - ((SENT(w, st_nent[w] - 1) & 0x4000u) ? 1u : 0u);
            }
            break;
        }
        if (policy == 1 && action && !stalled) {
            double by = -1.0;
            int yi = -1, yp = -1;
            for (uint32_t i = 0; i < nb; ++i) {
                if (res[i]) continue;
                int p = (int)ncached;
                if (full) {
                    uint64_t mn = 0xFFFFFFFFull;
                    p = 0;
                    for (uint32_t j = 0; j < ncached; ++j) {
                        const uint64_t v = pairs[(uint64_t)i * nb + cached[j]] + pairs[(uint64_t)cached[j] * nb + i];
                        if (v < mn) {
                            mn = v;
                            p = (int)j;
                        }
                    }
                }
                uint8_t r2[1024];
                memcpy(r2, res, nb);
                if (full) r2[cached[p]] = 0;
                r2[i] = 1;
                double y = 0.0;
                int d;
                for (uint32_t k = 0; k < nlive; ++k) {
                    const uint32_t w = live[k], cb = SBLK(w, e[w]), pb = e[w] ? SBLK(w, e[w] - 1) : cb;
                    if (cb == i || pb == i) y += study_run(e, flag, w, r2, lazy, 0, &d, NULL);
                }
                if (y > by) {
                    by = y;
                    yi = (int)i;
                    yp = p;
                }
            }
            if (yi >= 0 && by > 0) {
                blk = yi;
                pos = yp;
            }
        }
        if (policy == 2 && action == 2 && !stalled) {
            memset(need, 0, sizeof(uint64_t) * nb);
            for (uint32_t k = 0; k < nlive; ++k) {
                const uint32_t w = live[k];
                for (uint32_t d = 0; d < 4 && e[w] + d < st_nent[w]; ++d) need[SBLK(w, e[w] + d)]++;
            }
            uint64_t mn = ~0ull;
            for (uint32_t j = 0; j < ncached; ++j)
                if (need[cached[j]] < mn) {
                    mn = need[cached[j]];
                    pos = (int)j;
                }
        }
        if (policy >= 3 && action == 2 && !stalled) {
            /* 3: the fewest walkers at or from the block now; 4: the lowest
               running average of steps taken in it; 5: the longest unused */
            double mn = 1e300;
            for (uint32_t j = 0; j < ncached; ++j) {
                const uint32_t c = cached[j];
                double v;
                if (policy == 3) {
                    uint64_t inc = 0;
                    for (uint32_t k = 0; k < nb; ++k)
                        inc += pairs[(uint64_t)c * nb + k] + (k != c ? pairs[(uint64_t)k * nb + c] : 0);
                    v = (double)inc;
                } else if (policy == 4) {
                    v = use_ema[c];
                } else {
                    v = (double)last_use[c];
                }
                if (v < mn) {
                    mn = v;
                    pos = (int)j;
                }
            }
        }
        int load = -1, lpos = -1;
        if (action) {
            load = blk;
            lpos = action == 2 ? pos : -1;
        } else if (rblk >= 0 && (ncached < nslots || rpos >= 0)) {
            load = rblk;
            lpos = ncached >= nslots ? rpos : -1;
        } else {
            it = -1;
            break;
        }
        if (lpos >= 0) {
            res[cached[lpos]] = 0;
            cached[lpos] = (uint32_t)load;
        } else {
            cached[ncached++] = (uint32_t)load;
        }
        res[load] = 1;
        (*loads)++;
        uint32_t k2 = 0;
        const uint64_t steps0 = *steps;
        memset(usage, 0, sizeof(uint64_t) * nb);
        for (uint32_t k = 0; k < nlive; ++k) {
            const uint32_t w = live[k], before = e[w];
            int d;
            study_run(e, flag, w, res, lazy, 1, &d, usage);
            *steps += e[w] - before;
            if (!d) live[k2++] = w;
        }
        stalled = *steps == steps0 && k2 == nlive;
        nlive = k2;
        for (uint32_t b = 0; b < nb; ++b) {
            use_ema[b] = 0.5 * use_ema[b] + 0.5 * (double)usage[b];
            if (usage[b]) last_use[b] = it;
        }
    }
    free(usage);
    free(use_ema);
    free(last_use);
    free(e);
    free(flag);
    free(pairs);
    free(need);
    free(live);
    return it;
}
#undef SENT
#undef SBLK

/*
 * ref_step_harness.cu -- drives the GOWalker reference's own CPU walk step
 * (graph_engine::sidewalkupdate / SOPR_sidewalkupdate, engine/engine.hpp:158-404)
 * from its unmodified headers, for the differential test of the oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile from the reference
 * sources where they lie (-I<reference>), linked against the host CUDA stub
 * (cuda_host_stub.c), output to oracle/_ref/.  Nothing is copied from the
 * reference; the harness only includes its headers.
 *
 * Two builds of this file:
 *   default            RandNum::inlineRandPair (util/util.hpp:291-301) is
 *                      renamed away by the preprocessor and every call site in
 *                      engine/engine.hpp:207,332 is routed to a Philox draw
 *                      keyed by (seed, walker id, running trial index) -- the
 *                      same stream as the oracle's KEY_TRIAL mode.  Each draw
 *                      is logged, so the trial sequence can be compared.
 *   GW_REF_UNMODIFIED  the reference's xoroshiro128+ RandNum is left alone and
 *                      seeded deterministically; used for the chi-square test
 *                      of the unmodified transition law.
 *
 * The engine objects are built the way apps/Node2vec.cu:109-173 builds them,
 * from graph files written by the test in the reference's on-disk format.
 */
#include <cstdint>
#include <cstring>
#include <vector>
#include <iostream>
#include <fstream>
#include <functional>
#include <omp.h>
#include "api/types.hpp"

#ifndef GW_REF_UNMODIFIED
#define inlineRandPair inlineRandPair_xoroshiro128
#endif
#include "util/util.hpp"
#ifndef GW_REF_UNMODIFIED
#undef inlineRandPair

extern "C" void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

static uint64_t g_seed = 0;
static uint32_t *g_trace = nullptr;
static uint64_t g_trace_cap = 0, g_trace_n = 0;

/* RandNum state carries the key: rng_seed0 = walker id, rng_seed1 = trial index. */
static inline void gw_ref_draw_pair(RandNum *s, float max_val, size_t bound, float &rand_val,
                                    size_t &rand_pos)
{
    uint32_t wid = (uint32_t)s->rng_seed0;
    uint64_t t = s->rng_seed1++;
    uint32_t ctr[4] = {wid, (uint32_t)t, (uint32_t)(t >> 32), 0u};
    uint32_t key[2] = {(uint32_t)g_seed, (uint32_t)(g_seed >> 32)};
    uint32_t r[4];
    oracle_philox4x32_10(ctr, key, r);
    rand_pos = (size_t)((uint64_t)r[0] % (uint64_t)bound);
    rand_val = ((float)(r[1] >> 8) * 0x1p-24f) * max_val;
    if (g_trace && g_trace_n < g_trace_cap) {
        uint32_t *e = g_trace + 4 * g_trace_n;
        uint32_t mb, rb;
        memcpy(&mb, &max_val, 4);
        memcpy(&rb, &rand_val, 4);
        e[0] = (uint32_t)bound;
        e[1] = mb;
        e[2] = (uint32_t)rand_pos;
        e[3] = rb;
    }
    g_trace_n++;
}
/* `seed->inlineRandPair(a, b, c, d)` at engine/engine.hpp:207,332 becomes
 * `seed->rng_seed1 += 0, gw_ref_draw_pair(seed, a, b, c, d)`. */
#define inlineRandPair(MV, BD, RV, RP) rng_seed1 += 0, gw_ref_draw_pair(seed, MV, BD, RV, RP)
#endif

#include "api/constants.hpp"
#include "engine/config.hpp"
#include "engine/cache.hpp"
#include "engine/schedule.hpp"
#include "engine/walk.hpp"
#include "engine/engine.hpp"
#include "metrics/metrics.hpp"

namespace {
struct RefState {
    graph_config conf;
    metrics *m = nullptr;
    graph_block *blocks = nullptr;
    graph_driver *driver = nullptr;
    scheduler *sched = nullptr;
    graph_walk *walk = nullptr;
    graph_cache *cache = nullptr;
    graph_cache *g_cache = nullptr;
    graph_engine *engine = nullptr;
};
RefState *g_ref = nullptr;
const char *g_argv[] = {"ref_step_harness", "dataset", nullptr};
}  // namespace

extern "C" int ref_open(const char *base_name, uint32_t algo, float p, float q, float alpha,
                        uint32_t maxhops, uint32_t blocksize_mb, uint32_t cpu_batch)
{
    if (g_ref) return -1;
    set_argc(2, g_argv);
    vid_t nvertices;
    eid_t nedges;
    vid_t min_vert;
    load_graph_meta(base_name, &nvertices, &nedges, &min_vert, false);
    RefState *s = new RefState();
    size_t blocksize = (size_t)blocksize_mb * 1024 * 1024;
    s->conf = graph_config{base_name,
                           blocksize,            /* cache_size: one device slot */
                           blocksize,
                           (tid_t)1,             /* nthreads */
                           (tid_t)1,
                           nvertices,
                           nedges,
                           min_vert,
                           false,
                           nvertices,            /* numwalks */
                           1,                    /* walkpersource */
                           1,                    /* blockpergrid */
                           1,                    /* threadperblock */
                           1,                    /* cpu_threads */
                           (AlgorithmType)algo,
                           p,
                           q,
                           alpha,
                           maxhops,
                           cpu_batch,
                           16,                   /* gpu_batch */
                           0,
                           true,
                           true,
                           false};
    s->m = new metrics("ref_step_harness");
    s->blocks = new graph_block(&s->conf);
    s->driver = new graph_driver(&s->conf, *s->m);
    s->sched = new GOwalker_scheduler_t(*s->m);
    s->walk = new graph_walk(s->conf, *s->driver, *s->blocks);
    s->cache = new graph_cache(s->blocks->nblocks, blocksize);
    s->g_cache = new graph_cache(1, blocksize);
    s->engine = new graph_engine(*s->cache, *s->walk, *s->driver, s->conf, *s->m, *s->g_cache, s->sched);
    g_ref = s;
    return (int)s->blocks->nblocks;
}

extern "C" void ref_set_seed(uint64_t seed)
{
#ifndef GW_REF_UNMODIFIED
    g_seed = seed;
#else
    if (g_ref) g_ref->engine->seeds[0].reInit(seed);
#endif
}

/* Runs the reference step from walker state (prev, cur, hop, prev_blk, cur_blk).
 * Returns run_step.  trace (4 u32 per trial: deg, max_val bits, rand_pos,
 * rand_val bits) is filled in the shimmed build.  *pushed is 1 when the
 * reference re-bucketed the walker (engine/engine.hpp:275-285) and
 * pushed_state then holds (prev, cur, prev_blk, cur_blk, hop). */
extern "C" int ref_walk(uint32_t wid, uint32_t prev, uint32_t cur, uint32_t hop, uint32_t prev_blk,
                        uint32_t cur_blk, uint32_t *trace, uint64_t trace_cap, uint64_t *ntrace,
                        int *pushed, uint32_t *pushed_state)
{
    RefState *s = g_ref;
    if (!s) return -1;
    graph_walk *w = s->walk;
    bid_t tot = w->totblocks;
    std::vector<size_t> before(tot);
    for (bid_t b = 0; b < tot; ++b) before[b] = w->cpu_walkbuffer[b][0].bsize;

    walker_t walker;
    memset(&walker, 0, sizeof(walker));
    walker.id = wid;
    walker.source = cur;
    walker.previous = prev;
    walker.current = cur;
    walker.hop = hop;
    walker.prev_index = prev_blk;
    walker.cur_index = cur_blk;
#ifndef GW_REF_UNMODIFIED
    s->engine->seeds[0].rng_seed0 = wid;
    s->engine->seeds[0].rng_seed1 = 0;
    g_trace = trace;
    g_trace_cap = trace ? trace_cap : 0;
    g_trace_n = 0;
#else
    (void)trace;
    (void)trace_cap;
#endif
    int run;
    if (s->conf.algorithm == node2vec)
        run = s->engine->sidewalkupdate(walker, s->conf.p, s->conf.q, s->conf.maxhops, &s->engine->seeds[0],
                                        s->engine, 0);
    else
        run = s->engine->SOPR_sidewalkupdate(walker, s->conf.alpha, s->conf.maxhops, &s->engine->seeds[0],
                                             s->engine, 0);
#ifndef GW_REF_UNMODIFIED
    if (ntrace) *ntrace = g_trace_n;
    g_trace = nullptr;
#else
    if (ntrace) *ntrace = 0;
#endif
    *pushed = 0;
    for (bid_t b = 0; b < tot; ++b) {
        graph_buffer<walker_t> &buf = w->cpu_walkbuffer[b][0];
        if (buf.array && buf.bsize == before[b] + 1) {
            walker_t &o = buf.array[buf.bsize - 1];
            pushed_state[0] = o.previous;
            pushed_state[1] = o.current;
            pushed_state[2] = o.prev_index;
            pushed_state[3] = o.cur_index;
            pushed_state[4] = o.hop;
            buf.bsize--; /* keep the buffer from filling across calls */
            *pushed = 1;
            break;
        }
    }
    return run;
}

extern "C" uint32_t ref_get_block(uint32_t v)
{
    return g_ref ? g_ref->blocks->get_block(v) : 0xFFFFFFFFu;
}

/* GOwalker_scheduler_t::max_choose_blocks (engine/schedule.hpp:70-138), the
 * reference's own code, on given bucket counts: counts = nb*nb walkers per
 * (prev block, cur block) pair, nb = the opened dataset's block count;
 * cached = the scheduler's list (its `buckets`) in order; nslots = the device
 * cache's slot count (graph_cache::ncblock).  Returns 1 when the reference
 * chose a block; out_list receives its list afterwards (*out_n entries, room
 * for nb).  The counts are cleared again before returning. */
extern "C" int ref_max_choose_blocks(const uint32_t *counts, const uint32_t *cached, uint32_t ncached,
                                     uint32_t nslots, uint32_t zero_threshold, uint32_t *out_list,
                                     uint32_t *out_n)
{
    RefState *s = g_ref;
    if (!s || nslots == 0) return -1;
    graph_walk *w = s->walk;
    const bid_t nb = w->nblocks;
    for (bid_t b = 0; b < nb * nb; ++b) w->block_walks[b].num = counts[b];
    GOwalker_scheduler_t *g = static_cast<GOwalker_scheduler_t *>(s->sched);
    g->buckets.assign(cached, cached + ncached);
    graph_cache slots(nslots, s->conf.blocksize);
    s->conf.zero_threshold = zero_threshold;
    const bool chose = g->max_choose_blocks(s->conf, slots, *s->driver, *w, nullptr, nullptr, *s->g_cache, *s->m);
    *out_n = (uint32_t)g->buckets.size();
    for (size_t j = 0; j < g->buckets.size(); ++j) out_list[j] = g->buckets[j];
    for (bid_t b = 0; b < nb * nb; ++b) w->block_walks[b].num = 0;
    return chose ? 1 : 0;
}

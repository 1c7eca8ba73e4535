// Out-of-core kernels: walker records, bucketing, block choice, step kernel.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "gw_kernels.cuh"

namespace gw {

// Device walker record, 32 bytes like the reference's walker_t
// (api/types.hpp:49-56): id, previous, current, hop, prev/cur block (the
// reference's prev_index / cur_index), and the running 64-bit path hash in
// place of the source and totblk words, which the step never reads.
struct __align__(16) WalkerRec {
    uint32_t wid, prev, cur, hop;
    uint32_t prev_blk, cur_blk;
    uint32_t hash_lo, hash_hi;
};
static_assert(sizeof(WalkerRec) == 32, "walker record is 32 bytes");

constexpr uint32_t kFinished = 0xFFFFFFFFu;  // prev_blk of a finished walker
constexpr uint32_t kNoBucket = 0xFFFFFFFFu;  // bucket key of a finished walker
constexpr uint32_t kMaxBlocks = 1024;        // block table kept in shared memory
// cur_blk flag of a walker whose step needs N(prev) while prev's block is
// absent (lazy mode); such walkers sit in the second half of the buckets.
constexpr uint32_t kNeedPrev = 0x80000000u;

struct OocStepArgs {
    StepConsts c;
    const uint64_t *beg;             // [nverts+1] offsets of every vertex (global edge ids), resident
    const uint32_t *const *blk_csr;  // [nb] block neighbours, indexed from estart[b]; null = absent
    const uint2 *const *blk_alias;   // [nb] weighted walks: block alias tables {prob bits, alias column}
    const uint32_t *vstart;          // [nb+1]
    const uint64_t *estart;          // [nb+1]
    uint32_t nb, nverts;
    uint32_t lazy;                   // 1: a walker runs with only its current block resident
    const uint8_t *mapped;           // [nb] zero-copy tail: 1 = read through mapped host memory (counted)
    WalkerRec *recs;                 // one record per walker, never moved
    const uint32_t *order;           // record of each bucket-sorted position
    uint32_t *keys;                  // bucket of each sorted position; kNoBucket once finished
    const uint32_t *run_pre;         // [nrun+1] prefix of runnable bucket sizes
    const uint32_t *run_off;         // [nrun] first walker of each runnable bucket
    const uint32_t *nrun;            // runnable bucket count (device)
    uint32_t *paths;                 // or null
    uint32_t stride;
    uint32_t out_base;               // first walker id of the population: outputs at wid - out_base
    uint32_t *lens;
    uint64_t *hashes;
    unsigned long long *ctr;
    uint32_t *err;
};

// Decision of the block-choice kernel.
struct Decision {
    int32_t action;     // 0 none, 1 add to a free slot, 2 replace the block at `position`
    int32_t block;      // block to load
    int32_t position;   // index in the cached list to replace
    int32_t rescue_block;     // best block by all incident walkers (progress when nothing qualifies)
    int32_t rescue_position;  // cached block with the fewest incident walkers
    uint32_t live;      // live walkers after the last bucketing
    uint64_t score;
};

// Walkers are sorted by bucket through an index: records stay where
// k_init_walkers puts them; `order` and `keys` (record index and bucket of
// each sorted position) are what bucketing moves, 8 bytes per walker.
cudaError_t launch_init_walkers(const WalkerInit &in, const uint32_t *vstart, uint32_t nb, uint32_t wid0, uint64_t n,
                                WalkerRec *recs, uint32_t *order, uint32_t *keys, uint32_t *paths, uint32_t stride,
                                int num_sms, cudaStream_t s);
// `n` points at the number of sorted positions (a device word, so the
// bucketing sequence can be captured once and replayed).
cudaError_t launch_count(const uint32_t *keys, const uint32_t *n, uint32_t *counts, int num_sms, cudaStream_t s);
cudaError_t launch_scan(const uint32_t *counts, uint32_t n, uint32_t *offsets, cudaStream_t s);
cudaError_t launch_scatter(const uint32_t *keys_in, const uint32_t *order_in, const uint32_t *n, const uint32_t *offsets,
                           uint32_t *cursor, uint32_t *keys_out, uint32_t *order_out, int num_sms, cudaStream_t s);
// Buckets are 2 * nb^2: (prev_blk, cur_blk), then the same pairs for walkers
// flagged kNeedPrev.
cudaError_t launch_runnable(const uint32_t *counts, const uint32_t *offsets, const uint32_t *const *blk_csr,
                            uint32_t nb, uint32_t lazy, uint32_t *run_pre, uint32_t *run_off, uint32_t *nrun,
                            cudaStream_t s);
// Counters (kCtrCount) and the error word into out[0 .. kCtrCount] (mapped host memory).
cudaError_t launch_snapshot(const unsigned long long *ctr, const uint32_t *err, unsigned long long *out,
                            cudaStream_t s);
// combined[k] = counts[k] + counts[nb^2 + k]: walkers per (prev, cur) block pair.
cudaError_t launch_combine(const uint32_t *counts, uint32_t nb, uint32_t *combined, int num_sms, cudaStream_t s);
// `counts` are the nb^2 per-pair totals; `live` points at the live-walker count.
cudaError_t launch_schedule(const uint32_t *counts, const uint32_t *live, uint32_t nb, const uint32_t *cached,
                            uint32_t ncached, uint32_t nslots, uint32_t zero_threshold, const float *pred,
                            float pred_weight, Decision *out, cudaStream_t s);
// ---- SOWalker annealing policy (gw_sa.cu): the block set held across
// iterations until all of it is resident
struct SaState {
    uint32_t k;      // size of the held set, 0 = none
    uint32_t calls;  // annealing calls so far (the draws' second counter word)
    uint32_t set[kMaxBlocks];
};
// Anneals a new set when forced, when none is held or when the held one is
// all resident; then (unless forced) points `dec` at the set's first absent
// block.  counts: nb^2 walkers per (prev, cur) block pair.
cudaError_t launch_sa_choose(const uint32_t *counts, uint32_t nb, const uint32_t *cached, uint32_t ncached,
                             uint32_t k, uint64_t seed, bool force, SaState *st, Decision *dec, cudaStream_t s);
// ---- learned policy: per-block features, training targets, decisions

struct FeatureArgs {
    const uint32_t *counts;            // [nb*nb] bucket counts after the last bucketing
    const uint32_t *const *blk_csr;    // residency (non-null = resident)
    const float *emass, *vfrac;        // edge / vertex share of each block, times nb
    float *prev_col, *ema_arr;         // per-block history, updated in place
    uint32_t nb, iter;
    float live_frac, inv_live;
    float *x;                          // [nb][16] features out
    float *col;                        // [nb] walkers waiting with cur block = i (demand) out
};
cudaError_t launch_features(const FeatureArgs &f, cudaStream_t s);
// Samples t0 .. t0+T-1 from the trace ring (iteration t in slot t % ring) into
// train_x, with y[j][i] = log1p(mean demand over t+1 .. t+k) - x[t][i][0]: the
// network forecasts the change of log demand
cudaError_t launch_gather_train(const float *ring_x, const float *ring_col, uint32_t t0, uint32_t ring, uint32_t T,
                                uint32_t k, uint32_t nb, float *train_x, float *y, cudaStream_t s);
// level[i] = res[i] + x[i][0]
cudaError_t launch_add_level(const float *res, const float *x, float *level, uint32_t nb, cudaStream_t s);

int ooc_grid(bool sopr, bool paths, bool coop, int num_sms, bool weighted = false);
cudaError_t launch_walk_ooc(const OocStepArgs &a, bool sopr, bool coop, bool weighted, int grid, cudaStream_t s);

}  // namespace gw

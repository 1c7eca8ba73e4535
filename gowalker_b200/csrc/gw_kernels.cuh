// Launch interfaces of the engine's kernels (internal to libgowalker.so).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "gw_step.cuh"

namespace gw {

constexpr int kWalkThreads = 256;   // threads per CTA of the walk kernels
constexpr uint32_t kChunk = 64;     // walkers a warp claims per atomic

// Work / statistics counters of one run (device, zeroed per run).
enum Counter : int {
    kCtrCursor = 0,   // next walker index to hand out
    kCtrSteps = 1,
    kCtrTrials = 2,
    kCtrDone = 3,
    kCtrHashSum = 4,  // wrapping sum of finished walkers' path hashes
    kCtrCoopSmall = 5,     // hard steps decided from candidate positions (prev degree < 32)
    kCtrCoopSmallAtt = 6,  // attempts those steps took
    kCtrCoopLarge = 7,     // hard steps evaluated with candidate loads and searches
    kCtrCoopLargeAtt = 8,  // attempts those steps took
    kCtrZcSectors = 9,     // out-of-core zero-copy tail: 32-byte sectors read from mapped host memory
    kCtrModelSectors = 10, // out-of-core, blocks resident: the sectors those steps would read from mapped memory
    kCtrRunnable = 11,     // out-of-core: walkers handed to the step kernels (sum over launches)
    kCtrCount = 12
};

// Per-warp statistics a walk kernel keeps in shared memory and adds to the
// Counter slots when it ends.
enum WarpStat : int {
    kWsSteps = 0,
    kWsTrials,
    kWsDone,
    kWsHash,
    kWsCoopSmall,
    kWsCoopSmallAtt,
    kWsCoopLarge,
    kWsCoopLargeAtt,
    kWsCount
};

// Error word bits set by kernels instead of trapping.
enum ErrBit : uint32_t {
    kErrVertexRange = 1u,   // a neighbour id >= nverts
    kErrSource = 2u,        // a walker source >= nverts
    kErrBlock = 4u,         // a vertex outside every block, or a block scheduled absent
    kErrTrials = 8u,        // a step exceeded kMaxAttempts rejection trials
    kErrWeight = 16u,       // an edge weight that is not a positive finite number
};

// Rejection trials allowed for one step before the walker is stopped with
// kErrTrials.  Only degenerate parameters get near it (e.g. alpha = 1 on a
// directed graph whose N(cur) and N(prev) are disjoint): the worst R-MAT case
// of the SOPR rule, a step from a degree-1 vertex into a hub of degree d,
// needs 1 + alpha*d/(1-alpha) trials on average (~1.3e6 for d = 5e6), so a
// cap of 2^26 is never reached by a valid walk.
constexpr uint32_t kMaxAttempts = 1u << 26;

struct WalkerInit {
    uint32_t mode;       // GW_INIT_*
    uint32_t algo;       // GW_NODE2VEC / GW_SOPR / GW_SOSR
    uint32_t wps;        // walkers per vertex
    uint32_t numwalks;   // total walkers (single-source / random)
    uint32_t nverts;
    uint32_t key0, key1; // walk seed (random init)
};

struct IncoreArgs {
    StepConsts c;
    WalkerInit init;
    const uint64_t *beg;       // nverts+1 global offsets
    CsrIndex ix;               // nedges neighbour ids and their sample levels
    uint32_t nverts;
    uint32_t nwalkers;         // walkers of this launch: ids wid_base + i * wid_stride, i < nwalkers
    uint32_t wid_base;
    uint32_t wid_stride;       // 1 for a run; > 1 for the autotuner's sample
    uint32_t out_base;         // first walker id of the population: outputs are indexed by wid - out_base
    uint32_t chunk;            // walkers a warp claims per atomic (0: kChunk); the autotuner picks it
    uint32_t *paths;           // rows indexed by walker id, or null
    uint32_t stride;           // maxhops + 1
    uint32_t *lens;            // vertices per path
    uint64_t *hashes;          // FNV-1a per path
    unsigned long long *ctr;   // Counter slots
    uint32_t *err;             // ErrBit word
    const uint2 *alias;        // weighted Node2vec: {prob bits, alias column} per edge; null when unweighted
};

// Source vertex of walker `wid` (engine/walk.hpp:32-49 per-vertex ids
// v*wps+i; 82-95 and 355-384 single source 1, or 1 and 3 for SOSR).
__device__ __forceinline__ uint32_t walker_source(const WalkerInit &in, uint32_t wid)
{
    if (in.mode == 0u) return wid / in.wps;
    if (in.mode == 1u) {
        if (in.algo == 2u) return wid < in.numwalks / 2 ? 1u : 3u;
        return 1u;
    }
    const U4 r = philox4x32_10(wid, 0xFFFFFFFFu, 0u, kTagInit, in.key0, in.key1);
    return r.x % in.nverts;
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
    return v;
}

// Grid size (CTAs) for a persistent walk kernel on this device.
// `variant` selects the register cap (0: 4 CTAs/SM, 1: 5, 2: 6, 3: 8), see gw_walk.cu.
constexpr int kIncoreVariants = 4;
int incore_grid(bool sopr, bool paths, bool coop, int variant, int num_sms);
cudaError_t launch_walk_incore(const IncoreArgs &a, bool sopr, bool coop, int variant, int grid, cudaStream_t s);
// Weighted Node2vec through the same kernel (candidates from a.alias).
int incore_grid_weighted(bool paths, int variant, int num_sms);
cudaError_t launch_walk_incore_weighted(const IncoreArgs &a, int variant, int grid, cudaStream_t s);

// One launch per hop (gw_walk_hop.cu): walker state between launches.
struct HopState {
    uint32_t *prev, *cur, *hop;
    uint64_t *hash;
};
// Launch `round` (0 .. maxhops-1) of the one-launch-per-hop walk: round 0
// starts every walker; each advances every live walker by one step.
cudaError_t launch_walk_hop(const IncoreArgs &a, const HopState &st, bool sopr, uint32_t round, int num_sms,
                            cudaStream_t s);

// Whether a run needs the warp-cooperative path for hard steps: always for
// SOPR/SOSR (acceptance ~ deg(prev)/deg(cur) next to hubs); for Node2vec
// only when max/min of {1/p, 1/q, 1} exceeds 8 (otherwise a step accepts
// within 1/ratio >= 1/8 per trial and never gets hard).
inline bool needs_coop(uint32_t algo, const StepConsts &c)
{
    return algo != 0u || c.n2v_maxv > 8.0f * c.n2v_minv;
}
// One sample level: dst[j] = src[32 * j] for j < n.
cudaError_t launch_sample_level(const uint32_t *src, uint64_t n, uint32_t *dst, int num_sms, cudaStream_t s);
cudaError_t launch_validate_csr(const uint64_t *beg, const uint32_t *csr, uint32_t nverts, uint64_t nedges,
                                uint32_t *err, int num_sms, cudaStream_t s);

}  // namespace gw

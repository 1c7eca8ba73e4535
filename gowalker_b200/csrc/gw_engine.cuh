// The engine handle (internal).  One per host thread; owns its device memory
// and streams.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>
#include "gw_kernels.cuh"
#include "gw_weighted.cuh"
#include "../../include/gowalker.h"

namespace gw {
struct OocState;
// Step constants of a configuration (fp32 thresholds computed as the
// reference writes them, engine/engine.hpp:169-172).
void consts_from_config(const gw_config &c, StepConsts &k);
}

struct gw_handle {
    gw_config cfg{};
    int num_sms = 0;
    cudaStream_t s_compute = nullptr;  // step kernels, bucketing, scheduler
    cudaStream_t s_copy = nullptr;     // block copies host -> device slots
    cudaEvent_t ev_start = nullptr, ev_kernel0 = nullptr, ev_kernel1 = nullptr, ev_stop = nullptr;
    std::string err;

    // graph (graph_block, engine/cache.hpp:144-193)
    uint32_t nverts = 0;
    uint64_t nedges = 0;
    uint32_t nblocks = 0;
    std::vector<uint32_t> vblocks;
    std::vector<uint64_t> eblocks;
    std::vector<const uint64_t *> host_beg;  // borrowed host blocks
    std::vector<const uint32_t *> host_csr;

    // whole graph on the device (in-core)
    const uint64_t *dev_beg = nullptr;
    const uint32_t *dev_csr = nullptr;
    uint64_t *own_beg = nullptr;
    uint32_t *own_csr = nullptr;
    bool resident = false;
    bool device_graph = false;
    bool validated = false;
    // sample levels of the resident CSR, rebuilt whenever it is validated
    uint32_t *d_index = nullptr;
    uint64_t index_cap = 0;
    const uint32_t *index_lvl[gw::kIdxLevels] = {};
    uint32_t index_nlvl = 0;

    // edge weights (weighted Node2vec, in-core): per host block, or resident
    std::vector<const float *> host_w;
    const float *dev_w = nullptr;
    float *own_w = nullptr;
    bool weighted = false;
    gw::AliasEntry *d_alias = nullptr;  // alias tables, rebuilt when the graph or weights change
    bool alias_ready = false;

    // walker population
    uint64_t nwalkers = 0;      // walkers of the population: ids wid_first .. wid_first + nwalkers - 1
    uint32_t wid_first = 0;     // first walker id (a shard of the whole population)
    uint32_t numwalks_eff = 0;  // walkers of the whole population (SOSR's single-source split uses it)
    bool walkers_ready = false;
    bool ooc_walkers_stale = true;

    // per-walker outputs
    uint32_t *d_paths = nullptr;
    uint32_t *d_lens = nullptr;
    uint64_t *d_hashes = nullptr;
    uint64_t cap_walkers = 0;
    uint64_t cap_path_words = 0;
    uint64_t cap_path_walkers = 0;
    uint32_t path_stride = 0;

    // counters
    unsigned long long *d_ctr = nullptr;
    uint32_t *d_err = nullptr;
    unsigned long long *h_ctr = nullptr;  // pinned: kCtrCount counters + error word
    uint64_t last_hash_sum = 0;
    uint64_t last_steps = 0;

    // autotuner: best register-cap variant per in-core kernel class
    // (sopr, paths, coop) and the measured times of each variant
    int tuned_variant[16] = {-1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1};
    float tuned_ms[16][gw::kIncoreVariants] = {};
    uint32_t tuned_chunk[16] = {};  // walkers per warp claim the autotuner picked per kernel class
    int last_variant = -1;

    // out-of-core state (gw_ooc.cu)
    gw::OocState *ooc = nullptr;

    int fail(int status, const char *fmt, ...);
    int cuda(cudaError_t e, const char *what);
    int init_device();
    void release();
    uint64_t graph_bytes() const;
    bool host_graph_complete() const;
    int upload_whole_graph(cudaStream_t s, uint64_t *h2d);
    int ensure_outputs();
    int build_index(cudaStream_t s);
    int build_alias(cudaStream_t s);
    int run_incore(gw_stats *stats);
    int run_ooc(uint32_t policy, gw_stats *stats);
    void ooc_release();
    void ooc_invalidate(bool blocks_changed);
};

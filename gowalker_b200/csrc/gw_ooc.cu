// Out-of-core engine: device block cache fed from pinned host blocks,
// device bucketing and block choice, zero-copy tail.
//
// Replaces GOWalker's graph_engine::pipe_run / pipeline / zero_gpujob
// (engine/engine.hpp:406-638), the scheduler's copyblocks
// (engine/schedule.hpp:144-197) and gpu/memory.hpp:124-139, 209-224.
//
// Differences by design (B200: 180 GB HBM):
//  - every walker stays in device memory for the whole run (32-byte records,
//    double-buffered), so no walker crosses PCIe; only graph blocks do;
//  - the CPU never walks (no sidewalkupdate pool): walkers whose blocks are
//    absent wait in their bucket;
//  - each run starts from an empty cache, so H2D bytes per run are the whole
//    out-of-core cost of that run.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstring>
#include <vector>
#include <iterator>
#include <map>
#include "gw_engine.cuh"
#include "gw_ooc_kernels.cuh"

namespace gw {

struct OocState {
    uint32_t nb = 0;
    uint32_t nslots = 0;
    uint64_t slot_beg_words = 0, slot_csr_words = 0;
    uint64_t *slot_beg = nullptr;  // nslots * slot_beg_words
    uint32_t *slot_csr = nullptr;  // nslots * slot_csr_words
    std::vector<int> slot_block;   // block held by each slot, -1 = free
    std::vector<int> block_slot;   // slot of each block, -1 = absent
    std::vector<uint32_t> cached;  // the scheduler's cached list (GOwalker_scheduler_t::buckets)

    const uint64_t **h_blk_beg = nullptr;  // pinned mirrors of the block tables
    const uint32_t **h_blk_csr = nullptr;
    const uint64_t **d_blk_beg = nullptr;
    const uint32_t **d_blk_csr = nullptr;
    uint32_t *d_vstart = nullptr;
    uint64_t *d_estart = nullptr;
    uint32_t *h_cached = nullptr;  // pinned
    uint32_t *d_cached = nullptr;

    WalkerRec *w_a = nullptr, *w_b = nullptr;
    uint64_t w_cap = 0;
    uint32_t *d_counts = nullptr, *d_offsets = nullptr, *d_cursor = nullptr;
    uint32_t *d_run_pre = nullptr, *d_run_off = nullptr, *d_nrun = nullptr;
    Decision *d_dec = nullptr, *h_dec = nullptr;

    // zero-copy: device views of the host blocks, and what we registered
    std::vector<const uint64_t *> map_beg;
    std::vector<const uint32_t *> map_csr;
    std::map<uintptr_t, uintptr_t> reg;  // page ranges we registered: start -> end
    bool mapped = false;

    bool ready = false;
};

__global__ void k_validate_block(const uint64_t *beg, const uint32_t *csr, uint32_t nv, uint64_t e0, uint64_t e1,
                                 uint32_t nverts, uint32_t *err)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t t0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool bad = false;
    if (t0 == 0) bad |= (beg[0] != e0) | (beg[nv] != e1);
    for (uint64_t v = t0; v < nv; v += stride) bad |= beg[v] > beg[v + 1];
    for (uint64_t i = t0; i < e1 - e0; i += stride) bad |= csr[i] >= nverts;
    if (__any_sync(0xFFFFFFFFu, bad) && (threadIdx.x & 31u) == 0) atomicOr(err, kErrVertexRange);
}

}  // namespace gw

using namespace gw;

void gw_handle::ooc_release()
{
    if (!ooc) return;
    OocState &o = *ooc;
    cudaSetDevice(cfg.device);
    cudaFree(o.slot_beg);
    cudaFree(o.slot_csr);
    cudaFree((void *)o.d_blk_beg);
    cudaFree((void *)o.d_blk_csr);
    cudaFree(o.d_vstart);
    cudaFree(o.d_estart);
    cudaFree(o.d_cached);
    cudaFree(o.w_a);
    cudaFree(o.w_b);
    cudaFree(o.d_counts);
    cudaFree(o.d_offsets);
    cudaFree(o.d_cursor);
    cudaFree(o.d_run_pre);
    cudaFree(o.d_run_off);
    cudaFree(o.d_nrun);
    cudaFree(o.d_dec);
    if (o.h_blk_beg) cudaFreeHost((void *)o.h_blk_beg);
    if (o.h_blk_csr) cudaFreeHost((void *)o.h_blk_csr);
    if (o.h_cached) cudaFreeHost(o.h_cached);
    if (o.h_dec) cudaFreeHost(o.h_dec);
    for (auto &r : o.reg) cudaHostUnregister((void *)r.first);
    delete ooc;
    ooc = nullptr;
}

void gw_handle::ooc_invalidate()
{
    // host blocks changed: drop mappings so they are rebuilt on demand
    if (!ooc) return;
    cudaSetDevice(cfg.device);
    for (auto &r : ooc->reg) cudaHostUnregister((void *)r.first);
    ooc->reg.clear();
    ooc->mapped = false;
}

static int ooc_setup(gw_handle *h)
{
    if (h->ooc && h->ooc->ready) return GW_OK;
    if (h->nblocks > kMaxBlocks) return h->fail(GW_ERR_ARG, "at most %u blocks (got %u)", kMaxBlocks, h->nblocks);
    if (!h->ooc) h->ooc = new OocState();
    OocState &o = *h->ooc;
    const uint32_t nb = h->nblocks;
    o.nb = nb;
    uint64_t maxv = 0, maxe = 0;
    for (uint32_t b = 0; b < nb; ++b) {
        maxv = std::max<uint64_t>(maxv, (uint64_t)h->vblocks[b + 1] - h->vblocks[b]);
        maxe = std::max<uint64_t>(maxe, h->eblocks[b + 1] - h->eblocks[b]);
    }
    // slots hold the largest block (gpu/memory.hpp:65-107 sizes them the same way)
    o.slot_beg_words = (maxv + 1 + 1) & ~1ull;   // keep slots 16-byte aligned
    o.slot_csr_words = (std::max<uint64_t>(maxe, 1) + 3) & ~3ull;
    const uint64_t slot_bytes = o.slot_beg_words * 8 + o.slot_csr_words * 4;
    uint64_t ns = h->cfg.cache_size / slot_bytes;
    if (ns > nb) ns = nb;
    if (ns < 2) return h->fail(GW_ERR_ARG, "cache of %llu bytes holds fewer than 2 blocks of %llu bytes",
                               (unsigned long long)h->cfg.cache_size, (unsigned long long)slot_bytes);
    o.nslots = (uint32_t)ns;
    int st;
    if ((st = h->cuda(cudaMalloc(&o.slot_beg, o.nslots * o.slot_beg_words * 8), "slot offsets"))) return st;
    if ((st = h->cuda(cudaMalloc(&o.slot_csr, o.nslots * o.slot_csr_words * 4), "slot neighbours"))) return st;
    if ((st = h->cuda(cudaMalloc((void **)&o.d_blk_beg, nb * sizeof(void *)), "block table"))) return st;
    if ((st = h->cuda(cudaMalloc((void **)&o.d_blk_csr, nb * sizeof(void *)), "block table"))) return st;
    if ((st = h->cuda(cudaMallocHost((void **)&o.h_blk_beg, nb * sizeof(void *)), "block table"))) return st;
    if ((st = h->cuda(cudaMallocHost((void **)&o.h_blk_csr, nb * sizeof(void *)), "block table"))) return st;
    if ((st = h->cuda(cudaMalloc(&o.d_vstart, (nb + 1) * sizeof(uint32_t)), "vstart"))) return st;
    if ((st = h->cuda(cudaMalloc(&o.d_estart, (nb + 1) * sizeof(uint64_t)), "estart"))) return st;
    if ((st = h->cuda(cudaMalloc(&o.d_cached, nb * sizeof(uint32_t)), "cached list"))) return st;
    if ((st = h->cuda(cudaMallocHost(&o.h_cached, nb * sizeof(uint32_t)), "cached list"))) return st;
    const uint64_t nbk = (uint64_t)nb * nb;
    if ((st = h->cuda(cudaMalloc(&o.d_counts, nbk * sizeof(uint32_t)), "bucket counts"))) return st;
    if ((st = h->cuda(cudaMalloc(&o.d_offsets, (nbk + 1) * sizeof(uint32_t)), "bucket offsets"))) return st;
    if ((st = h->cuda(cudaMalloc(&o.d_cursor, nbk * sizeof(uint32_t)), "bucket cursors"))) return st;
    if ((st = h->cuda(cudaMalloc(&o.d_run_pre, (nbk + 1) * sizeof(uint32_t)), "runnable prefix"))) return st;
    if ((st = h->cuda(cudaMalloc(&o.d_run_off, nbk * sizeof(uint32_t)), "runnable offsets"))) return st;
    if ((st = h->cuda(cudaMalloc(&o.d_nrun, sizeof(uint32_t)), "runnable count"))) return st;
    if ((st = h->cuda(cudaMalloc(&o.d_dec, sizeof(Decision)), "decision"))) return st;
    if ((st = h->cuda(cudaMallocHost(&o.h_dec, sizeof(Decision)), "decision"))) return st;
    if ((st = h->cuda(cudaMemcpy(o.d_vstart, h->vblocks.data(), (nb + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice),
                      "vstart")))
        return st;
    if ((st = h->cuda(cudaMemcpy(o.d_estart, h->eblocks.data(), (nb + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice),
                      "estart")))
        return st;
    o.slot_block.assign(o.nslots, -1);
    o.block_slot.assign(nb, -1);
    o.ready = true;
    return GW_OK;
}

static int ooc_walkers(gw_handle *h)
{
    OocState &o = *h->ooc;
    if (h->nwalkers > o.w_cap) {
        cudaFree(o.w_a);
        cudaFree(o.w_b);
        o.w_a = o.w_b = nullptr;
        int st;
        if ((st = h->cuda(cudaMalloc(&o.w_a, h->nwalkers * sizeof(WalkerRec)), "walker records"))) return st;
        if ((st = h->cuda(cudaMalloc(&o.w_b, h->nwalkers * sizeof(WalkerRec)), "walker records"))) return st;
        o.w_cap = h->nwalkers;
    }
    return GW_OK;
}

// Make [p, p+bytes) readable by the device at address p.  Blocks handed to
// gw_host_block are often slices of one array: neighbouring blocks share a
// page (their offset ranges even share an entry), and a registration may not
// overlap an earlier one, so only the pages no registration covers yet are
// registered.  Memory that is already pinned (cudaHostAlloc, or registered by
// the caller) is used as it is.  Needs a device that reads registered host
// memory at its host address (checked by the caller).
static int map_range(gw_handle *h, OocState &o, const void *p, uint64_t bytes)
{
    if (!p || !bytes) return GW_OK;
    cudaPointerAttributes a0{}, a1{};
    const char *last = (const char *)p + bytes - 1;
    if (cudaPointerGetAttributes(&a0, p) == cudaSuccess && a0.type == cudaMemoryTypeHost &&
        cudaPointerGetAttributes(&a1, last) == cudaSuccess && a1.type == cudaMemoryTypeHost &&
        a0.devicePointer == p) {
        // both ends pinned, device address = host address: a block is one
        // array, so one pinned allocation covers it
        return GW_OK;
    }
    cudaGetLastError();
    const uintptr_t page = 4096;
    uintptr_t a = (uintptr_t)p & ~(page - 1);
    const uintptr_t b = ((uintptr_t)p + bytes + page - 1) & ~(page - 1);
    while (a < b) {
        // skip pages inside one of our registrations
        auto it = o.reg.upper_bound(a);
        if (it != o.reg.begin()) {
            auto pr = std::prev(it);
            if (pr->second > a) {
                a = pr->second;
                continue;
            }
        }
        uintptr_t end = b;
        if (it != o.reg.end() && it->first < end) end = it->first;
        // pages of the gap that somebody else already pinned are fine as they are
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, (const void *)a) == cudaSuccess && at.type == cudaMemoryTypeHost) {
            a += page;
            continue;
        }
        cudaGetLastError();
        const cudaError_t e = cudaHostRegister((void *)a, end - a, cudaHostRegisterMapped | cudaHostRegisterReadOnly);
        if (e == cudaErrorHostMemoryAlreadyRegistered) {
            cudaGetLastError();  // pinned elsewhere in the range: take it page by page
            a += page;
            continue;
        }
        if (e != cudaSuccess) return h->cuda(e, "cudaHostRegister (zero-copy)");
        o.reg[a] = end;
        a = end;
    }
    return GW_OK;
}

// Map every host block for device reads (zero-copy tail).
static int ooc_map_host(gw_handle *h)
{
    OocState &o = *h->ooc;
    if (o.mapped) return GW_OK;
    int direct = 0;
    cudaDeviceGetAttribute(&direct, cudaDevAttrCanUseHostPointerForRegisteredMem, h->cfg.device);
    if (!direct)
        return h->fail(GW_ERR_STATE, "zero-copy needs a device that reads registered host memory at its host address");
    o.map_beg.assign(o.nb, nullptr);
    o.map_csr.assign(o.nb, nullptr);
    for (uint32_t b = 0; b < o.nb; ++b) {
        const uint64_t nv = (uint64_t)h->vblocks[b + 1] - h->vblocks[b];
        const uint64_t ne = h->eblocks[b + 1] - h->eblocks[b];
        int st;
        if ((st = map_range(h, o, h->host_beg[b], (nv + 1) * 8))) return st;
        if ((st = map_range(h, o, h->host_csr[b], ne * 4))) return st;
        o.map_beg[b] = h->host_beg[b];
        o.map_csr[b] = h->host_csr[b];
    }
    o.mapped = true;
    return GW_OK;
}

int gw_handle::run_ooc(uint32_t policy, gw_stats *stats)
{
    int st;
    if ((st = ooc_setup(this))) return st;
    if ((st = ooc_walkers(this))) return st;
    OocState &o = *ooc;
    const uint32_t nb = o.nb;
    const uint64_t nbk = (uint64_t)nb * nb;
    cudaStream_t s = s_compute;
    const bool sopr = cfg.algorithm != GW_NODE2VEC;
    const bool paths = cfg.record_paths == GW_PATHS_FULL;
    uint64_t h2d = 0, loads = 0, zc_steps = 0;
    uint32_t iters = 0, launches = 0;
    float kernel_ms = 0.f;

    if ((st = cuda(cudaEventRecord(ev_start, s), "event"))) return st;
    // cold cache
    std::fill(o.slot_block.begin(), o.slot_block.end(), -1);
    std::fill(o.block_slot.begin(), o.block_slot.end(), -1);
    o.cached.clear();
    for (uint32_t b = 0; b < nb; ++b) {
        o.h_blk_beg[b] = nullptr;
        o.h_blk_csr[b] = nullptr;
    }
    auto push_tables = [&]() -> int {
        int e;
        if ((e = cuda(cudaMemcpyAsync((void *)o.d_blk_beg, o.h_blk_beg, nb * sizeof(void *), cudaMemcpyHostToDevice, s),
                      "block table")))
            return e;
        return cuda(cudaMemcpyAsync((void *)o.d_blk_csr, o.h_blk_csr, nb * sizeof(void *), cudaMemcpyHostToDevice, s),
                    "block table");
    };
    if ((st = push_tables())) return st;
    if ((st = cuda(cudaMemsetAsync(d_ctr, 0, sizeof(unsigned long long) * kCtrCount, s), "memset"))) return st;
    if ((st = cuda(cudaMemsetAsync(d_err, 0, sizeof(uint32_t), s), "memset"))) return st;

    WalkerInit in{};
    in.mode = cfg.init_mode;
    in.algo = cfg.algorithm;
    in.wps = cfg.walkpersource;
    in.numwalks = numwalks_eff;
    in.nverts = nverts;
    in.key0 = (uint32_t)cfg.seed;
    in.key1 = (uint32_t)(cfg.seed >> 32);
    const uint32_t stride = cfg.maxhops + 1;
    if ((st = cuda(launch_init_walkers(in, o.d_vstart, nb, nwalkers, o.w_a, paths ? d_paths : nullptr, stride, num_sms,
                                       s),
                   "init walkers")))
        return st;
    launches++;
    uint64_t nlive = nwalkers;  // records in w_a (unsorted)

    auto bucketize = [&](uint64_t n) -> int {
        int e;
        if ((e = cuda(cudaMemsetAsync(o.d_counts, 0, nbk * sizeof(uint32_t), s), "memset"))) return e;
        if ((e = cuda(launch_count(o.w_a, n, nb, o.d_counts, num_sms, s), "count"))) return e;
        if ((e = cuda(launch_scan(o.d_counts, (uint32_t)nbk, o.d_offsets, s), "scan"))) return e;
        if ((e = cuda(cudaMemsetAsync(o.d_cursor, 0, nbk * sizeof(uint32_t), s), "memset"))) return e;
        if ((e = cuda(launch_scatter(o.w_a, n, nb, o.d_offsets, o.d_cursor, o.w_b, num_sms, s), "scatter"))) return e;
        launches += 3;
        std::swap(o.w_a, o.w_b);  // w_a: bucket-sorted live walkers
        return GW_OK;
    };
    if ((st = bucketize(nlive))) return st;

    OocStepArgs a{};
    // step constants as for the in-core kernel
    {
        StepConsts &k = a.c;
        k.maxhops = cfg.maxhops;
        k.key0 = (uint32_t)cfg.seed;
        k.key1 = (uint32_t)(cfg.seed >> 32);
        const float inv_p = 1.0f / cfg.p;
        const float inv_q = 1.0f / cfg.q;
        const float mx_q1 = (inv_q < 1.0f) ? 1.0f : inv_q;
        const float mn_q1 = (1.0f < inv_q) ? 1.0f : inv_q;
        k.n2v_maxv = (inv_p < mx_q1) ? mx_q1 : inv_p;
        k.n2v_minv = (mn_q1 < inv_p) ? mn_q1 : inv_p;
        k.inv_p = inv_p;
        k.inv_q = inv_q;
        k.alpha = cfg.alpha;
        k.term_prob = cfg.term_prob;
        k.one_m_alpha = 1.0 - (double)cfg.alpha;
    }
    a.blk_beg = o.d_blk_beg;
    a.blk_csr = o.d_blk_csr;
    a.vstart = o.d_vstart;
    a.estart = o.d_estart;
    a.nb = nb;
    a.nverts = nverts;
    a.run_pre = o.d_run_pre;
    a.run_off = o.d_run_off;
    a.nrun = o.d_nrun;
    a.paths = paths ? d_paths : nullptr;
    a.stride = stride;
    a.lens = d_lens;
    a.hashes = d_hashes;
    a.ctr = d_ctr;
    a.err = d_err;
    const bool coop = needs_coop(cfg.algorithm, a.c);
    int grid = (int)cfg.blockpergrid;
    if (grid <= 0) grid = ooc_grid(sopr, paths, coop, num_sms);

    cudaEvent_t k0 = nullptr, k1 = nullptr;
    cudaEventCreate(&k0);
    cudaEventCreate(&k1);
    auto step = [&]() -> int {
        int e;
        if ((e = cuda(launch_runnable(o.d_counts, o.d_offsets, o.d_blk_beg, nb, o.d_run_pre, o.d_run_off, o.d_nrun, s),
                      "runnable")))
            return e;
        if ((e = cuda(cudaMemsetAsync(d_ctr + kCtrCursor, 0, sizeof(unsigned long long), s), "memset"))) return e;
        a.walkers = o.w_a;
        if ((e = cuda(cudaEventRecord(k0, s), "event"))) return e;
        if ((e = cuda(launch_walk_ooc(a, sopr, coop, grid, s), "walk kernel"))) return e;
        if ((e = cuda(cudaEventRecord(k1, s), "event"))) return e;
        launches += 2;
        return GW_OK;
    };

    const uint32_t kMaxIters = 1u << 20;
    bool done = false;
    while (!done) {
        if (++iters > kMaxIters) {
            st = fail(GW_ERR_STATE, "out-of-core run exceeded %u scheduler iterations", kMaxIters);
            break;
        }
        // ---- block choice on the device, decision read back
        const uint32_t ncached = (uint32_t)o.cached.size();
        for (uint32_t j = 0; j < ncached; ++j) o.h_cached[j] = o.cached[j];
        if (ncached &&
            (st = cuda(cudaMemcpyAsync(o.d_cached, o.h_cached, ncached * sizeof(uint32_t), cudaMemcpyHostToDevice, s),
                       "cached list")))
            break;
        (void)policy;
        if ((st = cuda(launch_schedule(o.d_counts, o.d_offsets, nb, o.d_cached, ncached, o.nslots, cfg.zero_threshold,
                                       nullptr, 0.f, o.d_dec, s),
                       "schedule")))
            break;
        launches++;
        if ((st = cuda(cudaMemcpyAsync(o.h_dec, o.d_dec, sizeof(Decision), cudaMemcpyDeviceToHost, s), "decision")))
            break;
        if ((st = cuda(cudaMemcpyAsync(h_ctr + kCtrCount, d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s),
                       "error word")))
            break;
        if ((st = cuda(cudaStreamSynchronize(s), "schedule sync"))) break;
        if (iters > 1) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, k0, k1) == cudaSuccess) kernel_ms += ms;
        }
        if ((uint32_t)h_ctr[kCtrCount] != 0) {
            st = fail(GW_ERR_GRAPH, "block data failed validation or a kernel reported 0x%x",
                      (uint32_t)h_ctr[kCtrCount]);
            break;
        }
        const Decision d = *o.h_dec;
        nlive = d.live;
        if (nlive == 0) break;

        int load_block = -1, position = -1;
        if (d.action == 1 || d.action == 2) {
            load_block = d.block;
            position = d.action == 2 ? d.position : -1;
        } else if (cfg.zero_copy) {
            // ---- zero-copy tail: every absent block read through mapped host memory
            if ((st = ooc_map_host(this))) break;
            for (uint32_t b = 0; b < nb; ++b)
                if (o.block_slot[b] < 0) {
                    o.h_blk_beg[b] = o.map_beg[b];
                    o.h_blk_csr[b] = o.map_csr[b];
                }
            if ((st = push_tables())) break;
            unsigned long long before[kCtrCount];
            if ((st = cuda(cudaMemcpyAsync(h_ctr, d_ctr, sizeof(before), cudaMemcpyDeviceToHost, s), "counters")))
                break;
            if ((st = cuda(cudaStreamSynchronize(s), "counters"))) break;
            memcpy(before, h_ctr, sizeof(before));
            if ((st = step())) break;
            if ((st = cuda(cudaMemcpyAsync(h_ctr, d_ctr, sizeof(before), cudaMemcpyDeviceToHost, s), "counters")))
                break;
            if ((st = cuda(cudaStreamSynchronize(s), "zero-copy"))) break;
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, k0, k1) == cudaSuccess) kernel_ms += ms;
            zc_steps += h_ctr[kCtrSteps] - before[kCtrSteps];
            // restore the table to device slots only
            for (uint32_t b = 0; b < nb; ++b)
                if (o.block_slot[b] < 0) {
                    o.h_blk_beg[b] = nullptr;
                    o.h_blk_csr[b] = nullptr;
                }
            if ((st = push_tables())) break;
            if ((st = bucketize(nlive))) break;
            iters++;
            done = true;
            break;
        } else if (d.rescue_block >= 0 && (o.cached.size() < o.nslots || d.rescue_position >= 0)) {
            load_block = d.rescue_block;
            position = (o.cached.size() >= o.nslots) ? d.rescue_position : -1;
        } else {
            st = fail(GW_ERR_STATE, "no block can make progress (%u live walkers)", (unsigned)nlive);
            break;
        }

        // ---- load the chosen block into a slot
        int slot = -1;
        if (position >= 0) {
            const uint32_t victim = o.cached[position];
            slot = o.block_slot[victim];
            o.block_slot[victim] = -1;
            o.h_blk_beg[victim] = nullptr;
            o.h_blk_csr[victim] = nullptr;
            o.cached[position] = (uint32_t)load_block;
        } else {
            for (uint32_t k = 0; k < o.nslots; ++k)
                if (o.slot_block[k] < 0) {
                    slot = (int)k;
                    break;
                }
            o.cached.push_back((uint32_t)load_block);
        }
        if (slot < 0) {
            st = fail(GW_ERR_STATE, "no free cache slot");
            break;
        }
        const uint32_t b = (uint32_t)load_block;
        const uint64_t nv = (uint64_t)vblocks[b + 1] - vblocks[b];
        const uint64_t ne = eblocks[b + 1] - eblocks[b];
        uint64_t *sb = o.slot_beg + (uint64_t)slot * o.slot_beg_words;
        uint32_t *sc = o.slot_csr + (uint64_t)slot * o.slot_csr_words;
        if ((st = cuda(cudaMemcpyAsync(sb, host_beg[b], (nv + 1) * 8, cudaMemcpyHostToDevice, s), "block offsets")))
            break;
        if (ne && (st = cuda(cudaMemcpyAsync(sc, host_csr[b], ne * 4, cudaMemcpyHostToDevice, s), "block neighbours")))
            break;
        h2d += (nv + 1) * 8 + ne * 4;
        loads++;
        k_validate_block<<<num_sms * 4, 256, 0, s>>>(sb, sc, (uint32_t)nv, eblocks[b], eblocks[b + 1], nverts, d_err);
        launches++;
        o.slot_block[slot] = (int)b;
        o.block_slot[b] = slot;
        o.h_blk_beg[b] = sb;
        o.h_blk_csr[b] = sc;
        if ((st = push_tables())) break;

        // ---- walk every runnable bucket, then re-bucket
        if ((st = step())) break;
        if ((st = bucketize(nlive))) break;
    }
    if (st == GW_OK) {
        if ((st = cuda(cudaMemcpyAsync(h_ctr, d_ctr, sizeof(unsigned long long) * kCtrCount, cudaMemcpyDeviceToHost, s),
                       "counters D2H")) == GW_OK &&
            (st = cuda(cudaMemcpyAsync(h_ctr + kCtrCount, d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s),
                       "error word")) == GW_OK &&
            (st = cuda(cudaEventRecord(ev_stop, s), "event")) == GW_OK)
            st = cuda(cudaStreamSynchronize(s), "run");
    } else {
        cudaStreamSynchronize(s);
    }
    cudaEventDestroy(k0);
    cudaEventDestroy(k1);
    if (st) return st;
    last_hash_sum = h_ctr[kCtrHashSum];
    last_steps = h_ctr[kCtrSteps];
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->steps = h_ctr[kCtrSteps];
        stats->trials = h_ctr[kCtrTrials];
        stats->walkers = h_ctr[kCtrDone];
        stats->h2d_bytes = h2d;
        stats->d2h_bytes = (uint64_t)iters * (sizeof(Decision) + 4) + sizeof(unsigned long long) * kCtrCount;
        stats->block_loads = loads;
        stats->zero_copy_steps = zc_steps;
        stats->iterations = iters;
        stats->launches = launches;
        stats->kernel_ms = kernel_ms;
        cudaEventElapsedTime(&stats->total_ms, ev_start, ev_stop);
    }
    const uint32_t errw = (uint32_t)h_ctr[kCtrCount];
    if (errw) return fail(GW_ERR_DEVICE, "kernel error word 0x%x", errw);
    if (h_ctr[kCtrDone] != nwalkers)
        return fail(GW_ERR_DEVICE, "out-of-core run finished %llu of %llu walkers", (unsigned long long)h_ctr[kCtrDone],
                    (unsigned long long)nwalkers);
    return GW_OK;
}

extern "C" int gw_bucket_counts(gw_handle *h, uint32_t *out)
{
    if (!h || !out) return GW_ERR_ARG;
    if (!h->ooc || !h->ooc->ready) return h->fail(GW_ERR_STATE, "no bucket counts: the out-of-core path has not run");
    cudaSetDevice(h->cfg.device);
    const uint64_t nbk = (uint64_t)h->ooc->nb * h->ooc->nb;
    return h->cuda(cudaMemcpy(out, h->ooc->d_counts, nbk * sizeof(uint32_t), cudaMemcpyDeviceToHost), "bucket counts");
}

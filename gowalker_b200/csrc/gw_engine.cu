// C ABI of the walk engine: handle, graph residency, walker population, runs.
//
// Replaces the device-side plumbing of GOWalker's graph_engine
// (engine/engine.hpp:54-102, 406-638), gpu/memory.hpp and the walker
// creation of engine/walk.hpp:272-389.  Every failure returns a status and
// records a message; nothing exits the process.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>
#include "gw_engine.cuh"

using namespace gw;

// ------------------------------------------------------------------ helpers

int gw_handle::fail(int status, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    err = buf;
    return status;
}

int gw_handle::cuda(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return GW_OK;
    cudaGetLastError();
    const int st = (e == cudaErrorMemoryAllocation) ? GW_ERR_NOMEM : GW_ERR_CUDA;
    return fail(st, "%s: %s", what, cudaGetErrorString(e));
}

void gw::consts_from_config(const gw_config &c, StepConsts &k)
{
    k.maxhops = c.maxhops;
    k.key0 = (uint32_t)c.seed;
    k.key1 = (uint32_t)(c.seed >> 32);
    // engine/engine.hpp:169-172, in fp32 exactly as the reference writes them
    const float inv_p = 1.0f / c.p;
    const float inv_q = 1.0f / c.q;
    const float mx_q1 = (inv_q < 1.0f) ? 1.0f : inv_q;
    const float mn_q1 = (1.0f < inv_q) ? 1.0f : inv_q;
    k.n2v_maxv = (inv_p < mx_q1) ? mx_q1 : inv_p;
    k.n2v_minv = (mn_q1 < inv_p) ? mn_q1 : inv_p;
    k.inv_p = inv_p;
    k.inv_q = inv_q;
    k.alpha = c.alpha;
    k.term_prob = c.term_prob;
    k.one_m_alpha = 1.0 - (double)c.alpha;
    philox_schedule(k.key0, k.key1, k.rk0, k.rk1);
}

static bool config_ok(const gw_config &c, std::string &why)
{
    if (c.algorithm > GW_SOSR) { why = "algorithm must be 0 (node2vec), 1 (SOPR) or 2 (SOSR)"; return false; }
    if (!(c.p > 0.0f) || !(c.q > 0.0f)) { why = "p and q must be positive"; return false; }
    if (!(c.alpha >= 0.0f) || !(c.alpha <= 1.0f)) { why = "alpha must lie in [0, 1]"; return false; }
    if (!(c.term_prob >= 0.0f) || !(c.term_prob < 1.0f)) { why = "term_prob must lie in [0, 1)"; return false; }
    if (c.init_mode > GW_INIT_RANDOM) { why = "unknown init_mode"; return false; }
    if (c.record_paths > GW_PATHS_FULL) { why = "unknown record_paths"; return false; }
    if (c.launch_mode > GW_LAUNCH_PER_HOP) { why = "unknown launch_mode"; return false; }
    if (c.learned_mode & ~(GW_LEARNED_EVICT | GW_LEARNED_ZERO_SWITCH)) { why = "unknown learned_mode bits"; return false; }
    if (c.threadperblock != 0 && (c.threadperblock % 32 != 0 || c.threadperblock > 1024)) {
        why = "threadperblock must be a multiple of 32 up to 1024";
        return false;
    }
    return true;
}

// ------------------------------------------------------------------ ABI: basics

extern "C" int gw_version(void) { return GW_ABI_VERSION; }

extern "C" const char *gw_status_string(int s)
{
    switch (s) {
    case GW_OK: return "ok";
    case GW_ERR_ARG: return "invalid argument";
    case GW_ERR_CUDA: return "CUDA runtime error";
    case GW_ERR_NOMEM: return "out of memory";
    case GW_ERR_STATE: return "call out of order";
    case GW_ERR_TIMEOUT: return "device wait timed out";
    case GW_ERR_DEVICE: return "kernel reported an error";
    case GW_ERR_GRAPH: return "graph failed validation";
    default: return "unknown status";
    }
}

extern "C" int gw_config_default(gw_config *c)
{
    if (!c) return GW_ERR_ARG;
    memset(c, 0, sizeof(*c));
    c->cache_size = 4ull << 30;    // "memory" 4 GB (api/constants.hpp MEMORY_CACHE)
    c->blocksize = 1024ull << 20;  // "blocksize" 1024 MB
    c->algorithm = GW_NODE2VEC;
    c->p = 0.5f;
    c->q = 2.0f;
    c->alpha = 0.2f;
    c->maxhops = 30;
    c->walkpersource = 1;
    c->numwalks = 0;
    c->init_mode = GW_INIT_PER_VERTEX;
    c->term_prob = 0.0f;
    c->seed = 42;
    c->record_paths = GW_PATHS_NONE;
    c->device = 0;
    return GW_OK;
}

extern "C" int gw_create(const gw_config *cfg, gw_handle **out)
{
    if (!cfg || !out) return GW_ERR_ARG;
    *out = nullptr;
    std::string why;
    if (!config_ok(*cfg, why)) return GW_ERR_ARG;
    gw_handle *h = new (std::nothrow) gw_handle();
    if (!h) return GW_ERR_NOMEM;
    h->cfg = *cfg;
    int st = h->init_device();
    if (st != GW_OK) {
        delete h;
        return st;
    }
    *out = h;
    return GW_OK;
}

extern "C" int gw_destroy(gw_handle *h)
{
    if (!h) return GW_ERR_ARG;
    h->release();
    delete h;
    return GW_OK;
}

extern "C" int gw_last_error(gw_handle *h, char *buf, size_t n)
{
    if (!h || !buf || n == 0) return GW_ERR_ARG;
    snprintf(buf, n, "%s", h->err.c_str());
    return GW_OK;
}

extern "C" int gw_set_config(gw_handle *h, const gw_config *cfg)
{
    if (!h || !cfg) return GW_ERR_ARG;
    std::string why;
    if (!config_ok(*cfg, why)) return h->fail(GW_ERR_ARG, "%s", why.c_str());
    if (cfg->device != h->cfg.device) return h->fail(GW_ERR_ARG, "device cannot change on a live handle");
    const bool paths_grow = cfg->record_paths == GW_PATHS_FULL &&
                            (h->cfg.record_paths != GW_PATHS_FULL || cfg->maxhops != h->cfg.maxhops);
    h->cfg = *cfg;
    if (paths_grow) h->walkers_ready = false;
    return GW_OK;
}

extern "C" int gw_stream(gw_handle *h, void **stream)
{
    if (!h || !stream) return GW_ERR_ARG;
    *stream = (void *)h->s_compute;
    return GW_OK;
}

// ------------------------------------------------------------------ handle internals

int gw_handle::init_device()
{
    int ndev = 0;
    int st = cuda(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
    if (st) return st;
    if (cfg.device < 0 || cfg.device >= ndev) return fail(GW_ERR_ARG, "device %d of %d", cfg.device, ndev);
    if ((st = cuda(cudaSetDevice(cfg.device), "cudaSetDevice"))) return st;
    cudaDeviceProp prop;
    if ((st = cuda(cudaGetDeviceProperties(&prop, cfg.device), "cudaGetDeviceProperties"))) return st;
    num_sms = prop.multiProcessorCount;
    if ((st = cuda(cudaStreamCreateWithFlags(&s_compute, cudaStreamNonBlocking), "stream"))) return st;
    if ((st = cuda(cudaStreamCreateWithFlags(&s_copy, cudaStreamNonBlocking), "stream"))) return st;
    if ((st = cuda(cudaEventCreate(&ev_start), "event"))) return st;
    if ((st = cuda(cudaEventCreate(&ev_kernel0), "event"))) return st;
    if ((st = cuda(cudaEventCreate(&ev_kernel1), "event"))) return st;
    if ((st = cuda(cudaEventCreate(&ev_stop), "event"))) return st;
    if ((st = cuda(cudaMalloc(&d_ctr, sizeof(unsigned long long) * kCtrCount), "counters"))) return st;
    if ((st = cuda(cudaMalloc(&d_err, sizeof(uint32_t)), "error word"))) return st;
    if ((st = cuda(cudaMallocHost(&h_ctr, sizeof(unsigned long long) * (kCtrCount + 1)), "pinned counters")))
        return st;
    memset(h_ctr, 0, sizeof(unsigned long long) * (kCtrCount + 1));
    return GW_OK;
}

void gw_handle::release()
{
    cudaSetDevice(cfg.device);
    if (s_compute) cudaStreamSynchronize(s_compute);
    if (s_copy) cudaStreamSynchronize(s_copy);
    cudaFree(own_beg);
    cudaFree(own_csr);
    cudaFree(own_w);
    cudaFree(d_alias);
    own_w = nullptr;
    d_alias = nullptr;
    alias_ready = false;
    cudaFree(d_paths);
    cudaFree(d_lens);
    cudaFree(d_hashes);
    cudaFree(d_ctr);
    cudaFree(d_err);
    cudaFree(d_index);
    d_index = nullptr;
    index_cap = 0;
    index_nlvl = 0;
    if (h_ctr) cudaFreeHost(h_ctr);
    ooc_release();
    if (ev_start) cudaEventDestroy(ev_start);
    if (ev_kernel0) cudaEventDestroy(ev_kernel0);
    if (ev_kernel1) cudaEventDestroy(ev_kernel1);
    if (ev_stop) cudaEventDestroy(ev_stop);
    if (s_compute) cudaStreamDestroy(s_compute);
    if (s_copy) cudaStreamDestroy(s_copy);
    own_beg = nullptr;
    own_csr = nullptr;
    d_paths = nullptr;
    d_lens = nullptr;
    d_hashes = nullptr;
}

uint64_t gw_handle::graph_bytes() const
{
    return ((uint64_t)nverts + 1) * sizeof(uint64_t) + nedges * sizeof(uint32_t) +
           (weighted ? nedges * (sizeof(float) + sizeof(gw::AliasEntry)) : 0);
}

bool gw_handle::host_graph_complete() const
{
    if (nblocks == 0 || host_beg.size() != nblocks) return false;
    for (uint32_t b = 0; b < nblocks; ++b)
        if (!host_beg[b] || (!host_csr[b] && eblocks[b + 1] > eblocks[b])) return false;
    return true;
}

// Copy every host block into one contiguous device CSR.  Blocks are
// consecutive vertex ranges and their offsets are absolute, so block b's
// nverts offsets land at vblocks[b] and its neighbours at eblocks[b].
int gw_handle::upload_whole_graph(cudaStream_t s, uint64_t *h2d)
{
    int st;
    if (!own_beg) {
        if ((st = cuda(cudaMalloc(&own_beg, ((uint64_t)nverts + 1) * sizeof(uint64_t)), "graph offsets")))
            return st;
        if ((st = cuda(cudaMalloc(&own_csr, (nedges ? nedges : 1) * sizeof(uint32_t)), "graph neighbours")))
            return st;
    }
    uint64_t bytes = 0;
    for (uint32_t b = 0; b < nblocks; ++b) {
        const uint64_t nv = (uint64_t)vblocks[b + 1] - vblocks[b];
        const uint64_t ne = eblocks[b + 1] - eblocks[b];
        const uint64_t nvc = (b + 1 == nblocks) ? nv + 1 : nv;
        if (nvc) {
            if ((st = cuda(cudaMemcpyAsync(own_beg + vblocks[b], host_beg[b], nvc * sizeof(uint64_t),
                                           cudaMemcpyHostToDevice, s), "block offsets H2D")))
                return st;
            bytes += nvc * sizeof(uint64_t);
        }
        if (ne) {
            if ((st = cuda(cudaMemcpyAsync(own_csr + eblocks[b], host_csr[b], ne * sizeof(uint32_t),
                                           cudaMemcpyHostToDevice, s), "block neighbours H2D")))
                return st;
            bytes += ne * sizeof(uint32_t);
        }
    }
    if (weighted && !device_graph) {
        if (!own_w && (st = cuda(cudaMalloc(&own_w, (nedges ? nedges : 1) * sizeof(float)), "edge weights")))
            return st;
        for (uint32_t b = 0; b < nblocks; ++b) {
            const uint64_t ne = eblocks[b + 1] - eblocks[b];
            if (!ne) continue;
            if ((st = cuda(cudaMemcpyAsync(own_w + eblocks[b], host_w[b], ne * sizeof(float), cudaMemcpyHostToDevice,
                                           s), "block weights H2D")))
                return st;
            bytes += ne * sizeof(float);
        }
        dev_w = own_w;
        alias_ready = false;
    }
    dev_beg = own_beg;
    dev_csr = own_csr;
    resident = true;
    validated = false;
    if (h2d) *h2d += bytes;
    return GW_OK;
}

int gw_handle::ensure_outputs()
{
    const uint64_t n = nwalkers;
    const uint32_t stride = cfg.maxhops + 1;
    int st;
    if (n > cap_walkers) {
        cudaFree(d_lens);
        cudaFree(d_hashes);
        d_lens = nullptr;
        d_hashes = nullptr;
        if ((st = cuda(cudaMalloc(&d_lens, n * sizeof(uint32_t)), "path lengths"))) return st;
        if ((st = cuda(cudaMalloc(&d_hashes, n * sizeof(uint64_t)), "path hashes"))) return st;
        cap_walkers = n;
        cap_path_walkers = 0;
    }
    if (cfg.record_paths == GW_PATHS_FULL) {
        const uint64_t need = n * (uint64_t)stride;
        if (need > cap_path_words) {
            cudaFree(d_paths);
            d_paths = nullptr;
            if ((st = cuda(cudaMalloc(&d_paths, need * sizeof(uint32_t)), "paths"))) return st;
            cap_path_words = need;
        }
        path_stride = stride;
        cap_path_walkers = n;
    }
    return GW_OK;
}

// ------------------------------------------------------------------ ABI: graph

extern "C" int gw_set_graph_meta(gw_handle *h, uint32_t nverts, uint64_t nedges, uint32_t nblocks,
                                 const uint32_t *vblocks, const uint64_t *eblocks)
{
    if (!h) return GW_ERR_ARG;
    if (!vblocks || !eblocks || nblocks == 0) return h->fail(GW_ERR_ARG, "block table missing");
    if (vblocks[0] != 0 || vblocks[nblocks] != nverts)
        return h->fail(GW_ERR_GRAPH, "vertex blocks must start at 0 and end at nverts");
    if (eblocks[0] != 0 || eblocks[nblocks] != nedges)
        return h->fail(GW_ERR_GRAPH, "edge blocks must start at 0 and end at nedges");
    for (uint32_t b = 0; b < nblocks; ++b) {
        if (vblocks[b + 1] < vblocks[b] || eblocks[b + 1] < eblocks[b])
            return h->fail(GW_ERR_GRAPH, "block table is not monotone at block %u", b);
    }
    cudaSetDevice(h->cfg.device);
    cudaStreamSynchronize(h->s_compute);
    h->nverts = nverts;
    h->nedges = nedges;
    h->nblocks = nblocks;
    h->vblocks.assign(vblocks, vblocks + nblocks + 1);
    h->eblocks.assign(eblocks, eblocks + nblocks + 1);
    h->host_beg.assign(nblocks, nullptr);
    h->host_csr.assign(nblocks, nullptr);
    h->host_w.assign(nblocks, nullptr);
    h->weighted = false;
    h->dev_w = nullptr;
    cudaFree(h->own_w);
    h->own_w = nullptr;
    h->alias_ready = false;
    h->dev_beg = nullptr;
    h->dev_csr = nullptr;
    h->resident = false;
    h->validated = false;
    cudaFree(h->own_beg);
    cudaFree(h->own_csr);
    h->own_beg = nullptr;
    h->own_csr = nullptr;
    h->ooc_release();
    h->walkers_ready = false;
    return GW_OK;
}

extern "C" int gw_host_block(gw_handle *h, uint32_t blk, const uint64_t *beg, const uint32_t *csr)
{
    if (!h) return GW_ERR_ARG;
    if (blk >= h->nblocks) return h->fail(GW_ERR_ARG, "block %u out of range (%u blocks)", blk, h->nblocks);
    if (!beg) return h->fail(GW_ERR_ARG, "block %u offsets missing", blk);
    const uint64_t nv = (uint64_t)h->vblocks[blk + 1] - h->vblocks[blk];
    if (beg[0] != h->eblocks[blk] || beg[nv] != h->eblocks[blk + 1])
        return h->fail(GW_ERR_GRAPH, "block %u offsets disagree with the edge block table", blk);
    h->host_beg[blk] = beg;
    h->host_csr[blk] = csr;
    h->resident = false;
    h->ooc_invalidate(true);
    return GW_OK;
}

extern "C" int gw_device_graph(gw_handle *h, const uint64_t *d_beg, const uint32_t *d_csr)
{
    if (!h) return GW_ERR_ARG;
    if (h->nblocks == 0) return h->fail(GW_ERR_STATE, "set the graph meta first");
    if (!d_beg || (!d_csr && h->nedges)) return h->fail(GW_ERR_ARG, "device graph pointers missing");
    cudaSetDevice(h->cfg.device);
    cudaFree(h->own_beg);
    cudaFree(h->own_csr);
    h->own_beg = nullptr;
    h->own_csr = nullptr;
    h->dev_beg = d_beg;
    h->dev_csr = d_csr;
    h->resident = true;
    h->device_graph = true;
    h->validated = false;
    h->alias_ready = false;
    return GW_OK;
}

extern "C" int gw_host_weights(gw_handle *h, uint32_t blk, const float *w)
{
    if (!h) return GW_ERR_ARG;
    if (blk >= h->nblocks) return h->fail(GW_ERR_ARG, "block %u out of range (%u blocks)", blk, h->nblocks);
    if (h->device_graph) return h->fail(GW_ERR_STATE, "the graph is on the device: use gw_device_weights");
    if (!w && h->eblocks[blk + 1] > h->eblocks[blk]) return h->fail(GW_ERR_ARG, "block %u weights missing", blk);
    h->host_w[blk] = w;
    bool all = true;
    for (uint32_t b = 0; b < h->nblocks; ++b) all &= h->host_w[b] != nullptr || h->eblocks[b + 1] == h->eblocks[b];
    h->weighted = all;
    h->resident = false;  // the next in-core run uploads the weights with the graph
    h->alias_ready = false;
    h->ooc_release();  // the out-of-core slots and alias tables follow the weights
    return GW_OK;
}

extern "C" int gw_device_weights(gw_handle *h, const float *d_w)
{
    if (!h) return GW_ERR_ARG;
    if (!h->device_graph) return h->fail(GW_ERR_STATE, "gw_device_weights needs a device graph (gw_device_graph)");
    if (!d_w && h->nedges) {
        h->weighted = false;
        h->dev_w = nullptr;
        return GW_OK;
    }
    cudaSetDevice(h->cfg.device);
    cudaFree(h->own_w);
    h->own_w = nullptr;
    h->dev_w = d_w;
    h->weighted = true;
    h->alias_ready = false;
    return GW_OK;
}

extern "C" int gw_cache_reset(gw_handle *h)
{
    if (!h) return GW_ERR_ARG;
    if (h->device_graph) return GW_OK;
    h->resident = false;
    h->ooc_invalidate(false);
    return GW_OK;
}

// ------------------------------------------------------------------ ABI: walkers

extern "C" int gw_init_walkers(gw_handle *h, uint32_t algo, uint32_t wps, uint64_t seed)
{
    return gw_init_walker_range(h, algo, wps, seed, 0, ~0ull);
}

extern "C" int gw_init_walker_range(gw_handle *h, uint32_t algo, uint32_t wps, uint64_t seed, uint64_t first,
                                    uint64_t count)
{
    if (!h) return GW_ERR_ARG;
    if (h->nblocks == 0) return h->fail(GW_ERR_STATE, "set the graph meta first");
    if (algo > GW_SOSR) return h->fail(GW_ERR_ARG, "unknown algorithm %u", algo);
    h->cfg.algorithm = algo;
    h->cfg.seed = seed;
    uint64_t n = 0;
    switch (h->cfg.init_mode) {
    case GW_INIT_PER_VERTEX:
        if (wps == 0) return h->fail(GW_ERR_ARG, "walkpersource must be positive");
        h->cfg.walkpersource = wps;
        n = (uint64_t)h->nverts * wps;
        break;
    case GW_INIT_SINGLE_SOURCE:
        if (h->nverts <= (algo == GW_SOSR ? 3u : 1u))
            return h->fail(GW_ERR_ARG, "single-source walks start at vertex 1 (and 3): graph too small");
        n = h->cfg.numwalks ? h->cfg.numwalks : (uint64_t)h->nverts * (wps ? wps : 1);
        break;
    default:
        n = h->cfg.numwalks ? h->cfg.numwalks : (uint64_t)h->nverts * (wps ? wps : 1);
        break;
    }
    if (n > 0xFFFFFFFFull) return h->fail(GW_ERR_ARG, "walker ids are 32-bit (wid_t); %llu walkers", (unsigned long long)n);
    if (n == 0) return h->fail(GW_ERR_ARG, "no walkers");
    if (first < n && count == ~0ull) count = n - first;  // to the end of the population
    if (first >= n || count == 0 || count > n - first)
        return h->fail(GW_ERR_ARG, "walker range [%llu, +%llu) outside the %llu walkers", (unsigned long long)first,
                       (unsigned long long)count, (unsigned long long)n);
    cudaSetDevice(h->cfg.device);
    h->nwalkers = count;
    h->wid_first = (uint32_t)first;
    h->numwalks_eff = (uint32_t)n;
    int st = h->ensure_outputs();
    if (st) return st;
    h->walkers_ready = true;
    h->ooc_walkers_stale = true;
    return GW_OK;
}

extern "C" int gw_num_walkers(gw_handle *h, uint64_t *n)
{
    if (!h || !n) return GW_ERR_ARG;
    *n = h->walkers_ready ? h->nwalkers : 0;
    return GW_OK;
}

// ------------------------------------------------------------------ ABI: run

// Sample levels of the resident CSR (CsrIndex): level L holds csr[j * 32^L]
// for every j, ceil(nedges / 32^L) words, about 3% of the CSR in all.  Built
// once per graph, after validation.
int gw_handle::build_index(cudaStream_t s)
{
    index_nlvl = 0;
    uint64_t n[kIdxLevels], total = 0;
    uint32_t nl = 0;
    for (uint64_t m = nedges; nl < (uint32_t)kIdxLevels && m > 64; ++nl) {
        m = (m + 31) / 32;
        n[nl] = m;
        total += m;
    }
    if (nl == 0) return GW_OK;
    if (total > index_cap) {
        cudaFree(d_index);
        d_index = nullptr;
        index_cap = 0;
        int st;
        if ((st = cuda(cudaMalloc(&d_index, total * sizeof(uint32_t)), "CSR sample levels"))) return st;
        index_cap = total;
    }
    uint32_t *dst = d_index;
    const uint32_t *src = dev_csr;
    for (uint32_t L = 0; L < nl; ++L) {
        int st;
        if ((st = cuda(launch_sample_level(src, n[L], dst, num_sms, s), "CSR sample level"))) return st;
        index_lvl[L] = dst;
        src = dst;
        dst += n[L];
    }
    index_nlvl = nl;
    return GW_OK;
}

// Alias tables of every vertex from the resident weights: 8 bytes per edge
// kept, 16 bytes per edge of scratch for the construction.
int gw_handle::build_alias(cudaStream_t s)
{
    int st;
    if (!d_alias && (st = cuda(cudaMalloc(&d_alias, (nedges ? nedges : 1) * sizeof(AliasEntry)), "alias tables")))
        return st;
    double *pd = nullptr;
    uint32_t *q = nullptr;
    if ((st = cuda(cudaMalloc(&pd, (nedges ? nedges : 1) * sizeof(double)), "alias scratch"))) return st;
    if ((st = cuda(cudaMalloc(&q, (2 * (nedges ? nedges : 1) + nverts + 2) * sizeof(uint32_t)), "alias scratch"))) {
        cudaFree(pd);
        return st;
    }
    st = cuda(cudaMemsetAsync(d_err, 0, sizeof(uint32_t), s), "memset");
    if (!st) st = cuda(launch_build_alias(dev_beg, dev_w, nverts, pd, q, q + nedges,
                                                      q + 2 * (nedges ? nedges : 1), d_alias, d_err, num_sms, s),
                       "alias build");
    if (!st) st = cuda(cudaMemcpyAsync(h_ctr + kCtrCount, d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "D2H");
    if (!st) st = cuda(cudaStreamSynchronize(s), "alias build");
    cudaFree(pd);
    cudaFree(q);
    if (st) return st;
    if ((uint32_t)h_ctr[kCtrCount] != 0) {
        h_ctr[kCtrCount] = 0;
        return fail(GW_ERR_GRAPH, "edge weights must be positive finite numbers");
    }
    alias_ready = true;
    return GW_OK;
}

int gw_handle::run_incore(gw_stats *stats)
{
    int st;
    cudaStream_t s = s_compute;
    uint64_t h2d = 0;
    if ((st = cuda(cudaEventRecord(ev_start, s), "event"))) return st;
    if (!resident) {
        if ((st = upload_whole_graph(s, &h2d))) return st;
    }
    if ((st = cuda(cudaMemsetAsync(d_err, 0, sizeof(uint32_t), s), "memset"))) return st;
    if (!validated) {
        // One pass over the resident CSR before any walk indexes through it.
        if ((st = cuda(launch_validate_csr(dev_beg, dev_csr, nverts, nedges, d_err, num_sms, s), "validate")))
            return st;
        if ((st = cuda(cudaMemcpyAsync(h_ctr + kCtrCount, d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s),
                       "error word D2H")))
            return st;
        if ((st = cuda(cudaStreamSynchronize(s), "validate"))) return st;
        if ((uint32_t)h_ctr[kCtrCount] != 0) {
            h_ctr[kCtrCount] = 0;
            return fail(GW_ERR_GRAPH, "graph failed validation: offsets not monotone or a neighbour id >= %u",
                        nverts);
        }
        uint64_t ends[2] = {1, 0};
        if ((st = cuda(cudaMemcpy(&ends[0], dev_beg, sizeof(uint64_t), cudaMemcpyDeviceToHost), "beg[0]")))
            return st;
        if ((st = cuda(cudaMemcpy(&ends[1], dev_beg + nverts, sizeof(uint64_t), cudaMemcpyDeviceToHost), "beg[V]")))
            return st;
        if (ends[0] != 0 || ends[1] != nedges)
            return fail(GW_ERR_GRAPH, "graph offsets must run from 0 to nedges (%llu..%llu)",
                        (unsigned long long)ends[0], (unsigned long long)ends[1]);
        if ((st = build_index(s))) return st;
        validated = true;
    }
    if (weighted) {
        if (cfg.algorithm != GW_NODE2VEC)
            return fail(GW_ERR_ARG, "weighted walks are Node2vec walks (algorithm %u given)", cfg.algorithm);
        if (!alias_ready && (st = build_alias(s))) return st;
    }
    IncoreArgs a{};
    consts_from_config(cfg, a.c);
    a.init.mode = cfg.init_mode;
    a.init.algo = cfg.algorithm;
    a.init.wps = cfg.walkpersource;
    a.init.numwalks = numwalks_eff;
    a.init.nverts = nverts;
    a.init.key0 = (uint32_t)cfg.seed;
    a.init.key1 = (uint32_t)(cfg.seed >> 32);
    a.beg = dev_beg;
    a.ix.csr = dev_csr;
    a.ix.nlvl = index_nlvl;
    for (uint32_t L = 0; L < index_nlvl; ++L) a.ix.lvl[L] = index_lvl[L];
    a.nverts = nverts;
    a.nwalkers = (uint32_t)nwalkers;
    a.wid_base = wid_first;
    a.wid_stride = 1;
    a.out_base = wid_first;
    a.paths = (cfg.record_paths == GW_PATHS_FULL) ? d_paths : nullptr;
    a.stride = cfg.maxhops + 1;
    a.lens = d_lens;
    a.hashes = d_hashes;
    a.ctr = d_ctr;
    a.err = d_err;
    const bool sopr = cfg.algorithm != GW_NODE2VEC;
    const bool coop = !weighted && needs_coop(cfg.algorithm, a.c);
    a.alias = weighted ? reinterpret_cast<const uint2 *>(d_alias) : nullptr;
    if (cfg.launch_mode == GW_LAUNCH_PER_HOP) {
        // ---- the plain form: one launch per hop, walker state in memory
        if (weighted) return fail(GW_ERR_ARG, "one launch per hop runs unweighted walks only");
        HopState hs{};
        const uint64_t n = nwalkers;
        int rc = GW_OK;
        if ((rc = cuda(cudaMalloc(&hs.prev, n * 4), "hop state")) || (rc = cuda(cudaMalloc(&hs.cur, n * 4), "hop state")) ||
            (rc = cuda(cudaMalloc(&hs.hop, n * 4), "hop state")) || (rc = cuda(cudaMalloc(&hs.hash, n * 8), "hop state"))) {
            cudaFree(hs.prev);
            cudaFree(hs.cur);
            cudaFree(hs.hop);
            cudaFree(hs.hash);
            return rc;
        }
        const uint32_t rounds = cfg.maxhops ? cfg.maxhops : 1;
        if (!(rc = cuda(cudaMemsetAsync(d_ctr, 0, sizeof(unsigned long long) * kCtrCount, s), "memset")) &&
            !(rc = cuda(cudaEventRecord(ev_kernel0, s), "event"))) {
            for (uint32_t k = 0; k < rounds && !rc; ++k) rc = cuda(launch_walk_hop(a, hs, sopr, k, num_sms, s), "hop launch");
        }
        if (!rc && !(rc = cuda(cudaEventRecord(ev_kernel1, s), "event")) &&
            !(rc = cuda(cudaMemcpyAsync(h_ctr, d_ctr, sizeof(unsigned long long) * kCtrCount, cudaMemcpyDeviceToHost, s),
                        "counters D2H")) &&
            !(rc = cuda(cudaMemcpyAsync(h_ctr + kCtrCount, d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s),
                        "error word D2H")) &&
            !(rc = cuda(cudaEventRecord(ev_stop, s), "event")))
            rc = cuda(cudaStreamSynchronize(s), "walk");
        cudaStreamSynchronize(s);
        cudaFree(hs.prev);
        cudaFree(hs.cur);
        cudaFree(hs.hop);
        cudaFree(hs.hash);
        if (rc) return rc;
        last_hash_sum = h_ctr[kCtrHashSum];
        last_steps = h_ctr[kCtrSteps];
        if (stats) {
            memset(stats, 0, sizeof(*stats));
            stats->steps = h_ctr[kCtrSteps];
            stats->trials = h_ctr[kCtrTrials];
            stats->walkers = h_ctr[kCtrDone];
            stats->h2d_bytes = h2d;
            stats->d2h_bytes = sizeof(unsigned long long) * kCtrCount + sizeof(uint32_t);
            stats->block_loads = h2d ? nblocks : 0;
            stats->iterations = rounds;
            stats->launches = rounds;
            stats->kernel_variant = 0xFFFFFFFFu;
            cudaEventElapsedTime(&stats->kernel_ms, ev_kernel0, ev_kernel1);
            cudaEventElapsedTime(&stats->total_ms, ev_start, ev_stop);
        }
        const uint32_t errw = (uint32_t)h_ctr[kCtrCount];
        if (errw) return fail(GW_ERR_DEVICE, "walk kernel error word 0x%x", errw);
        if (h_ctr[kCtrDone] != nwalkers)
            return fail(GW_ERR_DEVICE, "per-hop walk finished %llu of %llu walkers", (unsigned long long)h_ctr[kCtrDone],
                        (unsigned long long)nwalkers);
        return GW_OK;
    }
    // kernel class for the autotuner: (sopr, paths, coop), weighted Node2vec apart
    const int combo = weighted ? 8 | (a.paths ? 2 : 0) : (sopr ? 4 : 0) | (a.paths ? 2 : 0) | (coop ? 1 : 0);
    auto grid_of = [&](int v, bool paths_on) {
        return weighted ? incore_grid_weighted(paths_on, v, num_sms) : incore_grid(sopr, paths_on, coop, v, num_sms);
    };
    auto launch = [&](const IncoreArgs &x, int v, int g) {
        return weighted ? launch_walk_incore_weighted(x, v, g, s) : launch_walk_incore(x, sopr, coop, v, g, s);
    };
    int variant = tuned_variant[combo];
    // Walkers per warp claim: few lanes idle at the end of a run with small
    // claims, fewer atomics with large ones; the autotuner picks among these.
    static const uint32_t kChunks[] = {16, 64, 256};
    if (cfg.blockpergrid == 0 && variant < 0) {
        // Autotuner: time each register-cap variant with each claim size on
        // this run's walkers (their outputs are rewritten by the full run
        // below) and keep the fastest pair for every later run of this kernel
        // class.  Runs of up to 2^22 walkers are timed whole: with few walkers
        // per lane the tail of the last round decides, and a part of the run
        // would misrank the candidates.  Larger runs are timed on every 16th
        // walker id, which keeps the run's mix of source degrees (R-MAT ids
        // are not random in degree, so a contiguous range would not).  The
        // candidates run in a forward then a reverse pass and keep their best
        // time, so none gains from the caches the previous one warmed.
        const uint32_t stride = nwalkers > (1ull << 22) ? 16u : 1u;
        IncoreArgs c = a;
        c.wid_base = wid_first;
        c.wid_stride = stride;
        c.nwalkers = (uint32_t)(nwalkers / stride);
        constexpr int kCand = kIncoreVariants * 3;
        float best = 1e30f;
        float cand_ms[kCand];
        for (float &m : cand_ms) m = 1e30f;
        for (int i = 0; i < 2 * kCand; ++i) {
            const int k = i < kCand ? i : 2 * kCand - 1 - i;
            const int v = k / 3;
            c.chunk = kChunks[k % 3];
            if ((st = cuda(cudaMemsetAsync(d_ctr, 0, sizeof(unsigned long long) * kCtrCount, s), "memset"))) return st;
            if ((st = cuda(cudaEventRecord(ev_kernel0, s), "event"))) return st;
            if ((st = cuda(launch(c, v, grid_of(v, c.paths != nullptr)), "walk kernel launch (tuning)")))
                return st;
            if ((st = cuda(cudaEventRecord(ev_kernel1, s), "event"))) return st;
            if ((st = cuda(cudaEventSynchronize(ev_kernel1), "tuning"))) return st;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev_kernel0, ev_kernel1);
            cand_ms[k] = std::min(cand_ms[k], ms);
        }
        for (int k = 0; k < kCand; ++k) {
            tuned_ms[combo][k / 3] = std::min(k % 3 == 0 ? 1e30f : tuned_ms[combo][k / 3], cand_ms[k]);
            if (cand_ms[k] < best) {
                best = cand_ms[k];
                variant = k / 3;
                tuned_chunk[combo] = kChunks[k % 3];
            }
        }
        tuned_variant[combo] = variant;
    }
    if (variant < 0) variant = 1;
    last_variant = variant;
    a.chunk = tuned_chunk[combo] ? tuned_chunk[combo] : kChunk;
    if ((st = cuda(cudaMemsetAsync(d_ctr, 0, sizeof(unsigned long long) * kCtrCount, s), "memset"))) return st;
    int grid = (int)cfg.blockpergrid;
    if (grid <= 0) grid = grid_of(variant, a.paths != nullptr);
    if ((st = cuda(cudaEventRecord(ev_kernel0, s), "event"))) return st;
    if ((st = cuda(launch(a, variant, grid), "walk kernel launch"))) return st;
    if ((st = cuda(cudaEventRecord(ev_kernel1, s), "event"))) return st;
    if ((st = cuda(cudaMemcpyAsync(h_ctr, d_ctr, sizeof(unsigned long long) * kCtrCount, cudaMemcpyDeviceToHost, s),
                   "counters D2H")))
        return st;
    if ((st = cuda(cudaMemcpyAsync(h_ctr + kCtrCount, d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s),
                   "error word D2H")))
        return st;
    if ((st = cuda(cudaEventRecord(ev_stop, s), "event"))) return st;
    if ((st = cuda(cudaStreamSynchronize(s), "walk"))) return st;
    last_hash_sum = h_ctr[kCtrHashSum];
    last_steps = h_ctr[kCtrSteps];
    const uint32_t errw = (uint32_t)h_ctr[kCtrCount];
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->steps = h_ctr[kCtrSteps];
        stats->trials = h_ctr[kCtrTrials];
        stats->walkers = h_ctr[kCtrDone];
        stats->h2d_bytes = h2d;
        stats->d2h_bytes = sizeof(unsigned long long) * kCtrCount + sizeof(uint32_t);
        stats->block_loads = h2d ? nblocks : 0;
        stats->iterations = 1;
        stats->launches = 1;
        stats->kernel_variant = (uint32_t)variant;
        stats->walker_chunk = a.chunk;
        stats->coop_small_steps = h_ctr[kCtrCoopSmall];
        stats->coop_small_attempts = h_ctr[kCtrCoopSmallAtt];
        stats->coop_large_steps = h_ctr[kCtrCoopLarge];
        stats->coop_large_attempts = h_ctr[kCtrCoopLargeAtt];
        cudaEventElapsedTime(&stats->kernel_ms, ev_kernel0, ev_kernel1);
        cudaEventElapsedTime(&stats->total_ms, ev_start, ev_stop);
    }
    if (errw) return fail(GW_ERR_DEVICE, "walk kernel error word 0x%x (graph ids out of range)", errw);
    if (h_ctr[kCtrDone] != nwalkers)
        return fail(GW_ERR_DEVICE, "walk kernel finished %llu of %llu walkers", (unsigned long long)h_ctr[kCtrDone],
                    (unsigned long long)nwalkers);
    return GW_OK;
}

extern "C" int gw_run(gw_handle *h, uint32_t policy, gw_stats *stats)
{
    if (!h) return GW_ERR_ARG;
    if (policy > GW_POLICY_SA) return h->fail(GW_ERR_ARG, "unknown policy %u", policy);
    if (h->nblocks == 0) return h->fail(GW_ERR_STATE, "no graph");
    if (!h->walkers_ready) return h->fail(GW_ERR_STATE, "call gw_init_walkers first");
    cudaSetDevice(h->cfg.device);
    int st = h->ensure_outputs();
    if (st) return st;
    const bool incore = h->device_graph || h->graph_bytes() <= h->cfg.cache_size;
    if (incore) {
        if (!h->resident && !h->host_graph_complete())
            return h->fail(GW_ERR_STATE, "graph blocks missing: call gw_host_block for every block");
        return h->run_incore(stats);
    }
    if (!h->host_graph_complete())
        return h->fail(GW_ERR_STATE, "graph blocks missing: call gw_host_block for every block");
    return h->run_ooc(policy, stats);
}

// ------------------------------------------------------------------ ABI: results

namespace {
// Zero every path-row entry past its walk's length (the kernels write a row
// only up to the length; the rest holds whatever the buffer held before).
__global__ void k_zero_tails(uint32_t *rows, const uint32_t *lens, uint64_t n, uint32_t stride)
{
    const uint64_t total = n * stride;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t row = i / stride;
        if (i - row * stride >= __ldg(lens + row)) rows[i] = 0u;
    }
}
}  // namespace

extern "C" int gw_path_lengths(gw_handle *h, uint64_t first, uint64_t n, uint32_t *lens)
{
    if (!h || !lens) return GW_ERR_ARG;
    if (!h->walkers_ready || !h->d_lens) return h->fail(GW_ERR_STATE, "no walk has run");
    if (first + n > h->nwalkers) return h->fail(GW_ERR_ARG, "walker range out of bounds");
    cudaSetDevice(h->cfg.device);
    return h->cuda(cudaMemcpy(lens, h->d_lens + first, n * sizeof(uint32_t), cudaMemcpyDeviceToHost), "lengths D2H");
}

extern "C" int gw_get_paths(gw_handle *h, uint64_t first, uint64_t n, uint32_t *out, uint32_t *lens)
{
    if (!h) return GW_ERR_ARG;
    if (h->cfg.record_paths != GW_PATHS_FULL || !h->d_paths)
        return h->fail(GW_ERR_STATE, "paths were not recorded (record_paths = GW_PATHS_FULL)");
    if (first + n > h->nwalkers) return h->fail(GW_ERR_ARG, "walker range out of bounds");
    cudaSetDevice(h->cfg.device);
    int st;
    if (out && n) {
        // rows end with zeros past the walk's length: padded on the device,
        // then one copy
        k_zero_tails<<<h->num_sms * 8, 256, 0, h->s_compute>>>(h->d_paths + first * h->path_stride, h->d_lens + first,
                                                              n, h->path_stride);
        if ((st = h->cuda(cudaGetLastError(), "path padding"))) return st;
        if ((st = h->cuda(cudaMemcpyAsync(out, h->d_paths + first * h->path_stride,
                                          n * h->path_stride * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->s_compute),
                          "paths D2H")))
            return st;
    }
    if (lens && n) {
        if ((st = h->cuda(cudaMemcpyAsync(lens, h->d_lens + first, n * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                          h->s_compute),
                          "lengths D2H")))
            return st;
    }
    return h->cuda(cudaStreamSynchronize(h->s_compute), "paths D2H");
}

extern "C" int gw_path_hashes(gw_handle *h, uint64_t first, uint64_t n, uint64_t *out)
{
    if (!h || !out) return GW_ERR_ARG;
    if (first + n > h->nwalkers) return h->fail(GW_ERR_ARG, "walker range out of bounds");
    cudaSetDevice(h->cfg.device);
    return h->cuda(cudaMemcpy(out, h->d_hashes + first, n * sizeof(uint64_t), cudaMemcpyDeviceToHost),
                   "hashes D2H");
}

extern "C" int gw_checksum(gw_handle *h, uint64_t *hash_sum, uint64_t *steps)
{
    if (!h) return GW_ERR_ARG;
    if (hash_sum) *hash_sum = h->last_hash_sum;
    if (steps) *steps = h->last_steps;
    return GW_OK;
}

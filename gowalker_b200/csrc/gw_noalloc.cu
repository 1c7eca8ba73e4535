// gw_walk_noalloc: the in-core walk for callers that must not allocate device
// memory.
//
// Some callers cannot let a library call cudaMalloc: a plugin inside a server
// that owns every byte of device memory through its own pool, a runtime that
// forbids allocation once its start-up phase is over, a host language that
// hands the library buffers it manages itself.  For them this entry point
// walks a graph that is already on the device into output buffers the caller
// owns, and allocates nothing: the only memory it needs beyond those buffers
// -- the run's work cursor, its step/trial/walker counters, the path-hash sum
// and the kernels' error word -- lives in the file-scope array below, which
// every device that loads the library keeps until the process exits.
#include <cuda_runtime.h>
#include <cstring>
#include <mutex>
#include "gw_engine.cuh"

namespace {

// 32 words of 8 bytes = 256 bytes: kCtrCount counters, then the error word.
constexpr int kScratchWords = 32;
static_assert(gw::kCtrCount + 1 <= kScratchWords, "scratch holds the counters and the error word");

}  // namespace

static __device__ __align__(256) unsigned long long g_noalloc_scratch[kScratchWords];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
// Device address of g_noalloc_scratch per device, and the CUDA context it was
// looked up in: a cudaDeviceReset in the host process ends that context and
// the module is loaded again (at a new address, maybe) in the next one, so an
// address is reused only while the device's context is the same.
void *g_scratch_addr[kMaxDevices];
void *g_scratch_ctx[kMaxDevices];
typedef int (*CtxGetCurrentFn)(void **);
CtxGetCurrentFn g_ctx_get_current = nullptr;

// The current context of the calling thread (the device's primary context
// once the runtime has used that device), from the driver entry point the
// runtime hands out, so the library links no driver library of its own.
void *current_context()
{
    if (!g_ctx_get_current) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn) {
            cudaGetLastError();
            return nullptr;
        }
        g_ctx_get_current = (CtxGetCurrentFn)fn;
    }
    void *ctx = nullptr;
    return g_ctx_get_current(&ctx) == 0 ? ctx : nullptr;
}

// The array's name is a host-side stand-in in host code; its device address
// comes from cudaGetSymbolAddress, with the device current.
int scratch_address(int device, void **out)
{
    if (device < 0 || device >= kMaxDevices) return GW_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    void *ctx = current_context();
    if (!g_scratch_addr[device] || !ctx || ctx != g_scratch_ctx[device]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return GW_ERR_CUDA;
        }
        g_scratch_addr[device] = p;
        g_scratch_ctx[device] = current_context();
    }
    *out = g_scratch_addr[device];
    return GW_OK;
}

// Restores the calling thread's current device on every return path: the
// callers this entry point serves (plugins, pool-owning hosts) keep their own
// device selection.
struct DeviceGuard {
    int saved = -1;
    DeviceGuard()
    {
        if (cudaGetDevice(&saved) != cudaSuccess) {
            cudaGetLastError();
            saved = -1;
        }
    }
    ~DeviceGuard()
    {
        if (saved >= 0) cudaSetDevice(saved);
    }
};

}  // namespace

extern "C" int gw_walk_noalloc(const gw_config *cfg, const uint64_t *d_beg, const uint32_t *d_csr, uint32_t nverts,
                               uint64_t nedges, uint64_t nwalkers, uint64_t *d_hashes, uint32_t *d_lens,
                               uint32_t *d_paths, void *stream, gw_stats *stats)
{
    using namespace gw;
    if (!cfg || !d_beg || (!d_csr && nedges) || !d_hashes || !d_lens || nverts == 0) return GW_ERR_ARG;
    if (cfg->algorithm > GW_SOSR || !(cfg->p > 0.0f) || !(cfg->q > 0.0f) || !(cfg->alpha >= 0.0f) ||
        !(cfg->alpha <= 1.0f) || !(cfg->term_prob >= 0.0f) || !(cfg->term_prob < 1.0f) ||
        cfg->init_mode > GW_INIT_RANDOM || cfg->record_paths > GW_PATHS_FULL)
        return GW_ERR_ARG;
    if (cfg->record_paths == GW_PATHS_FULL && !d_paths) return GW_ERR_ARG;
    // the walker population the configuration implies must match the caller's buffers
    uint64_t implied;
    if (cfg->init_mode == GW_INIT_PER_VERTEX) {
        if (cfg->walkpersource == 0) return GW_ERR_ARG;
        implied = (uint64_t)nverts * cfg->walkpersource;
    } else {
        if (nverts <= (cfg->algorithm == GW_SOSR ? 3u : 1u) && cfg->init_mode == GW_INIT_SINGLE_SOURCE)
            return GW_ERR_ARG;
        implied = cfg->numwalks ? cfg->numwalks : (uint64_t)nverts * (cfg->walkpersource ? cfg->walkpersource : 1);
    }
    // walker ids are 32-bit (wid_t): larger populations are refused
    if (implied != nwalkers || nwalkers == 0 || nwalkers > 0xFFFFFFFFull) return GW_ERR_ARG;

    DeviceGuard keep_device;
    if (cudaSetDevice(cfg->device) != cudaSuccess) {
        cudaGetLastError();
        return GW_ERR_CUDA;
    }
    void *scratch = nullptr;
    int st = scratch_address(cfg->device, &scratch);
    if (st) return st;
    unsigned long long *ctr = (unsigned long long *)scratch;
    uint32_t *err = (uint32_t *)(ctr + kCtrCount);
    cudaStream_t s = (cudaStream_t)stream;
    int num_sms = 0;
    if (cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, cfg->device) != cudaSuccess) {
        cudaGetLastError();
        return GW_ERR_CUDA;
    }

    // The scratch keeps the previous call's contents: clear it first.
    unsigned long long host_ctr[kCtrCount + 1];
    uint64_t ends[2] = {1, 0};
    cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(unsigned long long) * kScratchWords, s);
    // path rows end with zeros past each walk's length, as gw_get_paths
    // returns them (the kernel writes only the visited entries)
    if (e == cudaSuccess && cfg->record_paths == GW_PATHS_FULL)
        e = cudaMemsetAsync(d_paths, 0, nwalkers * ((uint64_t)cfg->maxhops + 1) * sizeof(uint32_t), s);
    if (e == cudaSuccess) e = launch_validate_csr(d_beg, d_csr, nverts, nedges, err, num_sms, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(host_ctr, ctr, sizeof(host_ctr), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&ends[0], d_beg, sizeof(uint64_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&ends[1], d_beg + nverts, sizeof(uint64_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return GW_ERR_CUDA;
    }
    if ((uint32_t)host_ctr[kCtrCount] != 0 || ends[0] != 0 || ends[1] != nedges) return GW_ERR_GRAPH;

    IncoreArgs a{};
    consts_from_config(*cfg, a.c);
    a.init.mode = cfg->init_mode;
    a.init.algo = cfg->algorithm;
    a.init.wps = cfg->walkpersource;
    a.init.numwalks = (uint32_t)nwalkers;
    a.init.nverts = nverts;
    a.init.key0 = (uint32_t)cfg->seed;
    a.init.key1 = (uint32_t)(cfg->seed >> 32);
    a.beg = d_beg;
    a.ix = CsrIndex{d_csr, {}, 0};  // no sample levels: this entry point allocates nothing
    a.nverts = nverts;
    a.nwalkers = (uint32_t)nwalkers;
    a.wid_stride = 1;
    a.paths = (cfg->record_paths == GW_PATHS_FULL) ? d_paths : nullptr;
    a.stride = cfg->maxhops + 1;
    a.lens = d_lens;
    a.hashes = d_hashes;
    a.ctr = ctr;
    a.err = err;
    const bool sopr = cfg->algorithm != GW_NODE2VEC;
    const bool coop = needs_coop(cfg->algorithm, a.c);
    const int variant = 1;  // 5 CTAs per SM; this entry point keeps no tuning state
    const int grid =
        cfg->blockpergrid ? (int)cfg->blockpergrid : incore_grid(sopr, a.paths != nullptr, coop, variant, num_sms);
    e = launch_walk_incore(a, sopr, coop, variant, grid, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(host_ctr, ctr, sizeof(host_ctr), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return GW_ERR_CUDA;
    }
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->steps = host_ctr[kCtrSteps];
        stats->trials = host_ctr[kCtrTrials];
        stats->walkers = host_ctr[kCtrDone];
        stats->d2h_bytes = sizeof(host_ctr);
        stats->iterations = 1;
        stats->launches = 2;
    }
    if ((uint32_t)host_ctr[kCtrCount] != 0 || host_ctr[kCtrDone] != nwalkers) return GW_ERR_DEVICE;
    return GW_OK;
}

// One launch per hop: the in-core walk in the plain form, for comparison
// with the persistent work-stealing kernel (gw_walk.cu).
//
// This is the shape of the reference's GPU step (gpu/gpuwalk.hpp:193-205: a
// grid-stride loop, one thread per walker, the rejection loop inside the
// thread) cut into one launch per hop: launch k advances every live walker by
// one step and keeps its state (prev, cur, hop, hash) in global memory.  The
// draws, thresholds and acceptance are the persistent kernel's, so the walks
// are identical; what differs is the schedule -- a warp waits for its slowest
// lane every hop (a SOPR step next to a hub takes thousands of trials), lanes
// of finished walkers idle until the last hop, and the state makes a round
// trip through memory every hop.
#include <cuda_runtime.h>
#include <cstdint>
#include "gw_kernels.cuh"
#include "../../include/gowalker.h"

namespace gw {

constexpr uint32_t kHopDone = 0xFFFFFFFFu;  // hop word of a finished walker

template <bool SOPR, bool PATHS>
__global__ void __launch_bounds__(256) k_walk_hop(const __grid_constant__ IncoreArgs a, HopState st, uint32_t round)
{
    const uint64_t *__restrict__ beg = a.beg;
    const uint32_t *__restrict__ csr = a.ix.csr;
    const uint32_t maxhops = a.c.maxhops;
    unsigned long long n_steps = 0, n_trials = 0, n_done = 0, n_hash = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.nwalkers; i += stride) {
        const uint32_t wid = a.wid_base + (uint32_t)i;
        uint32_t prev, cur, hop;
        uint64_t h;
        if (round == 0) {
            const uint32_t src = walker_source(a.init, wid);
            prev = cur = src;
            hop = 0;
            h = hash_init(src);
            if (PATHS) a.paths[i * a.stride] = src;
            if (src >= a.nverts) {
                atomicOr(a.err, kErrSource);
                hop = maxhops;  // finished below
            }
        } else {
            hop = st.hop[i];
            if (hop == kHopDone) continue;
            prev = st.prev[i];
            cur = st.cur[i];
            h = st.hash[i];
        }
        bool done = hop >= maxhops;
        if (!done) {
            U4 r = draw(a.c, wid, hop, 0);
            uint32_t attempt = 1;
            const uint64_t head = __ldg(beg + cur);
            const uint32_t deg = (uint32_t)(__ldg(beg + cur + 1) - head);
            if ((hop > 0 && terminates(a.c, r.z)) || deg == 0) {
                done = true;  // termination draw, or a dead end (engine/engine.hpp:196-199)
            } else {
                const uint64_t phead = __ldg(beg + prev);
                const uint32_t pdeg = (uint32_t)(__ldg(beg + prev + 1) - phead);
                const StepThr t = step_thresholds<SOPR>(a.c, deg, pdeg);
                for (;;) {
                    const uint32_t pos = r.x % deg;
                    const float rv = rand_val(r.y, thr_max<SOPR>(a.c, t));
                    const uint32_t x = __ldg(csr + head + pos);
                    n_trials++;
                    if (accept_candidate<SOPR>(a.c, t, rv, x, prev, cur, a.ix, phead, pdeg)) {
                        hop++;
                        n_steps++;
                        h = hash_step(h, x);
                        if (PATHS) a.paths[i * a.stride + hop] = x;
                        prev = cur;
                        cur = x;
                        if (hop >= maxhops) done = true;
                        else if (x >= a.nverts) {
                            atomicOr(a.err, kErrVertexRange);
                            done = true;
                        }
                        break;
                    }
                    if (attempt >= kMaxAttempts) {
                        atomicOr(a.err, kErrTrials);
                        done = true;
                        break;
                    }
                    r = draw(a.c, wid, hop, attempt++);
                }
            }
        }
        if (done) {
            a.hashes[i] = h;
            a.lens[i] = hop + 1;
            st.hop[i] = kHopDone;
            n_done++;
            n_hash += h;
        } else {
            st.prev[i] = prev;
            st.cur[i] = cur;
            st.hop[i] = hop;
            st.hash[i] = h;
        }
    }
    n_steps = warp_sum(n_steps);
    n_trials = warp_sum(n_trials);
    n_done = warp_sum(n_done);
    n_hash = warp_sum(n_hash);
    if ((threadIdx.x & 31u) == 0) {
        if (n_steps) atomicAdd(&a.ctr[kCtrSteps], n_steps);
        if (n_trials) atomicAdd(&a.ctr[kCtrTrials], n_trials);
        if (n_done) atomicAdd(&a.ctr[kCtrDone], n_done);
        if (n_hash) atomicAdd(&a.ctr[kCtrHashSum], n_hash);
    }
}

cudaError_t launch_walk_hop(const IncoreArgs &a, const HopState &st, bool sopr, uint32_t round, int num_sms,
                            cudaStream_t s)
{
    const uint64_t need = (a.nwalkers + 255) / 256;
    const int grid = (int)(need < (uint64_t)num_sms * 16 ? (need ? need : 1) : (uint64_t)num_sms * 16);
    if (sopr) {
        if (a.paths) k_walk_hop<true, true><<<grid, 256, 0, s>>>(a, st, round);
        else k_walk_hop<true, false><<<grid, 256, 0, s>>>(a, st, round);
    } else {
        if (a.paths) k_walk_hop<false, true><<<grid, 256, 0, s>>>(a, st, round);
        else k_walk_hop<false, false><<<grid, 256, 0, s>>>(a, st, round);
    }
    return cudaGetLastError();
}

}  // namespace gw

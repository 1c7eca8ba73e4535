// SOWalker's annealing block choice on the device (GW_POLICY_SA).
//
// Restates SOwalker_scheduler_t::choose_blocks (engine/schedule.hpp:455-593):
//   1. walkers per (prev, cur) block pair; per block, the walkers whose
//      current block it is (partition_walks);
//   2. blocks ranked by that count (ties by block id: the reference's
//      std::sort leaves them unspecified);
//   3. the first k-1 ranked blocks plus the one block, among the rest, with
//      the most walkers between it and them (the first on ties, none if all
//      are zero);
//   4. simulated annealing over one-for-one swaps with the blocks outside the
//      set: score = walkers inside the set / blocks of the set not yet
//      resident (integer division, as the reference's wid_t / size_t); a
//      better score is taken, a worse positive one with probability
//      exp((y_tmp - y_can) / T) -- here when (y_tmp - y_can) / T > ln(u) for
//      the round's uniform draw u; T from 100 by x0.998 while above 0.001, at
//      most C(nblocks, k) rounds (schedule.hpp:523-583).
// The reference draws with std::rand seeded by the clock; here round i of
// annealing call c draws Philox4x32-10 (i, c, 0, 'SANN') under the walk seed,
// so the choice is reproducible.  A set with every block resident scores 0
// (the reference divides by zero there).
//
// As a policy the set is held until all of it is resident: each scheduler
// iteration loads its first absent block (into a free slot, else over the
// first cached block outside the set, as copyblocks does,
// schedule.hpp:384-437); once all of it is resident and stepped, the next
// iteration anneals a new set from the current counts.  Walks do not depend on
// the policy (counter-based draws), only the order of block loads does.
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include "gw_fixedmath.cuh"
#include "gw_ooc_kernels.cuh"
#include "gw_philox.cuh"
#include "../../include/gowalker.h"

namespace gw {

constexpr uint32_t kTagSa = 0x53414E4Eu;  // 'SANN'
constexpr uint32_t kSaSmemMaxNb = 200;     // counts staged in shared memory up to 200 blocks (160 KB)
constexpr uint32_t kSaMaxRounds = 1u << 20;
constexpr uint32_t kSaDraws = 1024;        // annealing draws made per CTA pass

// ln(u) of a round's 32-bit draw by the fixed steps of fm_log_u32 (the
// oracle restates them): acceptance "d > ln(u)" is the reference's
// "u < exp(d)", with the transcendental moved off the annealing chain into
// the parallel draw pass.
__device__ __forceinline__ double sa_log_draw(uint32_t z) { return fm_log_u32(z); }

__device__ __forceinline__ float sa_score(uint32_t score, uint32_t comm, uint32_t k)
{
    return comm < k ? __uint2float_rn(score / (k - comm)) : 0.f;
}

// One CTA of 1024 threads.  force: anneal regardless of the held set and
// leave `dec` alone (the stand-alone entry point).
__global__ void __launch_bounds__(1024)
    k_sa_choose(const uint32_t *__restrict__ counts, uint32_t nb, const uint32_t *__restrict__ cached,
                uint32_t ncached, uint32_t k, uint32_t key0, uint32_t key1, int force, SaState *st, Decision *dec)
{
    extern __shared__ uint32_t s_bw[];  // nb*nb counts when nb <= kSaSmemMaxNb
    __shared__ uint8_t s_isc[kMaxBlocks];
    __shared__ uint32_t s_idx[kMaxBlocks], s_cand[kMaxBlocks];
    __shared__ unsigned long long s_pw[kMaxBlocks];
    __shared__ unsigned long long s_link[kMaxBlocks];
    __shared__ uint16_t s_pos[kSaDraws], s_tp[kSaDraws];
    __shared__ double s_lnu[kSaDraws];
    __shared__ float s_temp[kSaDraws];
    __shared__ float s_tnext;
    __shared__ unsigned long long s_best, s_score;
    __shared__ int s_need, s_done;
    const uint32_t tid = threadIdx.x, lane = tid & 31u;
    const bool staged = nb <= kSaSmemMaxNb;
    const uint32_t *bw = staged ? s_bw : counts;
    if (k > nb) k = nb;
    for (uint32_t b = tid; b < nb; b += blockDim.x) s_isc[b] = 0;
    if (tid == 0) {
        s_best = 0;
        s_score = 0;
    }
    __syncthreads();
    for (uint32_t j = tid; j < ncached; j += blockDim.x) s_isc[cached[j]] = 1;
    if (staged)
        for (uint32_t i = tid; i < nb * nb; i += blockDim.x) s_bw[i] = counts[i];
    if (tid == 0) {
        int need = force || st->k != k || k == 0;
        if (!need) {
            need = 1;  // anneal again once the held set is all resident
            for (uint32_t j = 0; j < k; ++j)
                if (!s_isc[st->set[j]]) {
                    need = 0;
                    break;
                }
        }
        s_need = need;
    }
    __syncthreads();
    if (s_need) {
        // 1-2. walkers per current block, ranked
        for (uint32_t c = tid; c < nb; c += blockDim.x) {
            unsigned long long w = 0;
            for (uint32_t p = 0; p < nb; ++p) w += bw[p * nb + c];
            s_pw[c] = w;
        }
        __syncthreads();
        for (uint32_t b = tid; b < nb; b += blockDim.x) {
            uint32_t rank = 0;
            const unsigned long long v = s_pw[b];
            for (uint32_t x = 0; x < nb; ++x) rank += (s_pw[x] > v || (s_pw[x] == v && x < b)) ? 1u : 0u;
            s_idx[rank] = b;
        }
        __syncthreads();
        if (k > 0 && k < nb) {
            // 3. the block for rank k-1
            for (uint32_t pi = k - 1 + tid; pi < nb; pi += blockDim.x) {
                const uint32_t p = s_idx[pi];
                unsigned long long w = 0;
                for (uint32_t ci = 0; ci + 1 < k; ++ci) {
                    const uint32_t c = s_idx[ci];
                    w += (unsigned long long)bw[p * nb + c] + bw[c * nb + p];
                }
                if (w) atomicMax(&s_best, (w << 11) | (2047u - pi));
            }
            __syncthreads();
            if (tid == 0 && s_best) {
                const uint32_t bi = 2047u - (uint32_t)(s_best & 2047u);
                const uint32_t t = s_idx[k - 1];
                s_idx[k - 1] = s_idx[bi];
                s_idx[bi] = t;
            }
            __syncthreads();
        }
        for (uint32_t j = tid; j < k; j += blockDim.x) s_cand[j] = s_idx[j];
        __syncthreads();
        for (uint32_t t = tid; t < k * k; t += blockDim.x) {
            const uint32_t v = bw[s_cand[t / k] * nb + s_cand[t % k]];
            if (v) atomicAdd(&s_score, (unsigned long long)v);
        }
        __syncthreads();
        // 4. annealing.  link[x] = walkers between block x and the set (both
        // directions), kept current on every accepted swap, makes a round
        // O(1).  The rounds' draws, their ln(u) and the temperature sequence
        // are made 1024 rounds at a time by the whole CTA; warp 0 then runs
        // the rounds 32 at a time speculatively: every lane evaluates one
        // round against the current set, the first accepting round is
        // applied and the rounds after it are evaluated again -- exactly the
        // sequential chain, since a rejected round changes nothing.
        if (k > 0 && k < nb) {
            for (uint32_t x = tid; x < nb; x += blockDim.x) {
                unsigned long long w = 0;
                for (uint32_t j = 0; j < k; ++j) {
                    const uint32_t c = s_cand[j];
                    w += (unsigned long long)bw[x * nb + c] + bw[c * nb + x];
                }
                s_link[x] = w;
            }
            if (tid == 0) {
                s_done = 0;
                s_tnext = 100.0f;
            }
            const uint32_t call = st->calls;
            // C(nb, k), saturated: the temperature ends the loop after ~5,760 rounds anyway
            const uint32_t kk = min(k, nb - k);
            unsigned long long maxiter = 1;
            for (uint32_t i = 0; i < kk && maxiter <= kSaMaxRounds; ++i) maxiter = maxiter * (nb - i) / (i + 1);
            if (maxiter > kSaMaxRounds) maxiter = kSaMaxRounds;
            uint32_t score = (uint32_t)s_score;  // walkers inside the set: at most all live walkers (< 2^32)
            uint32_t comm = 0;
            for (uint32_t j = 0; j < k; ++j) comm += s_isc[s_cand[j]];
            float ycan = sa_score(score, comm, k);
            __syncthreads();
            for (uint32_t base = 0; !s_done; base += kSaDraws) {
                const uint32_t ri = base + tid;
                if (tid < kSaDraws && ri < maxiter) {
                    const U4 r = philox4x32_10(ri, call, 0u, kTagSa, key0, key1);
                    s_pos[tid] = (uint16_t)(k + r.x % (nb - k));
                    s_tp[tid] = (uint16_t)(r.y % k);
                    s_lnu[tid] = sa_log_draw(r.z);
                }
                if (tid == 0) {
                    float T = s_tnext;
                    for (uint32_t j = 0; j < kSaDraws; ++j) {
                        s_temp[j] = T;
                        T = __fmul_rn(T, 0.998f);
                    }
                    s_tnext = T;
                }
                __syncthreads();
                if (tid < 32) {
                    uint32_t j = 0;
                    bool finished = false;
                    while (j < kSaDraws) {
                        const uint32_t jl = j + lane;
                        const bool valid = jl < kSaDraws && base + jl < maxiter && s_temp[jl] > 0.001f;
                        const unsigned vmask = __ballot_sync(0xFFFFFFFFu, valid);
                        if (vmask == 0) {
                            finished = true;
                            break;
                        }
                        uint32_t pos = 0, tp = 0, out = 0, in = 0, score2 = 0, comm2 = 0;
                        float y2 = 0.f;
                        bool acc = false;
                        if (valid) {
                            pos = s_pos[jl];
                            tp = s_tp[jl];
                            out = s_cand[tp];
                            in = s_idx[pos];
                            const uint32_t b_oo = bw[out * nb + out], b_ii = bw[in * nb + in];
                            const uint32_t b_io = bw[in * nb + out], b_oi = bw[out * nb + in];
                            // the set minus out's links, plus in's links to the set without out
                            score2 = (uint32_t)((unsigned long long)score - (s_link[out] - b_oo) +
                                                (s_link[in] - b_io - b_oi + b_ii));
                            comm2 = comm - s_isc[out] + s_isc[in];
                            y2 = sa_score(score2, comm2, k);
                            acc = y2 > ycan ||
                                  (y2 > 0.f && (double)__fdiv_rn(__fsub_rn(y2, ycan), s_temp[jl]) > s_lnu[jl]);
                        }
                        const unsigned amask = __ballot_sync(0xFFFFFFFFu, acc);
                        if (amask == 0) {
                            j += (uint32_t)__popc(vmask);
                            continue;
                        }
                        const int f = __ffs(amask) - 1;
                        pos = __shfl_sync(0xFFFFFFFFu, pos, f);
                        tp = __shfl_sync(0xFFFFFFFFu, tp, f);
                        out = __shfl_sync(0xFFFFFFFFu, out, f);
                        in = __shfl_sync(0xFFFFFFFFu, in, f);
                        score = __shfl_sync(0xFFFFFFFFu, score2, f);
                        comm = __shfl_sync(0xFFFFFFFFu, comm2, f);
                        ycan = __shfl_sync(0xFFFFFFFFu, y2, f);
                        for (uint32_t x = lane; x < nb; x += 32)
                            s_link[x] += ((unsigned long long)bw[x * nb + in] + bw[in * nb + x]) -
                                         ((unsigned long long)bw[x * nb + out] + bw[out * nb + x]);
                        __syncwarp();
                        if (lane == 0) {
                            s_cand[tp] = in;
                            s_idx[pos] = out;
                        }
                        __syncwarp();
                        j += (uint32_t)f + 1;
                    }
                    if (lane == 0 && finished) s_done = 1;
                }
                __syncthreads();
            }
        }
        __syncthreads();
        for (uint32_t j = tid; j < k; j += blockDim.x) st->set[j] = s_cand[j];
        if (tid == 0) {
            st->k = k;
            st->calls += 1;
        }
        __syncthreads();
    }
    if (force || tid != 0) return;
    // first absent block of the set; its slot: a free one, else the first
    // cached block outside the set
    int32_t blk = -1;
    for (uint32_t j = 0; j < k; ++j)
        if (!s_isc[st->set[j]]) {
            blk = (int32_t)st->set[j];
            break;
        }
    if (blk < 0) return;  // a fresh set already resident: the plain rule's decision stands
    Decision d = *dec;
    if (ncached < k) {
        d.action = 1;
        d.block = blk;
        d.position = (int32_t)ncached;
    } else {
        int32_t pos = -1;
        for (uint32_t j = 0; j < ncached && pos < 0; ++j) {
            bool in_set = false;
            for (uint32_t i = 0; i < k; ++i) in_set |= st->set[i] == cached[j];
            if (!in_set) pos = (int32_t)j;
        }
        d.action = pos >= 0 ? 2 : 0;
        d.block = pos >= 0 ? blk : -1;
        d.position = pos;
    }
    *dec = d;
    __threadfence_system();  // `dec` may be mapped host memory
}

cudaError_t launch_sa_choose(const uint32_t *counts, uint32_t nb, const uint32_t *cached, uint32_t ncached,
                             uint32_t k, uint64_t seed, bool force, SaState *st, Decision *dec, cudaStream_t s)
{
    if (nb == 0 || nb > kMaxBlocks) return cudaErrorInvalidValue;
    const size_t smem = nb <= kSaSmemMaxNb ? (size_t)nb * nb * sizeof(uint32_t) : 0;
    const cudaError_t e = cudaFuncSetAttribute(k_sa_choose, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)(kSaSmemMaxNb * kSaSmemMaxNb * sizeof(uint32_t)));
    if (e != cudaSuccess) return e;
    k_sa_choose<<<1, 1024, smem, s>>>(counts, nb, cached, ncached, k, (uint32_t)seed, (uint32_t)(seed >> 32),
                                      force ? 1 : 0, st, dec);
    return cudaGetLastError();
}

}  // namespace gw

using namespace gw;

extern "C" int gw_sa_choose_blocks(const uint32_t *counts, uint32_t nblocks, const uint32_t *cached,
                                   uint32_t ncached, uint32_t k, uint64_t seed, uint32_t call, uint32_t *out)
{
    if (!counts || !out || (ncached && !cached) || nblocks == 0 || nblocks > kMaxBlocks || ncached > nblocks)
        return GW_ERR_ARG;
    for (uint32_t j = 0; j < ncached; ++j)
        if (cached[j] >= nblocks) return GW_ERR_ARG;
    const uint32_t kk = k < nblocks ? k : nblocks;
    uint32_t *d_counts = nullptr, *d_cached = nullptr;
    SaState *d_st = nullptr;
    int rc = GW_OK;
    SaState h{};
    h.k = 0;
    h.calls = call;
    do {
        if (cudaMalloc(&d_counts, (size_t)nblocks * nblocks * sizeof(uint32_t)) != cudaSuccess ||
            cudaMalloc(&d_cached, (ncached ? ncached : 1) * sizeof(uint32_t)) != cudaSuccess ||
            cudaMalloc(&d_st, sizeof(SaState)) != cudaSuccess) {
            rc = GW_ERR_NOMEM;
            break;
        }
        if (cudaMemcpy(d_counts, counts, (size_t)nblocks * nblocks * sizeof(uint32_t), cudaMemcpyHostToDevice) !=
                cudaSuccess ||
            (ncached && cudaMemcpy(d_cached, cached, ncached * sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess) ||
            cudaMemcpy(d_st, &h, sizeof(SaState), cudaMemcpyHostToDevice) != cudaSuccess ||
            launch_sa_choose(d_counts, nblocks, d_cached, ncached, kk, seed, true, d_st, nullptr, 0) != cudaSuccess ||
            cudaMemcpy(out, (const char *)d_st + offsetof(SaState, set), kk * sizeof(uint32_t),
                       cudaMemcpyDeviceToHost) != cudaSuccess) {
            rc = GW_ERR_CUDA;
            break;
        }
    } while (0);
    if (rc != GW_OK) cudaGetLastError();
    cudaFree(d_counts);
    cudaFree(d_cached);
    cudaFree(d_st);
    return rc;
}

// Weighted Node2vec walks, in-core (the reference has no counterpart: it loads
// edge weights, engine/cache.hpp:71, gpu/memory.hpp:134-137, and never samples
// with them).
//
// Semantics: from cur (with prev), candidate x is drawn in proportion to the
// weight of cur -> x, then accepted by the unweighted rule (1/p if x == prev,
// 1 if x is a neighbour of prev, 1/q otherwise, with the reference's
// thresholds and precision, engine/engine.hpp:209-258): P(x) is proportional
// to w(cur, x) times the Node2vec bias, the usual weighted Node2vec.
// The candidate comes from Walker's alias table of cur's out-edges: column
// i = lane x % deg of the trial's draw (the unweighted rand_pos), coin =
// float(lane w >> 8) * 2^-24; the trial takes column i when coin < prob[i],
// its alias otherwise.  Lanes y (rand value) and z (termination) keep their
// meaning, so a graph whose weights are all equal walks exactly as unweighted.
// The walk itself is the in-core kernel (gw_walk.cu) with its W flag; this
// file builds the alias tables.
//
// Alias tables (Vose's method, per vertex: one thread each, a CTA for each
// vertex above 256 neighbours): the weights are
// summed in double in index order, scaled to p_i = w_i * deg / sum, split
// into a queue of p < 1 and a queue of p >= 1 in index order; repeatedly the
// next small s takes the front large l as its alias (prob[s] = (float)p_s)
// and p_l = (p_l + p_s) - 1, l moving to the back of the small queue when it
// drops below 1; leftovers get probability 1.  Every operation is an IEEE
// double rounded to nearest, so the oracle's C restatement builds the same
// table bit for bit.
#include <cuda_runtime.h>
#include <cstdint>
#include "gw_kernels.cuh"
#include "gw_weighted.cuh"

namespace gw {

constexpr uint64_t kHubDeg = 256;            // vertices above this degree get a CTA each
constexpr uint64_t kHubSmemEntries = 20480;  // their probabilities in shared memory up to this degree (160 KB)

// Vose's loop for one vertex whose probabilities p[0, d) are scaled; the
// queues hold indices in the order they are pushed.  p and the queues may be
// shared or global memory.
__device__ void vose_loop(uint64_t d, double *p, uint32_t *small, uint32_t *large, AliasEntry *out)
{
    uint64_t ns = 0, nl = 0, hs = 0, hl = 0;
    for (uint64_t i = 0; i < d; ++i) {
        if (p[i] < 1.0) small[ns++] = (uint32_t)i;
        else large[nl++] = (uint32_t)i;
    }
    while (hs < ns && hl < nl) {
        const uint32_t sidx = small[hs++], lidx = large[hl];
        out[sidx] = AliasEntry{__double2float_rn(p[sidx]), lidx};
        p[lidx] = __dsub_rn(__dadd_rn(p[lidx], p[sidx]), 1.0);
        if (p[lidx] < 1.0) {
            ++hl;
            small[ns++] = lidx;
        }
    }
    while (hl < nl) {
        const uint32_t lidx = large[hl++];
        out[lidx] = AliasEntry{1.f, lidx};
    }
    while (hs < ns) {
        const uint32_t sidx = small[hs++];
        out[sidx] = AliasEntry{1.f, sidx};
    }
}

// Vertices of degree at most kHubDeg: one thread each.
__global__ void k_build_alias(const uint64_t *__restrict__ beg, const float *__restrict__ w, uint32_t nverts,
                              double *__restrict__ pd, uint32_t *__restrict__ qs, uint32_t *__restrict__ ql,
                              AliasEntry *__restrict__ out, uint32_t *err)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nverts; v += stride) {
        const uint64_t h = beg[v], d = beg[v + 1] - h;
        if (d == 0 || d > kHubDeg) continue;
        double sum = 0.0;
        bool bad = false;
        for (uint64_t i = 0; i < d; ++i) {
            const float wi = w[h + i];
            bad |= !(wi > 0.f && wi < __int_as_float(0x7F800000));
            sum = __dadd_rn(sum, (double)wi);
        }
        if (bad) {
            atomicOr(err, kErrWeight);
            for (uint64_t i = 0; i < d; ++i) out[h + i] = AliasEntry{1.f, (uint32_t)i};
            continue;
        }
        for (uint64_t i = 0; i < d; ++i) pd[h + i] = __ddiv_rn(__dmul_rn((double)w[h + i], (double)d), sum);
        vose_loop(d, pd + h, qs + h, ql + h, out + h);
    }
}

// Vertices of degree above kHubDeg: one CTA each.  The sum stays one
// sequential chain of double additions in index order (thread 0) and the
// loop stays Vose's serial loop, so the tables equal the small-vertex path's;
// the CTA scales the probabilities in parallel and the loop runs on
// shared-memory probabilities (up to kHubSmemEntries), where a serial chain
// of dependent accesses costs far less than in global memory.
__global__ void __launch_bounds__(128)
    k_build_alias_hubs(const uint64_t *__restrict__ beg, const float *__restrict__ w, uint32_t nverts,
                       double *__restrict__ pd, uint32_t *__restrict__ qs, uint32_t *__restrict__ ql,
                       AliasEntry *__restrict__ out, uint32_t *err)
{
    extern __shared__ double s_p[];
    __shared__ double s_sum;
    __shared__ int s_bad;
    for (uint64_t v = blockIdx.x; v < nverts; v += gridDim.x) {
        const uint64_t h = beg[v], d = beg[v + 1] - h;
        if (d <= kHubDeg) continue;  // uniform over the CTA
        if (threadIdx.x == 0) {
            double sum = 0.0;
            bool bad = false;
            for (uint64_t i = 0; i < d; ++i) {
                const float wi = w[h + i];
                bad |= !(wi > 0.f && wi < __int_as_float(0x7F800000));
                sum = __dadd_rn(sum, (double)wi);
            }
            s_sum = sum;
            s_bad = bad ? 1 : 0;
        }
        __syncthreads();
        if (s_bad) {
            if (threadIdx.x == 0) atomicOr(err, kErrWeight);
            for (uint64_t i = threadIdx.x; i < d; i += blockDim.x) out[h + i] = AliasEntry{1.f, (uint32_t)i};
        } else {
            double *p = d <= kHubSmemEntries ? s_p : pd + h;
            const double sum = s_sum;
            for (uint64_t i = threadIdx.x; i < d; i += blockDim.x)
                p[i] = __ddiv_rn(__dmul_rn((double)w[h + i], (double)d), sum);
            __syncthreads();
            if (threadIdx.x == 0) vose_loop(d, p, qs + h, ql + h, out + h);
        }
        __syncthreads();
    }
}

cudaError_t launch_build_alias(const uint64_t *beg, const float *w, uint32_t nverts, double *pd, uint32_t *qs,
                               uint32_t *ql, AliasEntry *out, uint32_t *err, int num_sms, cudaStream_t s)
{
    k_build_alias<<<num_sms * 8, 128, 0, s>>>(beg, w, nverts, pd, qs, ql, out, err);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const size_t smem = kHubSmemEntries * sizeof(double);
    if ((e = cudaFuncSetAttribute(k_build_alias_hubs, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
        cudaSuccess)
        return e;
    k_build_alias_hubs<<<num_sms * 2, 128, smem, s>>>(beg, w, nverts, pd, qs, ql, out, err);
    return cudaGetLastError();
}


}  // namespace gw

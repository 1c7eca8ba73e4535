// Weighted Node2vec walks (gw_weighted.cu), internal to libgowalker.so.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "gw_kernels.cuh"

namespace gw {

// One alias-table column: the probability of keeping the column and the
// index (within the vertex's neighbours) of its alias.
struct AliasEntry {
    float prob;
    uint32_t alias;
};
static_assert(sizeof(AliasEntry) == 8, "one 8-byte load per trial");

// Alias tables of every vertex's out-edges from its weights (w[e] per edge).
// pd, qs, ql: scratch of nedges doubles / u32 / u32; work: nverts + 2 u32.
// A weight that is not positive and finite sets kErrWeight (that vertex gets
// a uniform table).
cudaError_t launch_build_alias(const uint64_t *beg, const float *w, uint32_t nverts, double *pd, uint32_t *qs,
                               uint32_t *ql, uint32_t *work, AliasEntry *out, uint32_t *err, int num_sms,
                               cudaStream_t s);

}  // namespace gw

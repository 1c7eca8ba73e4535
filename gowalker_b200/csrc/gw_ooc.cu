// Out-of-core engine: device block cache, bucketing, block choice.
#include <cuda_runtime.h>
#include "gw_engine.cuh"

namespace gw {
struct OocState {
};
}  // namespace gw

int gw_handle::run_ooc(uint32_t policy, gw_stats *stats)
{
    (void)policy;
    (void)stats;
    return fail(GW_ERR_STATE, "graph does not fit the cache and the out-of-core path is not built yet");
}

void gw_handle::ooc_release()
{
    delete ooc;
    ooc = nullptr;
}

void gw_handle::ooc_invalidate() {}

extern "C" int gw_bucket_counts(gw_handle *h, uint32_t *out)
{
    if (!h || !out) return GW_ERR_ARG;
    return h->fail(GW_ERR_STATE, "no bucket counts: out-of-core path not run");
}

// Measured instruction-issue peak of the walk's random draws.
//
// A rejection trial costs at least one Philox4x32-10 evaluation (the draw
// keyed by walker, hop and attempt), so trials per second are bounded by how
// many such evaluations the device can issue.  This kernel measures that
// bound: every thread evaluates the same keyed generator with the same key
// schedule operand as the step kernels (philox4x32_10_sched), over
// consecutive attempt counters, and folds the outputs into one word so no
// evaluation is dropped.  Nothing else runs per evaluation, so the rate is an
// upper bound for any kernel that draws once per trial.
#include <cuda_runtime.h>
#include "gw_engine.cuh"
#include "gw_step.cuh"

namespace gw {
namespace {

__global__ void __launch_bounds__(256) k_philox_rate(StepConsts c, uint32_t per_thread, uint32_t *sink)
{
    const uint32_t wid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t acc = 0;
    for (uint32_t a = 0; a < per_thread; ++a) {
        const U4 r = draw(c, wid, a >> 8, a);
        acc ^= r.x + r.y + r.z + r.w;
    }
    if (acc == 0x9E3779B9u) sink[0] = wid;  // keeps the evaluations live; almost never taken
}

}  // namespace
}  // namespace gw

extern "C" int gw_philox_rate(int device, uint32_t per_thread, double *evals_per_s, float *ms)
{
    using namespace gw;
    if (!evals_per_s || per_thread == 0) return GW_ERR_ARG;
    int prev = -1;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return GW_ERR_CUDA;
    }
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_philox_rate, 256, 0);
    if (per_sm < 1) per_sm = 1;
    gw_config cfg{};
    gw_config_default(&cfg);
    StepConsts c{};
    consts_from_config(cfg, c);
    uint32_t *sink = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = GW_OK;
    const int grid = sms * per_sm;
    do {
        if (cudaMalloc(&sink, sizeof(uint32_t)) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
            cudaEventCreate(&e1) != cudaSuccess) {
            rc = GW_ERR_CUDA;
            break;
        }
        float best = 1e30f;
        for (int rep = 0; rep < 4 && rc == GW_OK; ++rep) {  // the first launch warms the clocks up
            cudaEventRecord(e0);
            k_philox_rate<<<grid, 256>>>(c, per_thread, sink);
            cudaEventRecord(e1);
            if (cudaEventSynchronize(e1) != cudaSuccess) {
                rc = GW_ERR_CUDA;
                break;
            }
            float t = 0.f;
            cudaEventElapsedTime(&t, e0, e1);
            if (rep > 0 && t < best) best = t;
        }
        if (rc != GW_OK) break;
        *evals_per_s = (double)grid * 256.0 * (double)per_thread / (best * 1e-3);
        if (ms) *ms = best;
    } while (0);
    if (rc != GW_OK) cudaGetLastError();
    cudaFree(sink);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (prev >= 0) cudaSetDevice(prev);
    return rc;
}

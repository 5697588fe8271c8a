// calib.cu -- FP32-pipe and SFU calibration kernels (the measured peaks of the roofline).
//
// Each thread runs 8 independent dependency chains of fused multiply-adds (or SFU ex2)
// in a loop, so issue, not latency, limits the rate.  The result is lane operations per
// second over the whole GPU, measured with CUDA events.
#include <cuda_runtime.h>

#include "context.hpp"

namespace dugma {

__global__ void __launch_bounds__(256) ffma_chains_kernel(float* out, int iters, float a, float b)
{
    float v0 = threadIdx.x * 1e-3f, v1 = v0 + 1.f, v2 = v0 + 2.f, v3 = v0 + 3.f;
    float v4 = v0 + 4.f, v5 = v0 + 5.f, v6 = v0 + 6.f, v7 = v0 + 7.f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            v0 = fmaf(v0, a, b); v1 = fmaf(v1, a, b); v2 = fmaf(v2, a, b); v3 = fmaf(v3, a, b);
            v4 = fmaf(v4, a, b); v5 = fmaf(v5, a, b); v6 = fmaf(v6, a, b); v7 = fmaf(v7, a, b);
        }
    }
    const float s = ((v0 + v1) + (v2 + v3)) + ((v4 + v5) + (v6 + v7));
    if (s == 12345.678f) out[blockIdx.x] = s;   // keeps the chains live
}

__global__ void __launch_bounds__(256) ex2_chains_kernel(float* out, int iters)
{
    float v0 = threadIdx.x * 1e-6f, v1 = v0 + 0.1f, v2 = v0 + 0.2f, v3 = v0 + 0.3f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            v0 = ex2(-v0); v1 = ex2(-v1); v2 = ex2(-v2); v3 = ex2(-v3);
        }
    }
    const float s = (v0 + v1) + (v2 + v3);
    if (s == 12345.678f) out[blockIdx.x] = s;
}

}  // namespace dugma

extern "C" int dugma_calibrate(int what, double* lane_ops_per_s, double* ms)
{
    using namespace dugma;
    if (!lane_ops_per_s) return set_error(DUGMA_ERR_ARG, "calibrate: null argument");
    int dev = 0, sms = 148;
    DUGMA_CK(cudaGetDevice(&dev));
    DUGMA_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    float* out = nullptr;
    DUGMA_CK(cudaMalloc(&out, sizeof(float) * 4096));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = sms * 8, threads = 256;
    const int iters = what == 0 ? 4096 : 1024;
    double best = 0, best_ms = 0;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0);
        if (what == 0) ffma_chains_kernel<<<blocks, threads>>>(out, iters, 0.999f, 1e-3f);
        else ex2_chains_kernel<<<blocks, threads>>>(out, iters);
        cudaEventRecord(e1);
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            cudaFree(out);
            return set_error(DUGMA_ERR_CUDA, "calibration kernel failed");
        }
        float t = 0;
        cudaEventElapsedTime(&t, e0, e1);
        const double ops = (double)blocks * threads * iters * 16.0 * (what == 0 ? 8.0 : 4.0);
        const double rate = ops / (t * 1e-3);
        if (rep > 0 && rate > best) {   // first launch is the warm-up
            best = rate;
            best_ms = t;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    *lane_ops_per_s = best;
    if (ms) *ms = best_ms;
    return DUGMA_OK;
}

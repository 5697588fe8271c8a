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

__global__ void __launch_bounds__(256) ffma2_chains_kernel(float* out, int iters, float a, float b)
{
    const float2 A = make_float2(a, a), B = make_float2(b, b);
    float2 v0 = make_float2(threadIdx.x * 1e-3f, 0.5f), v1 = make_float2(1.f, 1.5f), v2 = make_float2(2.f, 2.5f),
           v3 = make_float2(3.f, 3.5f), v4 = make_float2(4.f, 4.5f), v5 = make_float2(5.f, 5.5f),
           v6 = make_float2(6.f, 6.5f), v7 = make_float2(7.f, 7.5f);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            v0 = ffma2(v0, A, B); v1 = ffma2(v1, A, B); v2 = ffma2(v2, A, B); v3 = ffma2(v3, A, B);
            v4 = ffma2(v4, A, B); v5 = ffma2(v5, A, B); v6 = ffma2(v6, A, B); v7 = ffma2(v7, A, B);
        }
    }
    const float s = ((v0.x + v1.x) + (v2.x + v3.y)) + ((v4.y + v5.x) + (v6.x + v7.y));
    if (s == 12345.678f) out[blockIdx.x] = s;
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

// The bounded-wait path of the pair kernels, exercised on purpose: one mbarrier whose phase
// nothing completes (no arrival, no copy in flight), polled by every thread of one warp
// through mbar_wait_bounded with `polls` polls.  The wait runs out, the error word gets the
// timeout bit and the kernel returns; nothing is left pending on the device.
__global__ void wait_selftest_kernel(uint32_t polls, int* err)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    mbar_wait_bounded(&bar, 0u, err, polls);
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
    const int iters = what == 1 ? 1024 : 4096;
    double best = 0, best_ms = 0;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0);
        if (what == 0) ffma_chains_kernel<<<blocks, threads>>>(out, iters, 0.999f, 1e-3f);
        else if (what == 1) ex2_chains_kernel<<<blocks, threads>>>(out, iters);
        else ffma2_chains_kernel<<<blocks, threads>>>(out, iters / 2, 0.999f, 1e-3f);
        cudaEventRecord(e1);
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            cudaFree(out);
            return set_error(DUGMA_ERR_CUDA, "calibration kernel failed");
        }
        float t = 0;
        cudaEventElapsedTime(&t, e0, e1);
        const double ops = (double)blocks * threads * iters * 16.0 * (what == 1 ? 4.0 : 8.0);
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

extern "C" int dugma_wait_selftest(int polls, int* timed_out)
{
    using namespace dugma;
    if (!timed_out || polls < 1 || polls > (1 << 20))
        return set_error(DUGMA_ERR_ARG, "wait_selftest: need timed_out and 1 <= polls <= 2^20");
    int* err = nullptr;
    DUGMA_CK(cudaMalloc(&err, sizeof(int)));
    int rc = DUGMA_OK, h = 0;
    if (cudaMemset(err, 0, sizeof(int)) != cudaSuccess) rc = set_error(DUGMA_ERR_CUDA, "wait_selftest: memset");
    if (rc == DUGMA_OK) {
        wait_selftest_kernel<<<1, 32>>>((uint32_t)polls, err);
        if (cudaGetLastError() != cudaSuccess || cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = set_error(DUGMA_ERR_CUDA, "wait_selftest: kernel failed");
    }
    cudaFree(err);
    *timed_out = (h >> DUGMA_ERR_TIMEOUT) & 1;
    return rc;
}

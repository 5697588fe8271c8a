// common.cuh -- device helpers shared by the DUGMA sm_100a kernels.
//
// Conventions (identical to the C ABI in include/dugma.h):
//   * points are point-major floats (MATLAB D x N column-major);
//   * per-point covariances are D x D column-major blocks;
//   * R is D x D column-major and moves Y: y' = R y + t (update_sig.cu:247-249);
//   * symmetric matrices are packed (00,11,22,01,02,12) in 3D, (00,11,01) in 2D.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "dugma.h"

namespace dugma {

// ---------------------------------------------------------------------------
// Packed symmetric helpers
// ---------------------------------------------------------------------------
template <int D> struct Sym;
template <> struct Sym<3> {
    static constexpr int N = 6;
    static constexpr int NR = 3;   // rotation degrees of freedom
    __host__ __device__ static constexpr int a(int k) { return k < 3 ? k : (k == 5 ? 1 : 0); }
    __host__ __device__ static constexpr int b(int k) { return k < 3 ? k : (k == 3 ? 1 : 2); }
};
template <> struct Sym<2> {
    static constexpr int N = 3;
    static constexpr int NR = 1;
    __host__ __device__ static constexpr int a(int k) { return k < 2 ? k : 0; }
    __host__ __device__ static constexpr int b(int k) { return k < 2 ? k : 1; }
};

// -1/2 * log2(e): exp(-m/2) = 2^(K_EXP2 * m)
constexpr double K_EXP2 = -0.72134752044448170367996234050095;

// 2^x on the SFU (PTX ex2.approx.ftz.f32; ~2 ulp, denormal results flush to 0)
__device__ __forceinline__ float ex2(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// ---------------------------------------------------------------------------
// Packed FP32 pairs (sm_100 f32x2 arithmetic: two lanes' worth of FP32 work per instruction)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c)
{
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\tmov.b64 rc, {%6, %7};\n\t"
        "fma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return d;
}

__device__ __forceinline__ float2 fadd2(float2 a, float2 b)
{
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}

__device__ __forceinline__ float2 fmul2(float2 a, float2 b)
{
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}

// ---------------------------------------------------------------------------
// Record layouts in HBM (16-byte aligned so tiles can be moved by bulk copy)
// ---------------------------------------------------------------------------
// Streamed target record, one per y_j and pose (64 B):
//   v0 = (y'hi.x, y'hi.y, y'hi.z, lv)   y'hi = float(y'), lv = log2(v_j) - Lmax (<= 0, -inf: neglected/padding)
//   v1 = (y'lo.x, y'lo.y, y'lo.z, 0)    y'lo = float(y' - y'hi)
//   v2 = (c00, c11, c22, c01)           k * C'_j packed, k = -1/2 log2 e
//   v3 = (c02, c12, 0, 0)               (off-diagonals doubled in the Horner layout)
// In 2D the z components are 0 and v2 = (c00, c11, c01, 0).
struct __align__(16) YRec {
    float4 v0, v1, v2, v3;
};

// Paired target record (128 B) for the packed f32x2 kernels: targets 2p and 2p+1 side by side.
// Field f (f = 0..15) is the float2 (value of target 2p, value of target 2p+1):
//   f0..f2  -y'hi,  f3 lv,  f4..f6  -y'lo,  f7 + k  k C'_j packed entry k (Sym order),
//   f13 -lv, rest 0.
// Coordinates are stored negated so that d = (x + f0) + f4 needs only packed adds.
struct __align__(16) YRec2 {
    float4 q[8];   // q[k] = (field 2k even, field 2k odd, field 2k+1 even, field 2k+1 odd)
};

// Source record, one per x_i and sigma (64 B), in one of two forms:
//   v0 = (x.x, x.y, x.z, lw)            lw = log2(w_i) - Lmax_x
//   v1 = (0, 0, 0, 0)
// Horner form (scalar kernels):
//   v2 = (b00, b11, b22, 2 b01)         k * B_i packed, off-diagonals doubled
//   v3 = (2 b02, 2 b12, 0, 0)
// Cholesky form (packed kernels): U upper triangular with U^T U = |k| B_i, so the exponent is
// lv - |U d|^2, a sum of squares whatever the condition of B_i
//   v2 = (u00, u11, u22, u01)
//   v3 = (u02, u12, 0, 0)
// In 2D v2 = (b00, b11, 2 b01, 0) or (u00, u11, u01, 0).
struct __align__(16) XRec {
    float4 v0, v1, v2, v3;
};

// Upper Cholesky factor of a symmetric positive definite D x D matrix, both packed in Sym order
// (3D: 00, 11, 22, 01, 02, 12; 2D: 00, 11, 01): U^T U = P.  Returns false, with u zeroed, when a
// pivot is not above 1e-13 times its diagonal entry (P not safely positive definite).
template <int D>
__device__ inline bool chol_upper(const double* p, double* u)
{
    constexpr double kRel = 1e-13;
    bool ok = p[0] > 0.0;
    double u00 = ok ? sqrt(p[0]) : 0.0;
    if (D == 2) {
        const double u01 = ok ? p[2] / u00 : 0.0;
        const double piv = p[1] - u01 * u01;
        ok = ok && piv > kRel * p[1] && isfinite(piv);
        u[0] = u00;
        u[1] = ok ? sqrt(piv) : 0.0;
        u[2] = u01;
    } else {
        const double u01 = ok ? p[3] / u00 : 0.0, u02 = ok ? p[4] / u00 : 0.0;
        const double piv1 = p[1] - u01 * u01;
        ok = ok && piv1 > kRel * p[1];
        const double u11 = ok ? sqrt(piv1) : 1.0;
        const double u12 = (p[5] - u01 * u02) / u11;
        const double piv2 = p[2] - u02 * u02 - u12 * u12;
        ok = ok && piv2 > kRel * p[2] && isfinite(piv2);
        u[0] = u00;
        u[1] = u11;
        u[2] = ok ? sqrt(piv2) : 0.0;
        u[3] = u01;
        u[4] = u02;
        u[5] = u12;
    }
    if (!ok)
        for (int k = 0; k < (D == 3 ? 6 : 3); ++k) u[k] = 0.0;
    return ok;
}

// Coefficient-pass records (128 B): the 64-B record followed by the degree <= 2 monomials
// of the point, g = (1, v_0..v_{D-1}, packed v_a v_b) (10 in 3D, 6 in 2D), zero padded.
struct __align__(16) Rec128 {
    float4 v0, v1, v2, v3;
    float g[16];
};

// ---------------------------------------------------------------------------
// Programmatic dependent launch.  A kernel launched by launch_dependent() may be scheduled
// before the kernel ahead of it in the stream has finished: it calls pdl_wait() before it touches
// any memory that kernel writes or reads (pdl_wait returns once that kernel has completed and its
// writes are visible), and the kernel ahead calls pdl_trigger() to let it be scheduled early (it
// is scheduled only after every block of the kernel ahead has started, so it never takes an SM a
// block of that kernel still needs).  In a kernel launched without the attribute both are no-ops.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_dependent(bool pdl, void (*fn)(KArgs...), dim3 grid, dim3 block, size_t smem,
                                    cudaStream_t s, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, fn, args...);
}

// ---------------------------------------------------------------------------
// Bulk copy (TMA engine, non-tensor form) + mbarrier with bounded waits
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// global -> shared bulk copy completing on an mbarrier (no multicast).
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: gives up after `limit` polls (each poll may suspend the thread for a
// hardware-chosen interval), records DUGMA_ERR_TIMEOUT in *err and returns false.
constexpr uint32_t kWaitPolls = 1u << 24;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* err,
                                                  uint32_t limit = kWaitPolls)
{
    for (uint32_t it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    if (err) atomicOr(err, 1 << DUGMA_ERR_TIMEOUT);
    return false;
}

// ---------------------------------------------------------------------------
// Reductions
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum NV doubles per thread over the block (fixed order => deterministic); result valid in thread 0.
template <int NV, int NT>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* scratch /* [NT/32][NV] */)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) scratch[warp * NV + k] = v[k];
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double s = 0;
            for (int w = 0; w < NT / 32; ++w) s += scratch[w * NV + k];
            v[k] = s;
        }
    }
    __syncthreads();
}

}  // namespace dugma

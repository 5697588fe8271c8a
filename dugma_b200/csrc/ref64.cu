// ref64.cu -- the REF energy at the reference's per-pair precision (the plain form).
//
// compi.cu:732-772 evaluates each pair in FP64: d = x_i - (R y_j + t), the rotated
// target inverse covariance C'_j = R A_j R^T, both Mahalanobis forms and both exp() calls,
// on FP32 inputs (the init-time FP32 copies of the clouds and inverse covariances).  This
// kernel keeps exactly that precision: per-pose FP64 records of y'_j and C'_j (computed
// once per target instead of once per pair; the values are the same FP64 expressions),
// FP64 sources, FP64 quadratic forms and CUDA's double-precision exp().  It is the
// reference-precision arm of the plain energy + finite-difference form; the FP32 kernels
// in energy.cu are the optimised arm.
#include <cmath>

#include "pairs.cuh"
#include "context.hpp"

namespace dugma {

// 128-byte FP64 record: p[0..D) the point (y' for targets, x for sources), m[0..NS) the
// packed symmetric matrix scaled by -1/2 with off-diagonals doubled (C' for targets,
// B = s Sigma_x^-1 for sources), w the weight |Sigma|^-1/2 s^(D/2) (0 when neglected).
struct __align__(16) Rec64 {
    double p[3];
    double m[6];
    double w;
    double pad[6];
};
static_assert(sizeof(Rec64) == 128, "Rec64 is 128 bytes");

template <int D>
__global__ void ref64_prologue_kernel(const double* __restrict__ pose, const float* __restrict__ y,
                                      const float* __restrict__ yinv, const float* __restrict__ wy, int M, int M_pad,
                                      Rec64* __restrict__ yr, const float* __restrict__ x,
                                      const float* __restrict__ xinv, const float* __restrict__ wx, int N, int N_pad,
                                      Rec64* __restrict__ xr)
{
    constexpr int NS = Sym<D>::N;
    double R[9], t[3];
    for (int k = 0; k < D * D; ++k) R[k] = pose[k];
    for (int a = 0; a < D; ++a) t[a] = pose[kPoseT + a];
    const double s = 1.0 / pose[kPoseSig];
    const double ws = D == 3 ? s * sqrt(s) : s;
    const int stride = gridDim.x * blockDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < M_pad; j += stride) {
        Rec64 r = {};
        if (j < M) {
            for (int a = 0; a < D; ++a) {
                double v = R[a] * (double)y[(size_t)j * D] + R[a + D] * (double)y[(size_t)j * D + 1];
                if (D == 3) v = v + R[a + 6] * (double)y[(size_t)j * D + 2];
                r.p[a] = v + t[a];
            }
            // C' = R (s A) R^T with A the stored (column-major) inverse covariance
            double T[3][3];
            for (int r0 = 0; r0 < D; ++r0)
                for (int c0 = 0; c0 < D; ++c0) {
                    double acc = 0;
                    for (int k = 0; k < D; ++k) acc += (double)yinv[(size_t)j * D * D + r0 + D * k] * R[c0 + D * k];
                    T[r0][c0] = acc;
                }
            for (int k = 0; k < NS; ++k) {
                const int ra = Sym<D>::a(k), rb = Sym<D>::b(k);
                double acc = 0, acc2 = 0;
                for (int q = 0; q < D; ++q) {
                    acc += R[ra + D * q] * T[q][rb];
                    acc2 += R[rb + D * q] * T[q][ra];
                }
                // -1/2 s (C'_ab + C'_ba) for off-diagonals, -1/2 s C'_aa on the diagonal
                r.m[k] = -0.5 * s * (ra == rb ? acc : acc + acc2);
            }
            r.w = (double)wy[j] * ws;
        }
        yr[j] = r;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N_pad; i += stride) {
        Rec64 r = {};
        if (i < N) {
            for (int a = 0; a < D; ++a) r.p[a] = (double)x[(size_t)i * D + a];
            for (int k = 0; k < NS; ++k) {
                const int ra = Sym<D>::a(k), rb = Sym<D>::b(k);
                const double bab = (double)xinv[(size_t)i * D * D + ra + D * rb];
                const double bba = (double)xinv[(size_t)i * D * D + rb + D * ra];
                r.m[k] = -0.5 * s * (ra == rb ? bab : bab + bba);
            }
            r.w = (double)wx[i] * ws;
        }
        xr[i] = r;
    }
}

// d^T M d for a packed (-1/2, off-diagonals doubled) matrix, Horner form
template <int D>
__device__ __forceinline__ double quad64(const double* m, double d0, double d1, double d2)
{
    if (D == 3) {
        const double g0 = fma(m[4], d2, fma(m[3], d1, m[0] * d0));
        const double g1 = fma(m[5], d2, m[1] * d1);
        const double g2 = m[2] * d2;
        return fma(d0, g0, fma(d1, g1, d2 * g2));
    } else {
        const double g0 = fma(m[2], d1, m[0] * d0);
        const double g1 = m[1] * d1;
        return fma(d0, g0, d1 * g1);
    }
}

template <int D, int IPT_>
struct Ref64Body {
    using StreamRec = Rec64;
    static constexpr int IPT = IPT_;
    static constexpr int NV = 1;
    static constexpr int NS = Sym<D>::N;
    double x[IPT][3], b[IPT][NS], w[IPT], e[IPT];

    __device__ void setup(const PairArgs&) {}
    __device__ void load_src(const PairArgs& a, int ii, int i)
    {
        if (i < a.i_end) {
            const Rec64& r = static_cast<const Rec64*>(a.xrec)[i];
#pragma unroll
            for (int q = 0; q < D; ++q) x[ii][q] = r.p[q];
#pragma unroll
            for (int q = 0; q < NS; ++q) b[ii][q] = r.m[q];
            w[ii] = r.w;
        } else {
#pragma unroll
            for (int q = 0; q < D; ++q) x[ii][q] = 0.0;
#pragma unroll
            for (int q = 0; q < NS; ++q) b[ii][q] = 0.0;
            w[ii] = 0.0;
        }
    }
    __device__ void zero_all()
    {
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) e[ii] = 0.0;
    }
    __device__ __forceinline__ void consume(const Rec64& r, int)
    {
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            const double d0 = x[ii][0] - r.p[0], d1 = x[ii][1] - r.p[1], d2 = D == 3 ? x[ii][2] - r.p[2] : 0.0;
            const double q1 = quad64<D>(r.m, d0, d1, d2);
            const double q2 = quad64<D>(b[ii], d0, d1, d2);
            e[ii] = fma(r.w, exp(q1) + exp(q2), e[ii]);
        }
    }
    __device__ void fold() {}
    __device__ void finish(const PairArgs&, int, double (&acc)[NV])
    {
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) acc[0] += w[ii] * e[ii];
    }
};

template <class Body, int NT, int TJ>
__global__ void __launch_bounds__(NT) ref64_pair_kernel(PairArgs a)
{
    Body body;
    run_pairs<Body, NT, TJ, 4>(a, body);
}


template <int D>
static int ref64_impl(Context& c, const double* pose_dev, int i0, int i1, double* out_dev, cudaStream_t s)
{
    DUGMA_RET(c.ensure_coef_records());   // the 128-byte record buffers are shared with the coefficient passes
    Rec64* yr = reinterpret_cast<Rec64*>(c.yrec128);
    Rec64* xr = reinterpret_cast<Rec64*>(c.xrec128);
    const int n = std::max(c.M_pad, c.N_pad);
    ref64_prologue_kernel<D><<<std::min((n + 255) / 256, c.num_sms * 4), 256, 0, s>>>(
        pose_dev, c.y, c.yinv, c.wy, c.M, c.M_pad, yr, c.x, c.xinv, c.wx, c.N, c.N_pad, xr);
    DUGMA_CK(cudaGetLastError());
    const KernelShape sh{2, 128, 32};
    return launch_pair_variant(c, ref64_pair_kernel<Ref64Body<D, 2>, 128, 32>, sh, xr, yr, (size_t)c.M_pad, 1, 0.0,
                               pose_dev, i0, i1, out_dev, nullptr, nullptr, 0, nullptr, s);
}

int ref64_launch(Context& c, const double* pose_dev, int i0, int i1, double* out_dev, cudaStream_t s)
{
    return c.D == 3 ? ref64_impl<3>(c, pose_dev, i0, i1, out_dev, s) : ref64_impl<2>(c, pose_dev, i0, i1, out_dev, s);
}

}  // namespace dugma

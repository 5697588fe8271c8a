// conv.cu -- CONV model: every pair is a Gaussian with its own combined covariance,
//   E_c = sum_ij N(d_ij; 0, S_ij),  S_ij = sig (R Sigma_y_j R^T + Sigma_x_i),  d = x_i - R y_j - t.
//
// Covariances are stored divided by a per-context scale c (mean trace / D) so that the
// FP32 determinants stay far from under/overflow: S = lam * St with lam = sig * c and
// St = St_y' + St_x.  Per pair, with adj/det the adjugate and determinant of St:
//   h = adj d,  m~ = d.h / det,  N~ = det^-1/2 exp(-m~ / (2 lam)),
// and N = (2 pi lam)^(-D/2) N~.  The 3x3 inverse runs in FP64 whenever
// det < 1e-6 * (product of the diagonal), i.e. when the combined covariance is close
// to singular (condition number around 1e6 or more).
//
// Adjoint.  f = log N is invariant under rotating d and S together, so the derivative
// for rotating (R y, St_y') equals minus the derivative for rotating (x - t, St_x):
//   df/dw = p x u - (Sx u) x u + axial(Sx S^-1),   df/dt = u,   u = S^-1 d,  p = x_i - t,
// with axial(A) = (A12 - A21, A20 - A02, A01 - A10) (2D: A01 - A10).  Both extra terms are
// linear in per-source sums over targets, so the kernel accumulates per source
//   E~ = sum N~,  U = sum N~ u~,  UU = sum N~ u~ u~^T,  A = sum N~ St^-1     (u~ = St^-1 d)
// and contracts them with St_x once per source.  Per pair (3D): 48 FP32 for N~ and its sum
// (with the singularity test), 20 for the moments, 2 SFU (rsqrt, ex2).
// The packed kernels run every pair of a tile through the FP32 fast path without a branch
// and only flag a pair that fails the test; a flagged tile is redone from the per-source
// sums saved at its start with the exact per-pair rules, so the common case is straight-line.
#include <cmath>

#include "context.hpp"
#include "pairs.cuh"

namespace dugma {

// CONV records: y: v0 = (y'hi, 0), v1 = (y'lo, 0), v2/v3 = R St_y R^T packed (00,11,22,01 | 02,12)
//               x: v0 = (x, 0), v2/v3 = St_x packed
template <int D>
__global__ void conv_prologue_kernel(const double* __restrict__ pose, const float* __restrict__ y,
                                     const float* __restrict__ ycov, int M, int M_pad, YRec* __restrict__ yrec,
                                     const float* __restrict__ x, const float* __restrict__ xcov, int N, int N_pad,
                                     XRec* __restrict__ xrec)
{
    constexpr int NS = Sym<D>::N;
    double R[9], t[3];
    for (int k = 0; k < D * D; ++k) R[k] = pose[k];
    for (int a = 0; a < D; ++a) t[a] = pose[kPoseT + a];
    const int stride = gridDim.x * blockDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < M_pad; j += stride) {
        float hi[3] = {0, 0, 0}, lo[3] = {0, 0, 0}, sp[6] = {0, 0, 0, 0, 0, 0};
        float valid = 0.f;
        if (j < M) {
            valid = 1.f;
            for (int a = 0; a < D; ++a) {
                double v = R[a] * (double)y[(size_t)j * D] + R[a + D] * (double)y[(size_t)j * D + 1];
                if (D == 3) v = v + R[a + 6] * (double)y[(size_t)j * D + 2];
                v = v + t[a];
                hi[a] = __double2float_rn(v);
                lo[a] = __double2float_rn(v - (double)hi[a]);
            }
            double A[3][3], T[3][3];
            for (int k = 0; k < NS; ++k) {
                const int ra = Sym<D>::a(k), rb = Sym<D>::b(k);
                A[ra][rb] = A[rb][ra] = (double)ycov[(size_t)j * NS + k];
            }
            for (int r0 = 0; r0 < D; ++r0)
                for (int c0 = 0; c0 < D; ++c0) {
                    double acc = 0;
                    for (int k = 0; k < D; ++k) acc += A[r0][k] * R[c0 + D * k];
                    T[r0][c0] = acc;
                }
            for (int k = 0; k < NS; ++k) {
                double acc = 0;
                for (int q = 0; q < D; ++q) acc += R[Sym<D>::a(k) + D * q] * T[q][Sym<D>::b(k)];
                sp[k] = __double2float_rn(acc);
            }
        }
        YRec r;
        r.v0 = make_float4(hi[0], hi[1], hi[2], valid);
        r.v1 = make_float4(lo[0], lo[1], lo[2], 0.f);
        r.v2 = D == 3 ? make_float4(sp[0], sp[1], sp[2], sp[3]) : make_float4(sp[0], sp[1], sp[2], 0.f);
        r.v3 = D == 3 ? make_float4(sp[4], sp[5], 0.f, 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
        yrec[j] = r;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N_pad; i += stride) {
        float xv[3] = {0, 0, 0}, sp[6] = {0, 0, 0, 0, 0, 0};
        if (i < N) {
            for (int a = 0; a < D; ++a) xv[a] = x[(size_t)i * D + a];
            for (int k = 0; k < NS; ++k) sp[k] = xcov[(size_t)i * NS + k];
        }
        XRec r;
        r.v0 = make_float4(xv[0], xv[1], xv[2], 0.f);
        r.v1 = make_float4(0.f, 0.f, 0.f, 0.f);
        r.v2 = D == 3 ? make_float4(sp[0], sp[1], sp[2], sp[3]) : make_float4(sp[0], sp[1], sp[2], 0.f);
        r.v3 = D == 3 ? make_float4(sp[4], sp[5], 0.f, 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
        xrec[i] = r;
    }
}

// A near-singular pair recomputed entirely in FP64 from the stored FP32 inputs: the target
// covariance is rotated again from Sigma_y_j (packed, / c) with R in FP64, added to the
// source covariance, and the difference d is formed from x and the y' split exactly.
// Returns false (no contribution) when the combined covariance is not positive definite.
template <int D>
__device__ __forceinline__ bool conv_pair_f64(const float* xi, const float* sxi, float4 v0, float4 v1,
                                           const float* __restrict__ cy, const double* __restrict__ pose, double kl,
                                           float* adj, float* h, float* rd, float* Nt)
{
    constexpr int NS = Sym<D>::N;
    double A[3][3], T[3][3], S[6];
    for (int k = 0; k < NS; ++k) {
        const int ra = Sym<D>::a(k), rb = Sym<D>::b(k);
        A[ra][rb] = A[rb][ra] = (double)cy[k];
    }
    for (int r0 = 0; r0 < D; ++r0)
        for (int c0 = 0; c0 < D; ++c0) {
            double acc = 0;
            for (int k = 0; k < D; ++k) acc += A[r0][k] * pose[c0 + D * k];
            T[r0][c0] = acc;
        }
    for (int k = 0; k < NS; ++k) {
        double acc = 0;
        for (int q = 0; q < D; ++q) acc += pose[Sym<D>::a(k) + D * q] * T[q][Sym<D>::b(k)];
        S[k] = acc + (double)sxi[k];
    }
    const double yh[3] = {v0.x, v0.y, v0.z}, yl[3] = {v1.x, v1.y, v1.z};
    double d[3], ad[6], det;
    for (int q = 0; q < D; ++q) d[q] = ((double)xi[q] - yh[q]) - yl[q];
    if (D == 3) {
        const double a = S[0], b = S[1], c = S[2], e4 = S[3], f5 = S[4], g6 = S[5];
        ad[0] = b * c - g6 * g6;
        ad[1] = a * c - f5 * f5;
        ad[2] = a * b - e4 * e4;
        ad[3] = f5 * g6 - e4 * c;
        ad[4] = e4 * g6 - b * f5;
        ad[5] = e4 * f5 - a * g6;
        det = a * ad[0] + e4 * ad[3] + f5 * ad[4];
    } else {
        ad[0] = S[1];
        ad[1] = S[0];
        ad[2] = -S[2];
        det = S[0] * S[1] - S[2] * S[2];
    }
    if (!(det > 0)) return false;
    double hh[3], m = 0;
    if (D == 3) {
        hh[0] = ad[0] * d[0] + ad[3] * d[1] + ad[4] * d[2];
        hh[1] = ad[3] * d[0] + ad[1] * d[1] + ad[5] * d[2];
        hh[2] = ad[4] * d[0] + ad[5] * d[1] + ad[2] * d[2];
    } else {
        hh[0] = ad[0] * d[0] + ad[2] * d[1];
        hh[1] = ad[2] * d[0] + ad[1] * d[1];
    }
    for (int q = 0; q < D; ++q) m += d[q] * hh[q];
    const double r = 1.0 / det;
    *Nt = (float)(sqrt(r) * exp2(m * r * kl));
    *rd = (float)r;
    for (int q = 0; q < D; ++q) h[q] = (float)hh[q];
    for (int k = 0; k < NS; ++k) adj[k] = (float)ad[k];
    return true;
}

// Per-source contraction of the CONV moments into the energy and the pose gradient (and
// dE/dx when requested): E~ = sum N~, U = sum N~ u~, UU = sum N~ u~ u~^T, A = sum N~ St^-1
// over the item's targets, with the source's own x and St_x.
template <int D, int NV, bool GRAD>
__device__ void conv_contract(const PairArgs& a, int jc, int row, const float* xv, const float* sxv, double E,
                              const double* Ur, const double* UUr, const double* Ar, double lam, double c0,
                              const double* t, double (&acc)[NV])
{
    constexpr int NS = Sym<D>::N, NR = Sym<D>::NR;
    acc[0] += c0 * E;
    if (!GRAD) return;
    double S[3][3] = {}, UUm[3][3] = {}, Am[3][3] = {};
#pragma unroll
    for (int q = 0; q < NS; ++q) {
        const int ra = Sym<D>::a(q), rb = Sym<D>::b(q);
        S[ra][rb] = S[rb][ra] = (double)sxv[q];
        UUm[ra][rb] = UUm[rb][ra] = UUr[q];
        Am[ra][rb] = Am[rb][ra] = Ar[q];
    }
    double u[3], p[3];
#pragma unroll
    for (int q = 0; q < D; ++q) {
        u[q] = Ur[q] / lam;        // sum N~ S^-1 d
        p[q] = (double)xv[q] - t[q];
    }
    // B1 = S_x UU (for (S_x u) x u),  B2 = S_x A (for axial(S_x S^-1))
    double B1[3][3] = {}, B2[3][3] = {};
    for (int r0 = 0; r0 < D; ++r0)
        for (int c1 = 0; c1 < D; ++c1)
            for (int k = 0; k < D; ++k) {
                B1[r0][c1] += S[r0][k] * UUm[k][c1];
                B2[r0][c1] += S[r0][k] * Am[k][c1];
            }
    // (S_x u~) x u~ summed: component k = eps_kab (S_x UU)_ab ; / lam for the S scale
    if (D == 3) {
        const double q0 = (B1[1][2] - B1[2][1]) / lam, q1 = (B1[2][0] - B1[0][2]) / lam,
                     q2 = (B1[0][1] - B1[1][0]) / lam;
        const double x0 = B2[1][2] - B2[2][1], x1 = B2[2][0] - B2[0][2], x2 = B2[0][1] - B2[1][0];
        acc[1] += c0 * (p[1] * u[2] - p[2] * u[1] - q0 + x0);
        acc[2] += c0 * (p[2] * u[0] - p[0] * u[2] - q1 + x1);
        acc[3] += c0 * (p[0] * u[1] - p[1] * u[0] - q2 + x2);
    } else {
        const double q0 = (B1[0][1] - B1[1][0]) / lam;
        const double x0 = B2[0][1] - B2[1][0];
        acc[1] += c0 * (p[0] * u[1] - p[1] * u[0] - q0 + x0);
    }
#pragma unroll
    for (int q = 0; q < D; ++q) acc[1 + NR + q] += c0 * u[q];
    if (a.dx_part) {
        const int rows = a.i_end - a.i0;
        for (int q = 0; q < D; ++q) a.dx_part[((size_t)jc * rows + (row - a.i0)) * D + q] = -c0 * u[q];
    }
}

template <int D, int IPT_, bool GRAD>
struct ConvBody {
    using StreamRec = YRec;
    static constexpr int IPT = IPT_;
    static constexpr int NS = Sym<D>::N, NR = Sym<D>::NR;
    static constexpr int NV = GRAD ? 1 + NR + D : 1;
    float x[IPT][D], sx[IPT][NS];
    float e[IPT], U[IPT][GRAD ? D : 1], UU[IPT][GRAD ? NS : 1], A[IPT][GRAD ? NS : 1];
    double E64[IPT], Ur[IPT][GRAD ? D : 1], UUr[IPT][GRAD ? NS : 1], Ar[IPT][GRAD ? NS : 1];
    int row[IPT];
    float kl;          // -1/2 log2(e) / lam
    double c0, lam, t[3];
    const float* ycov;
    const double* pose;

    __device__ void setup(const PairArgs& a)
    {
        lam = a.pose[kPoseSig] * a.Lmax;   // Lmax carries the covariance scale c for this body
        kl = (float)(K_EXP2 / lam);
        ycov = a.ycov;
        pose = a.pose;
        c0 = pow(2.0 * 3.14159265358979323846 * lam, -0.5 * D);
        for (int q = 0; q < D; ++q) t[q] = a.pose[kPoseT + q];
    }
    __device__ void load_src(const PairArgs& a, int ii, int i)
    {
        row[ii] = i < a.i_end ? i : -1;
        const XRec r = static_cast<const XRec*>(a.xrec)[i < a.i_end ? i : 0];
        const bool ok = i < a.i_end;
        const float xv[3] = {r.v0.x, r.v0.y, r.v0.z};
        const float sv[6] = {r.v2.x, r.v2.y, r.v2.z, r.v2.w, r.v3.x, r.v3.y};
#pragma unroll
        for (int q = 0; q < D; ++q) x[ii][q] = ok ? xv[q] : 0.f;
#pragma unroll
        for (int q = 0; q < NS; ++q) sx[ii][q] = ok ? sv[q] : (Sym<D>::a(q) == Sym<D>::b(q) ? 1.f : 0.f);
    }
    __device__ void zero_tile()
    {
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            e[ii] = 0.f;
            if (GRAD) {
#pragma unroll
                for (int q = 0; q < D; ++q) U[ii][q] = 0.f;
#pragma unroll
                for (int q = 0; q < NS; ++q) { UU[ii][q] = 0.f; A[ii][q] = 0.f; }
            }
        }
    }
    __device__ void zero_all()
    {
        zero_tile();
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            E64[ii] = 0.0;
            if (GRAD) {
#pragma unroll
                for (int q = 0; q < D; ++q) Ur[ii][q] = 0.0;
#pragma unroll
                for (int q = 0; q < NS; ++q) { UUr[ii][q] = 0.0; Ar[ii][q] = 0.0; }
            }
        }
    }
    __device__ __forceinline__ void consume(const YRec& r, int j)
    {
        const float4 v0 = r.v0, v1 = r.v1, v2 = r.v2, v3 = r.v3;
        if (v0.w == 0.f) return;   // padding target (uniform across the block)
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            float d[3], s[6], adj[6], det, h[3], rd, Nt;
            d[0] = (x[ii][0] - v0.x) - v1.x;
            d[1] = (x[ii][1] - v0.y) - v1.y;
            if (D == 3) d[2] = (x[ii][2] - v0.z) - v1.z;
            bool near_singular;
            if (D == 3) {
                s[0] = sx[ii][0] + v2.x; s[1] = sx[ii][1] + v2.y; s[2] = sx[ii][2] + v2.z;
                s[3] = sx[ii][3] + v2.w; s[4] = sx[ii][4] + v3.x; s[5] = sx[ii][5] + v3.y;
                adj[0] = fmaf(s[1], s[2], -s[5] * s[5]);
                adj[1] = fmaf(s[0], s[2], -s[4] * s[4]);
                adj[2] = fmaf(s[0], s[1], -s[3] * s[3]);
                adj[3] = fmaf(s[4], s[5], -s[3] * s[2]);
                adj[4] = fmaf(s[3], s[5], -s[1] * s[4]);
                adj[5] = fmaf(s[3], s[4], -s[0] * s[5]);
                det = fmaf(s[4], adj[4], fmaf(s[3], adj[3], s[0] * adj[0]));
                near_singular = det < 1e-6f * (s[0] * s[1] * s[2]);
                h[0] = fmaf(adj[4], d[2], fmaf(adj[3], d[1], adj[0] * d[0]));
                h[1] = fmaf(adj[5], d[2], fmaf(adj[1], d[1], adj[3] * d[0]));
                h[2] = fmaf(adj[2], d[2], fmaf(adj[5], d[1], adj[4] * d[0]));
            } else {
                s[0] = sx[ii][0] + v2.x; s[1] = sx[ii][1] + v2.y; s[2] = sx[ii][2] + v2.z;
                adj[0] = s[1];
                adj[1] = s[0];
                adj[2] = -s[2];
                det = fmaf(s[0], s[1], -s[2] * s[2]);
                near_singular = det < 1e-6f * (s[0] * s[1]);
                h[0] = fmaf(adj[2], d[1], adj[0] * d[0]);
                h[1] = fmaf(adj[1], d[1], adj[2] * d[0]);
            }
            if (near_singular) {
                // condition around 1e6 or worse: the whole pair in FP64
                if (!conv_pair_f64<D>(x[ii], sx[ii], v0, v1, ycov + (size_t)j * NS, pose, (double)kl, adj, h, &rd,
                                      &Nt))
                    continue;
            } else {
                if (!(det > 0.f)) continue;   // not positive definite: no contribution (as the oracle)
                float m = d[0] * h[0];
#pragma unroll
                for (int q = 1; q < D; ++q) m = fmaf(d[q], h[q], m);
                const float rs = rsqrtf(det);
                rd = rs * rs;
                Nt = rs * ex2(m * (rd * kl));
            }
            e[ii] += Nt;
            if (GRAD) {
                const float nr = Nt * rd, nr2 = nr * rd;
                float w[3];
#pragma unroll
                for (int q = 0; q < D; ++q) {
                    U[ii][q] = fmaf(nr, h[q], U[ii][q]);
                    w[q] = nr2 * h[q];
                }
#pragma unroll
                for (int q = 0; q < NS; ++q) {
                    UU[ii][q] = fmaf(w[Sym<D>::a(q)], h[Sym<D>::b(q)], UU[ii][q]);
                    A[ii][q] = fmaf(nr, adj[q], A[ii][q]);
                }
            }
        }
    }
    __device__ void fold()
    {
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            E64[ii] += (double)e[ii];
            if (GRAD) {
#pragma unroll
                for (int q = 0; q < D; ++q) Ur[ii][q] += (double)U[ii][q];
#pragma unroll
                for (int q = 0; q < NS; ++q) { UUr[ii][q] += (double)UU[ii][q]; Ar[ii][q] += (double)A[ii][q]; }
            }
        }
        zero_tile();
    }
    __device__ void finish(const PairArgs& a, int jc, double (&acc)[NV])
    {
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            if (row[ii] < 0) continue;
            conv_contract<D, NV, GRAD>(a, jc, row[ii], x[ii], sx[ii], E64[ii], Ur[ii], UUr[ii], Ar[ii], lam, c0, t,
                                       acc);
        }
    }
};

// ---------------------------------------------------------------------------
// Packed CONV: two targets per f32x2 operation (YRec2 pair records).
//   f0..f2 -y'hi, f3 lv (0, or -inf for padding), f4..f6 -y'lo, f7 + k  R St_y R^T packed
//   entry k (Sym order), then the negated off-diagonal entries (3D: f13..f15, 2D: f10), so
//   that every adjugate entry is one multiply and one fused multiply-add without negation.
// Padding targets: y' = 0, St_y = I, lv = -inf (finite arithmetic, zero contribution).
// ---------------------------------------------------------------------------
template <int D>
__global__ void conv_prologue2_kernel(const double* __restrict__ pose, const float* __restrict__ y,
                                      const float* __restrict__ ycov, int M, int M_pad, YRec2* __restrict__ yrec)
{
    constexpr int NS = Sym<D>::N;
    double R[9], t[3];
    for (int k = 0; k < D * D; ++k) R[k] = pose[k];
    for (int a = 0; a < D; ++a) t[a] = pose[kPoseT + a];
    const int stride = gridDim.x * blockDim.x;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < M_pad / 2; p += stride) {
        float f[2][16];
        for (int h = 0; h < 2; ++h) {
            const int j = 2 * p + h;
            for (int q = 0; q < 16; ++q) f[h][q] = 0.f;
            float hi[3] = {0, 0, 0}, lo[3] = {0, 0, 0}, sp[6] = {0, 0, 0, 0, 0, 0};
            for (int k = 0; k < D; ++k) sp[k] = 1.f;
            float lv = -INFINITY;
            if (j < M) {
                lv = 0.f;
                for (int a = 0; a < D; ++a) {
                    double v = R[a] * (double)y[(size_t)j * D] + R[a + D] * (double)y[(size_t)j * D + 1];
                    if (D == 3) v = v + R[a + 6] * (double)y[(size_t)j * D + 2];
                    v = v + t[a];
                    hi[a] = __double2float_rn(v);
                    lo[a] = __double2float_rn(v - (double)hi[a]);
                }
                double A[3][3], T[3][3];
                for (int k = 0; k < NS; ++k) {
                    const int ra = Sym<D>::a(k), rb = Sym<D>::b(k);
                    A[ra][rb] = A[rb][ra] = (double)ycov[(size_t)j * NS + k];
                }
                for (int r0 = 0; r0 < D; ++r0)
                    for (int c0 = 0; c0 < D; ++c0) {
                        double acc = 0;
                        for (int k = 0; k < D; ++k) acc += A[r0][k] * R[c0 + D * k];
                        T[r0][c0] = acc;
                    }
                for (int k = 0; k < NS; ++k) {
                    double acc = 0;
                    for (int q = 0; q < D; ++q) acc += R[Sym<D>::a(k) + D * q] * T[q][Sym<D>::b(k)];
                    sp[k] = __double2float_rn(acc);
                }
            }
            for (int a = 0; a < D; ++a) {
                f[h][a] = -hi[a];
                f[h][4 + a] = -lo[a];
            }
            f[h][3] = lv;
            for (int k = 0; k < NS; ++k) f[h][7 + k] = sp[k];
            for (int k = D; k < NS; ++k) f[h][7 + NS + (k - D)] = -sp[k];
        }
        YRec2 r;
        for (int q = 0; q < 8; ++q) r.q[q] = make_float4(f[0][2 * q], f[1][2 * q], f[0][2 * q + 1], f[1][2 * q + 1]);
        yrec[p] = r;
    }
}

__device__ __forceinline__ float2 fld2(const YRec2& r, int f)
{
    const float4 q = r.q[f >> 1];
    return (f & 1) ? make_float2(q.z, q.w) : make_float2(q.x, q.y);
}

template <int D, int IPT_, bool GRAD, int NT>
struct PackedConvBody {
    using StreamRec = YRec2;
    static constexpr int IPT = IPT_;
    static constexpr int NS = Sym<D>::N, NR = Sym<D>::NR, NO = NS - D;
    static constexpr int NV = GRAD ? 1 + NR + D : 1;
    float2 X[IPT][D], SX[IPT][NS], OX[IPT][NO];  // duplicated in both halves; OX = -off-diagonals
    float2 e[IPT];                               // energy, tile level
    float2 U[IPT][GRAD ? D : 1], UU[IPT][GRAD ? NS : 1], A[IPT][GRAD ? NS : 1];   // item level
    double E64[IPT];
    // the largest fast-path term N~ of each source in this item, redone in FP64 at the item's end
    // (a sum carried by a few far pairs has exponents of 40-80, where FP32 holds the exponent to
    // only ~|exponent| x 6e-8): key = float bits of N~ (>= 0, so they order as integers) with the
    // low 10 bits replaced by the pair's place in the item (an item spans at most 512 records)
    uint32_t key[IPT];
    int j0;   // the item's first record
    // set when a pair of the current tile fails the fast path's test; the tile is then redone
    // from the item-level sums saved at its start (a per-thread copy in shared memory)
    bool bad;
    static constexpr int NCK = GRAD ? IPT * (D + 2 * NS) : 1;
    __device__ static float2* checkpoint()
    {
        __shared__ float2 ck[NCK][NT];
        return &ck[0][threadIdx.x];
    }
    int row[IPT];
    float kl;
    double c0, lam, t[3];
    const float* ycov;
    const double* pose;

    __device__ void setup(const PairArgs& a)
    {
        lam = a.pose[kPoseSig] * a.Lmax;   // Lmax carries the covariance scale c for this body
        kl = (float)(K_EXP2 / lam);
        ycov = a.ycov;
        pose = a.pose;
        c0 = pow(2.0 * 3.14159265358979323846 * lam, -0.5 * D);
        for (int q = 0; q < D; ++q) t[q] = a.pose[kPoseT + q];
    }
    __device__ void load_src(const PairArgs& a, int ii, int i)
    {
        row[ii] = i < a.i_end ? i : -1;
        const XRec r = static_cast<const XRec*>(a.xrec)[i < a.i_end ? i : 0];
        const bool ok = i < a.i_end;
        const float xv[3] = {r.v0.x, r.v0.y, r.v0.z};
        const float sv[6] = {r.v2.x, r.v2.y, r.v2.z, r.v2.w, r.v3.x, r.v3.y};
#pragma unroll
        for (int q = 0; q < D; ++q) {
            const float v = ok ? xv[q] : 0.f;
            X[ii][q] = make_float2(v, v);
        }
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            const float v = ok ? sv[q] : (q < D ? 1.f : 0.f);
            SX[ii][q] = make_float2(v, v);
            if (q >= D) OX[ii][q - D] = make_float2(-v, -v);
        }
    }
    __device__ void zero_all()
    {
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            e[ii] = make_float2(0.f, 0.f);
            E64[ii] = 0.0;
            if (GRAD) {
#pragma unroll
                for (int q = 0; q < D; ++q) U[ii][q] = make_float2(0.f, 0.f);
#pragma unroll
                for (int q = 0; q < NS; ++q) { UU[ii][q] = make_float2(0.f, 0.f); A[ii][q] = make_float2(0.f, 0.f); }
            }
        }
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) key[ii] = 0u;
        j0 = 0x7fffffff;
        bad = false;
        save();
    }
    __device__ __forceinline__ void save()
    {
        if (!GRAD) return;
        float2* ck = checkpoint();
        int k = 0;
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
#pragma unroll
            for (int q = 0; q < D; ++q) ck[(k++) * NT] = U[ii][q];
#pragma unroll
            for (int q = 0; q < NS; ++q) ck[(k++) * NT] = UU[ii][q];
#pragma unroll
            for (int q = 0; q < NS; ++q) ck[(k++) * NT] = A[ii][q];
        }
    }
    __device__ __forceinline__ void restore()
    {
        if (!GRAD) return;
        const float2* ck = checkpoint();
        int k = 0;
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
#pragma unroll
            for (int q = 0; q < D; ++q) U[ii][q] = ck[(k++) * NT];
#pragma unroll
            for (int q = 0; q < NS; ++q) UU[ii][q] = ck[(k++) * NT];
#pragma unroll
            for (int q = 0; q < NS; ++q) A[ii][q] = ck[(k++) * NT];
        }
    }
    // One half of a pack the fast path cannot take (near-singular, not positive definite):
    // the scalar rules of ConvBody, FP64 for near-singular pairs.
    __device__ __forceinline__ void rare_half(int ii, const YRec2& r, int j, int h, const float* d, const float* sv,
                                              const float* ad, float det, float& Nt, float& rd, float* hv, float* av)
    {
        Nt = 0.f;
        rd = 0.f;
        for (int q = 0; q < D; ++q) hv[q] = 0.f;
        for (int k = 0; k < NS; ++k) av[k] = 0.f;
        const float lvh = h ? fld2(r, 3).y : fld2(r, 3).x;
        if (lvh == -INFINITY) return;   // padding target
        float prod = sv[0] * sv[1];
        if (D == 3) prod *= sv[2];
        if (det < 1e-6f * prod) {
            float yh[3] = {0, 0, 0}, yl[3] = {0, 0, 0};
            for (int q = 0; q < D; ++q) {
                const float2 a = fld2(r, q), b = fld2(r, 4 + q);
                yh[q] = -(h ? a.y : a.x);
                yl[q] = -(h ? b.y : b.x);
            }
            const float4 v0 = make_float4(yh[0], yh[1], yh[2], 1.f), v1 = make_float4(yl[0], yl[1], yl[2], 0.f);
            float xs[3] = {0, 0, 0}, sxs[6] = {0, 0, 0, 0, 0, 0};
            for (int q = 0; q < D; ++q) xs[q] = X[ii][q].x;
            for (int k = 0; k < NS; ++k) sxs[k] = SX[ii][k].x;
            if (!conv_pair_f64<D>(xs, sxs, v0, v1, ycov + (size_t)j * NS, pose, (double)kl, av, hv, &rd, &Nt)) {
                Nt = 0.f;
                rd = 0.f;
                for (int q = 0; q < D; ++q) hv[q] = 0.f;
                for (int k = 0; k < NS; ++k) av[k] = 0.f;
            }
            return;
        }
        if (!(det > 0.f)) return;   // not positive definite: no contribution
        for (int k = 0; k < NS; ++k) av[k] = ad[k];
        float m = 0.f;
        for (int q = 0; q < D; ++q) {
            float acc = 0.f;
            for (int c = 0; c < D; ++c) {
                const int k = q == c ? q : (D == 2 ? 2 : (q + c == 1 ? 3 : (q + c == 2 ? 4 : 5)));
                acc = fmaf(ad[k], d[c], acc);
            }
            hv[q] = acc;
            m = fmaf(d[q], acc, m);
        }
        const float rs = rsqrtf(det);
        rd = rs * rs;
        Nt = rs * ex2(m * (rd * kl));
    }
    __device__ __forceinline__ void consume(const YRec2& r, int jrec) { pass<false>(r, jrec); }
    // EXACT = false: the fast path for every pair, straight-line, and a flag when any pair fails
    // its test (results of that tile are then discarded and redone); EXACT = true: a pack with a
    // failing half goes through rare_half (FP64 when near-singular)
    template <bool EXACT>
    __device__ __forceinline__ void pass(const YRec2& r, int jrec)
    {
        float2 ny[3], nl[3], cy[6], oy[3];
#pragma unroll
        for (int q = 0; q < D; ++q) { ny[q] = fld2(r, q); nl[q] = fld2(r, 4 + q); }
        const float2 lv = fld2(r, 3);
#pragma unroll
        for (int k = 0; k < NS; ++k) cy[k] = fld2(r, 7 + k);
#pragma unroll
        for (int k = 0; k < NO; ++k) oy[k] = fld2(r, 7 + NS + k);
        const float2 KL = make_float2(kl, kl), EPS = make_float2(1e6f, 1e6f);
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            float2 d[3], sm[6], o[3], adj[6], det, h[3], rd, Nt;
#pragma unroll
            for (int q = 0; q < D; ++q) d[q] = fadd2(fadd2(X[ii][q], ny[q]), nl[q]);
#pragma unroll
            for (int k = 0; k < NS; ++k) sm[k] = fadd2(SX[ii][k], cy[k]);
#pragma unroll
            for (int k = 0; k < NO; ++k) o[k] = fadd2(OX[ii][k], oy[k]);
            float2 prod;
            if (D == 3) {
                adj[0] = ffma2(o[2], sm[5], fmul2(sm[1], sm[2]));
                adj[1] = ffma2(o[1], sm[4], fmul2(sm[0], sm[2]));
                adj[2] = ffma2(o[0], sm[3], fmul2(sm[0], sm[1]));
                adj[3] = ffma2(sm[4], sm[5], fmul2(o[0], sm[2]));
                adj[4] = ffma2(sm[3], sm[5], fmul2(o[1], sm[1]));
                adj[5] = ffma2(sm[3], sm[4], fmul2(o[2], sm[0]));
                det = ffma2(sm[4], adj[4], ffma2(sm[3], adj[3], fmul2(sm[0], adj[0])));
                prod = fmul2(fmul2(sm[0], sm[1]), sm[2]);
            } else {
                adj[0] = sm[1];
                adj[1] = sm[0];
                adj[2] = o[0];
                det = ffma2(o[0], sm[2], fmul2(sm[0], sm[1]));
                prod = fmul2(sm[0], sm[1]);
            }
            // fast path: both halves positive definite and well conditioned (NaN fails too)
            const float2 dd = fmul2(det, EPS);
            const bool fast = (dd.x >= prod.x) & (dd.y >= prod.y) & (det.x > 0.f) & (det.y > 0.f);
            if (!EXACT) bad |= !fast;
            if (!EXACT || fast) {
                if (D == 3) {
                    h[0] = ffma2(adj[4], d[2], ffma2(adj[3], d[1], fmul2(adj[0], d[0])));
                    h[1] = ffma2(adj[5], d[2], ffma2(adj[1], d[1], fmul2(adj[3], d[0])));
                    h[2] = ffma2(adj[2], d[2], ffma2(adj[5], d[1], fmul2(adj[4], d[0])));
                } else {
                    h[0] = ffma2(adj[2], d[1], fmul2(adj[0], d[0]));
                    h[1] = ffma2(adj[1], d[1], fmul2(adj[2], d[0]));
                }
                float2 m = fmul2(d[0], h[0]);
#pragma unroll
                for (int q = 1; q < D; ++q) m = ffma2(d[q], h[q], m);
                const float2 rs = make_float2(rsqrtf(det.x), rsqrtf(det.y));
                rd = fmul2(rs, rs);
                const float2 arg = ffma2(m, fmul2(rd, KL), lv);
                Nt = fmul2(rs, make_float2(ex2(arg.x), ex2(arg.y)));
                if (!EXACT) {   // (a redone tile's fast pairs have these same values)
                    const uint32_t jl = 2u * ((uint32_t)jrec & 511u);
                    key[ii] = max(key[ii], (__float_as_uint(fmaxf(Nt.x, 0.f)) & 0xfffffc00u) | jl);
                    key[ii] = max(key[ii], (__float_as_uint(fmaxf(Nt.y, 0.f)) & 0xfffffc00u) | (jl | 1u));
                }
            } else {
                float dv[2][3], sv[2][6], av[2][6], hv[2][3], nt[2], rdv[2];
                for (int hh = 0; hh < 2; ++hh) {
                    for (int q = 0; q < D; ++q) dv[hh][q] = hh ? d[q].y : d[q].x;
                    for (int k = 0; k < NS; ++k) {
                        sv[hh][k] = hh ? sm[k].y : sm[k].x;
                        av[hh][k] = hh ? adj[k].y : adj[k].x;
                    }
                }
                float ao[2][6];
                rare_half(ii, r, 2 * jrec, 0, dv[0], sv[0], av[0], det.x, nt[0], rdv[0], hv[0], ao[0]);
                rare_half(ii, r, 2 * jrec + 1, 1, dv[1], sv[1], av[1], det.y, nt[1], rdv[1], hv[1], ao[1]);
                Nt = make_float2(nt[0], nt[1]);
                rd = make_float2(rdv[0], rdv[1]);
                for (int q = 0; q < D; ++q) h[q] = make_float2(hv[0][q], hv[1][q]);
                for (int k = 0; k < NS; ++k) adj[k] = make_float2(ao[0][k], ao[1][k]);
            }
            e[ii] = fadd2(e[ii], Nt);
            if (GRAD) {
                const float2 nr = fmul2(Nt, rd), nr2 = fmul2(nr, rd);
                float2 w[3];
#pragma unroll
                for (int q = 0; q < D; ++q) {
                    U[ii][q] = ffma2(nr, h[q], U[ii][q]);
                    w[q] = fmul2(nr2, h[q]);
                }
#pragma unroll
                for (int k = 0; k < NS; ++k) {
                    UU[ii][k] = ffma2(w[Sym<D>::a(k)], h[Sym<D>::b(k)], UU[ii][k]);
                    A[ii][k] = ffma2(nr, adj[k], A[ii][k]);
                }
            }
        }
    }
    __device__ void fold_tile(const YRec2* tile, int jbase, int ntile)
    {
        j0 = min(j0, jbase);
        if (bad) {   // rare: redo this tile with the exact per-pair rules
            restore();
#pragma unroll
            for (int ii = 0; ii < IPT; ++ii) e[ii] = make_float2(0.f, 0.f);
            for (int jj = 0; jj < ntile; ++jj) pass<true>(tile[jj], jbase + jj);
            bad = false;
        }
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            E64[ii] += (double)e[ii].x + (double)e[ii].y;
            e[ii] = make_float2(0.f, 0.f);
        }
        save();
    }
    // Source ii's largest term of this item: its fast-path contribution re-evaluated in FP32 by the
    // same operations, one half at a time (f32x2 arithmetic rounds each half as the scalar
    // operation does, so the values are the ones accumulated), replaced by the exact FP64 pair.
    __device__ void top_pair_in_fp64(const PairArgs& a, int ii, const float* xs, const float* sxs, double* ur,
                                     double* uur, double* ar)
    {
        const int loc = (int)(key[ii] & 1023u), h = loc & 1;
        const int jrec = j0 + (((loc >> 1) - (j0 & 511)) & 511);
        const int j = 2 * jrec + h;
        const YRec2& r = static_cast<const YRec2*>(a.yrec)[j >> 1];
        float ny[3] = {0, 0, 0}, nl[3] = {0, 0, 0}, cy[6] = {0, 0, 0, 0, 0, 0}, oy[3] = {0, 0, 0};
#pragma unroll
        for (int q = 0; q < D; ++q) {
            const float2 u0 = fld2(r, q), u1 = fld2(r, 4 + q);
            ny[q] = h ? u0.y : u0.x;
            nl[q] = h ? u1.y : u1.x;
        }
        const float2 l2 = fld2(r, 3);
        const float lv = h ? l2.y : l2.x;
#pragma unroll
        for (int k = 0; k < NS; ++k) {
            const float2 u = fld2(r, 7 + k);
            cy[k] = h ? u.y : u.x;
        }
#pragma unroll
        for (int k = 0; k < NO; ++k) {
            const float2 u = fld2(r, 7 + NS + k);
            oy[k] = h ? u.y : u.x;
        }
        float d[3], sm[6], o[3], adj[6], hv[3], det;
#pragma unroll
        for (int q = 0; q < D; ++q) d[q] = __fadd_rn(__fadd_rn(xs[q], ny[q]), nl[q]);
#pragma unroll
        for (int k = 0; k < NS; ++k) sm[k] = __fadd_rn(sxs[k], cy[k]);
#pragma unroll
        for (int k = 0; k < NO; ++k) o[k] = __fadd_rn(-sxs[D + k], oy[k]);
        if (D == 3) {
            adj[0] = __fmaf_rn(o[2], sm[5], __fmul_rn(sm[1], sm[2]));
            adj[1] = __fmaf_rn(o[1], sm[4], __fmul_rn(sm[0], sm[2]));
            adj[2] = __fmaf_rn(o[0], sm[3], __fmul_rn(sm[0], sm[1]));
            adj[3] = __fmaf_rn(sm[4], sm[5], __fmul_rn(o[0], sm[2]));
            adj[4] = __fmaf_rn(sm[3], sm[5], __fmul_rn(o[1], sm[1]));
            adj[5] = __fmaf_rn(sm[3], sm[4], __fmul_rn(o[2], sm[0]));
            det = __fmaf_rn(sm[4], adj[4], __fmaf_rn(sm[3], adj[3], __fmul_rn(sm[0], adj[0])));
            hv[0] = __fmaf_rn(adj[4], d[2], __fmaf_rn(adj[3], d[1], __fmul_rn(adj[0], d[0])));
            hv[1] = __fmaf_rn(adj[5], d[2], __fmaf_rn(adj[1], d[1], __fmul_rn(adj[3], d[0])));
            hv[2] = __fmaf_rn(adj[2], d[2], __fmaf_rn(adj[5], d[1], __fmul_rn(adj[4], d[0])));
        } else {
            adj[0] = sm[1];
            adj[1] = sm[0];
            adj[2] = o[0];
            det = __fmaf_rn(o[0], sm[2], __fmul_rn(sm[0], sm[1]));
            hv[0] = __fmaf_rn(adj[2], d[1], __fmul_rn(adj[0], d[0]));
            hv[1] = __fmaf_rn(adj[1], d[1], __fmul_rn(adj[2], d[0]));
        }
        float m = __fmul_rn(d[0], hv[0]);
#pragma unroll
        for (int q = 1; q < D; ++q) m = __fmaf_rn(d[q], hv[q], m);
        float prod = __fmul_rn(sm[0], sm[1]);
        if (D == 3) prod = __fmul_rn(prod, sm[2]);
        if (!(__fmul_rn(det, 1e6f) >= prod) || !(det > 0.f)) return;   // that pair took the exact path
        const float rs = rsqrtf(det), rd = __fmul_rn(rs, rs);
        const float Nt = __fmul_rn(rs, ex2(__fmaf_rn(m, __fmul_rn(rd, kl), lv)));
        // the exact pair (FP64 throughout, from the stored inputs)
        const float4 v0 = make_float4(-ny[0], -ny[1], D == 3 ? -ny[2] : 0.f, 1.f);
        const float4 v1 = make_float4(-nl[0], -nl[1], D == 3 ? -nl[2] : 0.f, 0.f);
        float adj64[6] = {0, 0, 0, 0, 0, 0}, h64[3] = {0, 0, 0}, rd64 = 0.f, Nt64 = 0.f;
        if (!conv_pair_f64<D>(xs, sxs, v0, v1, ycov + (size_t)j * NS, pose, (double)kl, adj64, h64, &rd64, &Nt64))
            Nt64 = rd64 = 0.f;
        E64[ii] += (double)Nt64 - (double)Nt;
        if (!GRAD) return;
        const float nr = __fmul_rn(Nt, rd), nr2 = __fmul_rn(nr, rd);
        const double nx = (double)Nt64 * rd64, nx2 = nx * rd64;
        float w[3];
#pragma unroll
        for (int q = 0; q < D; ++q) {
            w[q] = __fmul_rn(nr2, hv[q]);
            ur[q] += nx * h64[q] - (double)nr * hv[q];
        }
#pragma unroll
        for (int k = 0; k < NS; ++k) {
            const int ka = Sym<D>::a(k), kb = Sym<D>::b(k);
            uur[k] += nx2 * h64[ka] * h64[kb] - (double)w[ka] * hv[kb];
            ar[k] += nx * adj64[k] - (double)nr * adj[k];
        }
    }
    __device__ void finish(const PairArgs& a, int jc, double (&acc)[NV])
    {
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            if (row[ii] < 0) continue;
            double ur[3] = {0, 0, 0}, uur[6] = {0, 0, 0, 0, 0, 0}, ar[6] = {0, 0, 0, 0, 0, 0};
            if (GRAD) {
#pragma unroll
                for (int q = 0; q < D; ++q) ur[q] = (double)U[ii][q].x + (double)U[ii][q].y;
#pragma unroll
                for (int k = 0; k < NS; ++k) {
                    uur[k] = (double)UU[ii][k].x + (double)UU[ii][k].y;
                    ar[k] = (double)A[ii][k].x + (double)A[ii][k].y;
                }
            }
            float xs[3] = {0, 0, 0}, sxs[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
            for (int q = 0; q < D; ++q) xs[q] = X[ii][q].x;
#pragma unroll
            for (int k = 0; k < NS; ++k) sxs[k] = SX[ii][k].x;
            if (key[ii] & 0xfffffc00u) top_pair_in_fp64(a, ii, xs, sxs, ur, uur, ar);
            conv_contract<D, NV, GRAD>(a, jc, row[ii], xs, sxs, E64[ii], ur, uur, ar, lam, c0, t, acc);
        }
    }
};

template <class Body, int NT, int TJ, int MINB = 1>
__global__ void __launch_bounds__(NT, MINB) conv_kernel(PairArgs a)
{
    Body body;
    run_pairs<Body, NT, TJ, 4>(a, body);
}


struct ConvVariant {
    KernelShape shape;
    KernelFn fn;
};

// compiled CONV shapes; the first of each list is the default
template <int D>
static const std::vector<ConvVariant>& conv_variants(bool grad)
{
    static const std::vector<ConvVariant> g = {
        {{2, 64, 32, 2, 512}, conv_kernel<PackedConvBody<D, 2, true, 64>, 64, 32, 4>},
        {{2, 128, 32, 2, 512}, conv_kernel<PackedConvBody<D, 2, true, 128>, 128, 32, 2>},
        {{1, 64, 32, 2, 512}, conv_kernel<PackedConvBody<D, 1, true, 64>, 64, 32, 6>},
        {{1, 128, 32, 2, 512}, conv_kernel<PackedConvBody<D, 1, true, 128>, 128, 32, 3>},
        {{1, 128, 64, 2, 512}, conv_kernel<PackedConvBody<D, 1, true, 128>, 128, 64, 2>},
        {{1, 128, 64}, conv_kernel<ConvBody<D, 1, true>, 128, 64>},
        {{2, 128, 64}, conv_kernel<ConvBody<D, 2, true>, 128, 64>},
        {{1, 256, 32}, conv_kernel<ConvBody<D, 1, true>, 256, 32>},
        {{1, 64, 64}, conv_kernel<ConvBody<D, 1, true>, 64, 64>},
    };
    static const std::vector<ConvVariant> e = {
        {{1, 128, 32, 2, 512}, conv_kernel<PackedConvBody<D, 1, false, 128>, 128, 32, 4>},
        {{2, 128, 32, 2, 512}, conv_kernel<PackedConvBody<D, 2, false, 128>, 128, 32, 3>},
        {{2, 128, 64}, conv_kernel<ConvBody<D, 2, false>, 128, 64>},
        {{1, 128, 64}, conv_kernel<ConvBody<D, 1, false>, 128, 64>},
        {{4, 128, 64}, conv_kernel<ConvBody<D, 4, false>, 128, 64>},
        {{2, 256, 32}, conv_kernel<ConvBody<D, 2, false>, 256, 32>},
    };
    return grad ? g : e;
}

std::vector<KernelShape> conv_shapes(bool grad)
{
    std::vector<KernelShape> s;
    for (auto& v : conv_variants<3>(grad)) s.push_back(v.shape);
    return s;
}

int conv_launch(Context& c, const double* pose_dev, bool grad, int i0, int i1, double* out_dev, double* dEdx_dev,
                cudaStream_t s, const KernelShape* force)
{
    const KernelShape want = force ? *force : (grad ? c.shape_conv_adj : c.shape_conv_energy);
    const std::vector<ConvVariant>& vars = c.D == 3 ? conv_variants<3>(grad) : conv_variants<2>(grad);
    const ConvVariant* v = &vars[0];
    for (auto& cand : vars)
        if (cand.shape.same(want)) v = &cand;
    const bool packed = v->shape.pack == 2;
    // source records always; target records scalar (YRec) or paired (YRec2, same bytes)
    const int n = std::max(c.M_pad, c.N_pad);
    const int g = std::min((n + 255) / 256, c.num_sms * 4);
    const int my = packed ? 0 : c.M, myp = packed ? 0 : c.M_pad;
    if (c.D == 3)
        conv_prologue_kernel<3><<<g, 256, 0, s>>>(pose_dev, c.y, c.ycov, my, myp, c.yrec, c.x, c.xcov, c.N, c.N_pad,
                                                  c.xrec);
    else
        conv_prologue_kernel<2><<<g, 256, 0, s>>>(pose_dev, c.y, c.ycov, my, myp, c.yrec, c.x, c.xcov, c.N, c.N_pad,
                                                  c.xrec);
    DUGMA_CK(cudaGetLastError());
    if (packed) {
        YRec2* y2 = reinterpret_cast<YRec2*>(c.yrec);
        const int g2 = std::min((c.M_pad / 2 + 255) / 256, c.num_sms * 4);
        if (c.D == 3)
            conv_prologue2_kernel<3><<<g2, 256, 0, s>>>(pose_dev, c.y, c.ycov, c.M, c.M_pad, y2);
        else
            conv_prologue2_kernel<2><<<g2, 256, 0, s>>>(pose_dev, c.y, c.ycov, c.M, c.M_pad, y2);
        DUGMA_CK(cudaGetLastError());
    }
    const int nv = grad ? 1 + (c.D == 3 ? 6 : 3) : 1;
    return launch_pair_variant(c, v->fn, v->shape, c.xrec, c.yrec, (size_t)c.M_pad / v->shape.pack, nv, c.cscale,
                               pose_dev, i0, i1, out_dev, grad ? dEdx_dev : nullptr, nullptr, 0, nullptr, s);
}

}  // namespace dugma

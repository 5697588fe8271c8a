// bodies.cuh -- per-pair bodies of the REF energy and fused adjoint kernels (scalar and packed
// f32x2 forms), shared by the single-problem launcher (energy.cu) and the batched one (batch.cu).
// The arithmetic of each body is described in energy.cu.
#pragma once

#include <cmath>

#include "context.hpp"
#include "pairs.cuh"

namespace dugma {

template <int D>
__device__ __forceinline__ void load_xrec(const XRec& r, float* x, float* b)
{
    x[0] = r.v0.x;
    x[1] = r.v0.y;
    if (D == 3) x[2] = r.v0.z;
    b[0] = r.v2.x;
    b[1] = r.v2.y;
    b[2] = r.v2.z;
    if (D == 3) {
        b[3] = r.v2.w;
        b[4] = r.v3.x;
        b[5] = r.v3.y;
    }
}

// ---------------------------------------------------------------------------
// Energy only (the "plain" form's kernel).  Horner quadratic forms: 26 FP32 + 2 SFU / pair (3D).
// ---------------------------------------------------------------------------
template <int D, int IPT_>
struct RefEnergyBody {
    using StreamRec = YRec;
    static constexpr int IPT = IPT_;
    static constexpr int NV = 1;
    static constexpr int NS = Sym<D>::N;
    float x[IPT][D], b[IPT][NS], e[IPT];
    double E64[IPT];
    int row[IPT];
    double G;

    __device__ void setup(const PairArgs& a)
    {
        const double s = 1.0 / a.pose[kPoseSig];
        G = pow(s, (double)D) * exp2(a.Lmax);
    }
    __device__ void load_src(const PairArgs& a, int ii, int i)
    {
        if (i < a.i_end) {
            row[ii] = i;
            load_xrec<D>(static_cast<const XRec*>(a.xrec)[i], x[ii], b[ii]);
        } else {
            row[ii] = -1;
#pragma unroll
            for (int q = 0; q < D; ++q) x[ii][q] = 0.f;
#pragma unroll
            for (int q = 0; q < NS; ++q) b[ii][q] = 0.f;
        }
    }
    __device__ void zero_all()
    {
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) { e[ii] = 0.f; E64[ii] = 0.0; }
    }
    __device__ __forceinline__ void consume(const YRec& r, int)
    {
        const float4 v0 = r.v0, v1 = r.v1, v2 = r.v2, v3 = r.v3;
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            if (D == 3) {
                const float d0 = (x[ii][0] - v0.x) - v1.x, d1 = (x[ii][1] - v0.y) - v1.y,
                            d2 = (x[ii][2] - v0.z) - v1.z;
                const float g0 = fmaf(v3.x, d2, fmaf(v2.w, d1, v2.x * d0));
                const float g1 = fmaf(v3.y, d2, v2.y * d1);
                const float g2 = v2.z * d2;
                const float t1 = fmaf(d0, g0, fmaf(d1, g1, fmaf(d2, g2, v0.w)));
                const float* B = b[ii];
                const float h0 = fmaf(B[4], d2, fmaf(B[3], d1, B[0] * d0));
                const float h1 = fmaf(B[5], d2, B[1] * d1);
                const float h2 = B[2] * d2;
                const float t2 = fmaf(d0, h0, fmaf(d1, h1, fmaf(d2, h2, v0.w)));
                e[ii] += ex2(t1);
                e[ii] += ex2(t2);
            } else {
                const float d0 = (x[ii][0] - v0.x) - v1.x, d1 = (x[ii][1] - v0.y) - v1.y;
                const float g0 = fmaf(v2.z, d1, v2.x * d0);
                const float g1 = v2.y * d1;
                const float t1 = fmaf(d0, g0, fmaf(d1, g1, v0.w));
                const float* B = b[ii];
                const float h0 = fmaf(B[2], d1, B[0] * d0);
                const float h1 = B[1] * d1;
                const float t2 = fmaf(d0, h0, fmaf(d1, h1, v0.w));
                e[ii] += ex2(t1);
                e[ii] += ex2(t2);
            }
        }
    }
    __device__ void fold()
    {
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) { E64[ii] += (double)e[ii]; e[ii] = 0.f; }
    }
    __device__ void finish(const PairArgs& a, int, double (&acc)[NV])
    {
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii)
            if (row[ii] >= 0) acc[0] += (double)a.wx[row[ii]] * G * E64[ii];
    }
};

// ---------------------------------------------------------------------------
// Fused adjoint.  Per pair (3D): d 6, u = kC'd 9, exponent 3, q = d d^T 6, exponent 6,
// accumulations 14  -> 44 FP32 + 2 SFU.
// ---------------------------------------------------------------------------
template <int D, int IPT_>
struct RefAdjointBody {
    using StreamRec = YRec;
    static constexpr int IPT = IPT_;
    static constexpr int NS = Sym<D>::N;
    static constexpr int NR = Sym<D>::NR;
    static constexpr int NV = 1 + NR + D;
    float x[IPT][D], b[IPT][NS];
    float e[IPT], S1[IPT][D], D2[IPT][D], Q2[IPT][NS];        // tile level
    float S1r[IPT][D], D2r[IPT][D], Q2r[IPT][NS];             // item level
    double E64[IPT];
    int row[IPT];
    double G, t[3];

    __device__ void setup(const PairArgs& a)
    {
        const double s = 1.0 / a.pose[kPoseSig];
        G = pow(s, (double)D) * exp2(a.Lmax);
#pragma unroll
        for (int q = 0; q < D; ++q) t[q] = a.pose[kPoseT + q];
    }
    __device__ void load_src(const PairArgs& a, int ii, int i)
    {
        if (i < a.i_end) {
            row[ii] = i;
            load_xrec<D>(static_cast<const XRec*>(a.xrec)[i], x[ii], b[ii]);
        } else {
            row[ii] = -1;
#pragma unroll
            for (int q = 0; q < D; ++q) x[ii][q] = 0.f;
#pragma unroll
            for (int q = 0; q < NS; ++q) b[ii][q] = 0.f;
        }
    }
    __device__ void zero_tile()
    {
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            e[ii] = 0.f;
#pragma unroll
            for (int q = 0; q < D; ++q) { S1[ii][q] = 0.f; D2[ii][q] = 0.f; }
#pragma unroll
            for (int q = 0; q < NS; ++q) Q2[ii][q] = 0.f;
        }
    }
    __device__ void zero_all()
    {
        zero_tile();
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            E64[ii] = 0.0;
#pragma unroll
            for (int q = 0; q < D; ++q) { S1r[ii][q] = 0.f; D2r[ii][q] = 0.f; }
#pragma unroll
            for (int q = 0; q < NS; ++q) Q2r[ii][q] = 0.f;
        }
    }
    __device__ __forceinline__ void consume(const YRec& r, int)
    {
        const float4 v0 = r.v0, v1 = r.v1, v2 = r.v2, v3 = r.v3;
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            const float* B = b[ii];
            if (D == 3) {
                const float d0 = (x[ii][0] - v0.x) - v1.x, d1 = (x[ii][1] - v0.y) - v1.y,
                            d2 = (x[ii][2] - v0.z) - v1.z;
                // u = k C' d with C' packed (c00, c11, c22, c01 | c02, c12)
                const float u0 = fmaf(v3.x, d2, fmaf(v2.w, d1, v2.x * d0));
                const float u1 = fmaf(v3.y, d2, fmaf(v2.y, d1, v2.w * d0));
                const float u2 = fmaf(v2.z, d2, fmaf(v3.y, d1, v3.x * d0));
                const float t1 = fmaf(d2, u2, fmaf(d1, u1, fmaf(d0, u0, v0.w)));
                // B exponent in Horner form (off-diagonals doubled in the x record)
                const float h0 = fmaf(B[4], d2, fmaf(B[3], d1, B[0] * d0));
                const float h1 = fmaf(B[5], d2, B[1] * d1);
                const float h2 = B[2] * d2;
                const float t2 = fmaf(d0, h0, fmaf(d1, h1, fmaf(d2, h2, v0.w)));
                const float e1 = ex2(t1), e2 = ex2(t2);
                e[ii] += e1;
                e[ii] += e2;
                S1[ii][0] = fmaf(e1, u0, S1[ii][0]);
                S1[ii][1] = fmaf(e1, u1, S1[ii][1]);
                S1[ii][2] = fmaf(e1, u2, S1[ii][2]);
                // moments of e2 through w = e2 d
                const float w0 = e2 * d0, w1 = e2 * d1, w2 = e2 * d2;
                D2[ii][0] += w0;
                D2[ii][1] += w1;
                D2[ii][2] += w2;
                Q2[ii][0] = fmaf(w0, d0, Q2[ii][0]);
                Q2[ii][1] = fmaf(w1, d1, Q2[ii][1]);
                Q2[ii][2] = fmaf(w2, d2, Q2[ii][2]);
                Q2[ii][3] = fmaf(w0, d1, Q2[ii][3]);
                Q2[ii][4] = fmaf(w0, d2, Q2[ii][4]);
                Q2[ii][5] = fmaf(w1, d2, Q2[ii][5]);
            } else {
                const float d0 = (x[ii][0] - v0.x) - v1.x, d1 = (x[ii][1] - v0.y) - v1.y;
                // C' packed (c00, c11, c01)
                const float u0 = fmaf(v2.z, d1, v2.x * d0);
                const float u1 = fmaf(v2.y, d1, v2.z * d0);
                const float t1 = fmaf(d1, u1, fmaf(d0, u0, v0.w));
                const float h0 = fmaf(B[2], d1, B[0] * d0);
                const float h1 = B[1] * d1;
                const float t2 = fmaf(d0, h0, fmaf(d1, h1, v0.w));
                const float e1 = ex2(t1), e2 = ex2(t2);
                e[ii] += e1;
                e[ii] += e2;
                S1[ii][0] = fmaf(e1, u0, S1[ii][0]);
                S1[ii][1] = fmaf(e1, u1, S1[ii][1]);
                const float w0 = e2 * d0, w1 = e2 * d1;
                D2[ii][0] += w0;
                D2[ii][1] += w1;
                Q2[ii][0] = fmaf(w0, d0, Q2[ii][0]);
                Q2[ii][1] = fmaf(w1, d1, Q2[ii][1]);
                Q2[ii][2] = fmaf(w0, d1, Q2[ii][2]);
            }
        }
    }
    __device__ void fold()
    {
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            E64[ii] += (double)e[ii];
#pragma unroll
            for (int q = 0; q < D; ++q) { S1r[ii][q] += S1[ii][q]; D2r[ii][q] += D2[ii][q]; }
#pragma unroll
            for (int q = 0; q < NS; ++q) Q2r[ii][q] += Q2[ii][q];
        }
        zero_tile();
    }
    __device__ void finish(const PairArgs& a, int jc, double (&acc)[NV])
    {
        const double kinv = 1.0 / K_EXP2;
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            if (row[ii] < 0) continue;
            const int i = row[ii];
            const double w = (double)a.wx[i] * G;
            double Bm[3][3], Qm[3][3];
#pragma unroll
            for (int q = 0; q < NS; ++q) {
                const int ra = Sym<D>::a(q), rb = Sym<D>::b(q);
                const double bv = (double)b[ii][q] * kinv * (ra == rb ? 1.0 : 0.5);
                Bm[ra][rb] = bv;
                Bm[rb][ra] = bv;
                Qm[ra][rb] = (double)Q2r[ii][q];
                Qm[rb][ra] = (double)Q2r[ii][q];
            }
            double gt[3], p[3];
#pragma unroll
            for (int q = 0; q < D; ++q) {
                double bd = 0;
#pragma unroll
                for (int c = 0; c < D; ++c) bd += Bm[q][c] * (double)D2r[ii][c];
                gt[q] = (double)S1r[ii][q] * kinv + bd;
                p[q] = (double)x[ii][q] - t[q];
            }
            acc[0] += w * E64[ii];
            if (D == 3) {
                double qx[3] = {0, 0, 0};
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    qx[0] += Bm[2][c] * Qm[1][c] - Bm[1][c] * Qm[2][c];
                    qx[1] += Bm[0][c] * Qm[2][c] - Bm[2][c] * Qm[0][c];
                    qx[2] += Bm[1][c] * Qm[0][c] - Bm[0][c] * Qm[1][c];
                }
                acc[1] += w * (p[1] * gt[2] - p[2] * gt[1] - qx[0]);
                acc[2] += w * (p[2] * gt[0] - p[0] * gt[2] - qx[1]);
                acc[3] += w * (p[0] * gt[1] - p[1] * gt[0] - qx[2]);
            } else {
                double qx = 0;
#pragma unroll
                for (int c = 0; c < 2; ++c) qx += Bm[1][c] * Qm[0][c] - Bm[0][c] * Qm[1][c];
                acc[1] += w * (p[0] * gt[1] - p[1] * gt[0] - qx);
            }
#pragma unroll
            for (int q = 0; q < D; ++q) acc[1 + NR + q] += w * gt[q];
            if (a.dx_part) {
                const int rows = a.i_end - a.i0;
#pragma unroll
                for (int q = 0; q < D; ++q) a.dx_part[((size_t)jc * rows + (i - a.i0)) * D + q] = -w * gt[q];
            }
        }
    }
};

// ---------------------------------------------------------------------------
// Packed-pair forms: the same per-pair arithmetic on two targets at once with the sm_100
// f32x2 instructions (each lane computes pair (i, 2p) in the low half and (i, 2p+1) in
// the high half), so each FP32 instruction issue does two pairs' work.  The algorithmic
// FP32 work per pair is unchanged; issue slots per pair drop from ~50 to ~27, leaving the
// FP32 pipe itself as the bound.  Targets arrive as YRec2 pair records.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 fld(const YRec2& r, int f)
{
    const float4 q = r.q[f >> 1];
    return (f & 1) ? make_float2(q.z, q.w) : make_float2(q.x, q.y);
}

// CHOL: the source side in the Cholesky form of the x record (U^T U = |k| B_i, z = U d): the B
// exponent is lv - |z|^2 (9 FP32 operations in 3D, as the Horner form), a sum of squares, so the FP32
// rounding of the record moves it by ~sqrt(cond B_i) ulps instead of ~cond B_i; the e2 moments are
// kept in the z frame (D2 = sum e2 z, Q2 = sum e2 z z^T) and mapped back per source in FP64.
// !CHOL: the Horner form of k B_i (sources whose sym(Sigma_x^-1) has no Cholesky factor).
template <int D, int IPT_, bool GRAD, bool CHOL = true>
struct PackedBody {
    using StreamRec = YRec2;
    static constexpr int IPT = IPT_;
    static constexpr int NS = Sym<D>::N;
    static constexpr int NR = Sym<D>::NR;
    static constexpr int NV = GRAD ? 1 + NR + D : 1;
    float2 X[IPT][D], B[IPT][NS];                 // source coordinates and k B_i (or U), duplicated in both halves
    float2 e[IPT];                                // energy, tile level
    float2 S1[IPT][GRAD ? D : 1], D2[IPT][GRAD ? D : 1], Q2[IPT][GRAD ? NS : 1];   // item level
    double E64[IPT];
    int row[IPT];
    double G, t[3];

    __device__ void setup(const PairArgs& a)
    {
        const double s = 1.0 / a.pose[kPoseSig];
        G = pow(s, (double)D) * exp2(a.Lmax);
#pragma unroll
        for (int q = 0; q < D; ++q) t[q] = a.pose[kPoseT + q];
    }
    __device__ void load_src(const PairArgs& a, int ii, int i)
    {
        float x[3] = {0, 0, 0}, b[6] = {0, 0, 0, 0, 0, 0};
        row[ii] = i < a.i_end ? i : -1;
        if (i < a.i_end) load_xrec<D>(static_cast<const XRec*>(a.xrec)[i], x, b);
#pragma unroll
        for (int q = 0; q < D; ++q) X[ii][q] = make_float2(x[q], x[q]);
#pragma unroll
        for (int q = 0; q < NS; ++q) B[ii][q] = make_float2(b[q], b[q]);
    }
    __device__ void zero_all()
    {
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            e[ii] = make_float2(0.f, 0.f);
            E64[ii] = 0.0;
            if (GRAD) {
#pragma unroll
                for (int q = 0; q < D; ++q) { S1[ii][q] = make_float2(0.f, 0.f); D2[ii][q] = make_float2(0.f, 0.f); }
#pragma unroll
                for (int q = 0; q < NS; ++q) Q2[ii][q] = make_float2(0.f, 0.f);
            }
        }
    }
    __device__ __forceinline__ void consume(const YRec2& r, int)
    {
        float2 ny[3], nl[3], c[6];
#pragma unroll
        for (int q = 0; q < D; ++q) { ny[q] = fld(r, q); nl[q] = fld(r, 4 + q); }
        const float2 lv = fld(r, 3);
        const float2 nlv = fld(r, 13);
#pragma unroll
        for (int k = 0; k < NS; ++k) c[k] = fld(r, 7 + k);
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            float2 d[3];
#pragma unroll
            for (int q = 0; q < D; ++q) d[q] = fadd2(fadd2(X[ii][q], ny[q]), nl[q]);
            const float2* b = B[ii];
            float2 t1, t2;
            float2 u[3], z[3];   // u = k C' d (gradient); z = U d (Cholesky form) or d (Horner form)
            if (!GRAD) {
                // Horner form of k C' (off-diagonals doubled)
                if (D == 3) {
                    const float2 g0 = ffma2(c[4], d[2], ffma2(c[3], d[1], fmul2(c[0], d[0])));
                    const float2 g1 = ffma2(c[5], d[2], fmul2(c[1], d[1]));
                    const float2 g2 = fmul2(c[2], d[2]);
                    t1 = ffma2(d[0], g0, ffma2(d[1], g1, ffma2(d[2], g2, lv)));
                } else {
                    const float2 g0 = ffma2(c[2], d[1], fmul2(c[0], d[0]));
                    const float2 g1 = fmul2(c[1], d[1]);
                    t1 = ffma2(d[0], g0, ffma2(d[1], g1, lv));
                }
            } else {
                if (D == 3) {
                    u[0] = ffma2(c[4], d[2], ffma2(c[3], d[1], fmul2(c[0], d[0])));
                    u[1] = ffma2(c[5], d[2], ffma2(c[1], d[1], fmul2(c[3], d[0])));
                    u[2] = ffma2(c[2], d[2], ffma2(c[5], d[1], fmul2(c[4], d[0])));
                    t1 = ffma2(d[2], u[2], ffma2(d[1], u[1], ffma2(d[0], u[0], lv)));
                } else {
                    u[0] = ffma2(c[2], d[1], fmul2(c[0], d[0]));
                    u[1] = ffma2(c[1], d[1], fmul2(c[2], d[0]));
                    t1 = ffma2(d[1], u[1], ffma2(d[0], u[0], lv));
                }
            }
            float2 e2;
            if (CHOL) {
                // z = U d; e2 = 2^(lv - |z|^2)
                float2 m2;
                if (D == 3) {
                    z[0] = ffma2(b[4], d[2], ffma2(b[3], d[1], fmul2(b[0], d[0])));
                    z[1] = ffma2(b[5], d[2], fmul2(b[1], d[1]));
                    z[2] = fmul2(b[2], d[2]);
                    m2 = ffma2(z[0], z[0], ffma2(z[1], z[1], ffma2(z[2], z[2], nlv)));
                } else {
                    z[0] = ffma2(b[2], d[1], fmul2(b[0], d[0]));
                    z[1] = fmul2(b[1], d[1]);
                    m2 = ffma2(z[0], z[0], ffma2(z[1], z[1], nlv));
                }
                e2 = make_float2(ex2(-m2.x), ex2(-m2.y));
            } else {
                // Horner form of k B_i (the x record's off-diagonals are doubled)
                if (D == 3) {
                    const float2 h0 = ffma2(b[4], d[2], ffma2(b[3], d[1], fmul2(b[0], d[0])));
                    const float2 h1 = ffma2(b[5], d[2], fmul2(b[1], d[1]));
                    const float2 h2 = fmul2(b[2], d[2]);
                    t2 = ffma2(d[0], h0, ffma2(d[1], h1, ffma2(d[2], h2, lv)));
                } else {
                    const float2 h0 = ffma2(b[2], d[1], fmul2(b[0], d[0]));
                    const float2 h1 = fmul2(b[1], d[1]);
                    t2 = ffma2(d[0], h0, ffma2(d[1], h1, lv));
                }
#pragma unroll
                for (int q = 0; q < D; ++q) z[q] = d[q];
                e2 = make_float2(ex2(t2.x), ex2(t2.y));
            }
            const float2 e1 = make_float2(ex2(t1.x), ex2(t1.y));
            e[ii] = fadd2(fadd2(e[ii], e1), e2);
            if (GRAD) {
                // moments of e2: w = e2 z, then sum w and w z^T (only z lives across the SFU latency)
                float2 w[3];
#pragma unroll
                for (int q = 0; q < D; ++q) {
                    S1[ii][q] = ffma2(e1, u[q], S1[ii][q]);
                    w[q] = fmul2(e2, z[q]);
                    D2[ii][q] = fadd2(D2[ii][q], w[q]);
                }
#pragma unroll
                for (int k = 0; k < NS; ++k) Q2[ii][k] = ffma2(w[Sym<D>::a(k)], z[Sym<D>::b(k)], Q2[ii][k]);
            }
        }
    }
    __device__ void fold()
    {
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            E64[ii] += (double)e[ii].x + (double)e[ii].y;
            e[ii] = make_float2(0.f, 0.f);
        }
    }
    __device__ void finish(const PairArgs& a, int jc, double (&acc)[NV])
    {
        if (CHOL)
            finish_chol(a, jc, acc);
        else
            finish_horner(a, jc, acc);
    }
    // Cholesky form: with U the record's factor (U^T U = |k| B), V = U^-1 and the z-frame moments,
    //   B D2 = U^T D2z / |k|,   sum e2 d x B d = sum_ab Q2z_ab (V e_a) x (U^T e_b) / |k|.
    __device__ void finish_chol(const PairArgs& a, int jc, double (&acc)[NV])
    {
        const double kinv = 1.0 / K_EXP2, rk = -kinv;
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            if (row[ii] < 0) continue;
            const int i = row[ii];
            const double w = (double)a.wx[i] * G;
            acc[0] += w * E64[ii];
            if (!GRAD) continue;
            double gt[3] = {0, 0, 0};
            if (w != 0.0) {   // neglected sources carry U = 0 and weight 0
                double U[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, Qm[3][3], s1[3], d2[3];
#pragma unroll
                for (int q = 0; q < NS; ++q) {
                    const int ra = Sym<D>::a(q), rb = Sym<D>::b(q);
                    U[ra][rb] = (double)B[ii][q].x;
                    Qm[ra][rb] = Qm[rb][ra] = (double)Q2[ii][q].x + (double)Q2[ii][q].y;
                }
#pragma unroll
                for (int q = 0; q < D; ++q) {
                    s1[q] = (double)S1[ii][q].x + (double)S1[ii][q].y;
                    d2[q] = (double)D2[ii][q].x + (double)D2[ii][q].y;
                }
                double V[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
                V[0][0] = 1.0 / U[0][0];
                V[1][1] = 1.0 / U[1][1];
                V[0][1] = -U[0][1] * V[0][0] * V[1][1];
                if (D == 3) {
                    V[2][2] = 1.0 / U[2][2];
                    V[1][2] = -U[1][2] * V[1][1] * V[2][2];
                    V[0][2] = (U[0][1] * U[1][2] - U[0][2] * U[1][1]) * V[0][0] * V[1][1] * V[2][2];
                }
                double p[3];
#pragma unroll
                for (int q = 0; q < D; ++q) {
                    double bd = 0;
#pragma unroll
                    for (int cc = 0; cc < D; ++cc) bd += U[cc][q] * d2[cc];
                    gt[q] = s1[q] * kinv + rk * bd;
                    p[q] = (double)X[ii][q].x - t[q];
                }
                if (D == 3) {
                    double qx[3] = {0, 0, 0};
#pragma unroll
                    for (int aa = 0; aa < 3; ++aa)
#pragma unroll
                        for (int bb = 0; bb < 3; ++bb) {
                            const double q = Qm[aa][bb];
                            qx[0] += q * (V[1][aa] * U[bb][2] - V[2][aa] * U[bb][1]);
                            qx[1] += q * (V[2][aa] * U[bb][0] - V[0][aa] * U[bb][2]);
                            qx[2] += q * (V[0][aa] * U[bb][1] - V[1][aa] * U[bb][0]);
                        }
                    acc[1] += w * (p[1] * gt[2] - p[2] * gt[1] - rk * qx[0]);
                    acc[2] += w * (p[2] * gt[0] - p[0] * gt[2] - rk * qx[1]);
                    acc[3] += w * (p[0] * gt[1] - p[1] * gt[0] - rk * qx[2]);
                } else {
                    double qx = 0;
#pragma unroll
                    for (int aa = 0; aa < 2; ++aa)
#pragma unroll
                        for (int bb = 0; bb < 2; ++bb) qx += Qm[aa][bb] * (V[0][aa] * U[bb][1] - V[1][aa] * U[bb][0]);
                    acc[1] += w * (p[0] * gt[1] - p[1] * gt[0] - rk * qx);
                }
#pragma unroll
                for (int q = 0; q < D; ++q) acc[1 + NR + q] += w * gt[q];
            }
            if (a.dx_part) {
                const int rows = a.i_end - a.i0;
#pragma unroll
                for (int q = 0; q < D; ++q) a.dx_part[((size_t)jc * rows + (i - a.i0)) * D + q] = -w * gt[q];
            }
        }
    }
    __device__ void finish_horner(const PairArgs& a, int jc, double (&acc)[NV])
    {
        const double kinv = 1.0 / K_EXP2;
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            if (row[ii] < 0) continue;
            const int i = row[ii];
            const double w = (double)a.wx[i] * G;
            acc[0] += w * E64[ii];
            if (!GRAD) continue;
            double Bm[3][3], Qm[3][3], s1[3], d2[3];
#pragma unroll
            for (int q = 0; q < NS; ++q) {
                const int ra = Sym<D>::a(q), rb = Sym<D>::b(q);
                const double bv = (double)B[ii][q].x * kinv * (ra == rb ? 1.0 : 0.5);
                Bm[ra][rb] = Bm[rb][ra] = bv;
                Qm[ra][rb] = Qm[rb][ra] = (double)Q2[ii][q].x + (double)Q2[ii][q].y;
            }
#pragma unroll
            for (int q = 0; q < D; ++q) {
                s1[q] = (double)S1[ii][q].x + (double)S1[ii][q].y;
                d2[q] = (double)D2[ii][q].x + (double)D2[ii][q].y;
            }
            double gt[3], p[3];
#pragma unroll
            for (int q = 0; q < D; ++q) {
                double bd = 0;
#pragma unroll
                for (int cc = 0; cc < D; ++cc) bd += Bm[q][cc] * d2[cc];
                gt[q] = s1[q] * kinv + bd;
                p[q] = (double)X[ii][q].x - t[q];
            }
            if (D == 3) {
                double qx[3] = {0, 0, 0};
#pragma unroll
                for (int cc = 0; cc < 3; ++cc) {
                    qx[0] += Bm[2][cc] * Qm[1][cc] - Bm[1][cc] * Qm[2][cc];
                    qx[1] += Bm[0][cc] * Qm[2][cc] - Bm[2][cc] * Qm[0][cc];
                    qx[2] += Bm[1][cc] * Qm[0][cc] - Bm[0][cc] * Qm[1][cc];
                }
                acc[1] += w * (p[1] * gt[2] - p[2] * gt[1] - qx[0]);
                acc[2] += w * (p[2] * gt[0] - p[0] * gt[2] - qx[1]);
                acc[3] += w * (p[0] * gt[1] - p[1] * gt[0] - qx[2]);
            } else {
                double qx = 0;
#pragma unroll
                for (int cc = 0; cc < 2; ++cc) qx += Bm[1][cc] * Qm[0][cc] - Bm[0][cc] * Qm[1][cc];
                acc[1] += w * (p[0] * gt[1] - p[1] * gt[0] - qx);
            }
#pragma unroll
            for (int q = 0; q < D; ++q) acc[1 + NR + q] += w * gt[q];
            if (a.dx_part) {
                const int rows = a.i_end - a.i0;
#pragma unroll
                for (int q = 0; q < D; ++q) a.dx_part[((size_t)jc * rows + (i - a.i0)) * D + q] = -w * gt[q];
            }
        }
    }
};


}  // namespace dugma

// energy.cu -- REF energy and fused adjoint (energy + pose gradient + dE/dx) kernels.
//
// Per pair (compi.cu:753-772 restated):  d = x_i - y'_j,
//   e1 = exp(-1/2 d^T C'_j d),  e2 = exp(-1/2 d^T B_i d),  P_ij = w_i v_j (e1 + e2).
// FP32 per pair; d from the double-float split of y' (y'hi, y'lo) so that the
// cancellation x - y' is exact for near pairs; the -1/2 log2 e factor is folded into
// C' and B, and log2 v_j into the exponent, so each exponential is one SFU ex2.
//
// Adjoint (left perturbation R <- exp([w]x) R, t <- t + dt), per source row i:
//   S1 = sum_j e1' k C'd,   D2 = sum_j e2' d,   Q2 = sum_j e2' d d^T,   E = sum_j (e1' + e2')
//   dE/dt     += w_i (S1/k + B_i D2)
//   dE/dw     += w_i ((x_i - t) x (S1/k + B_i D2) - sum_j e2' d x B_i d)   [from Q2 and B_i]
//   dE/dx_i    = -w_i (S1/k + B_i D2)
// (e' = v_j e / 2^Lmax; w_i = |Sx|^-1/2 s^D 2^Lmax; the e2 rotation term uses R y_j = (x_i - t) - d.)
// Accumulation: FP32 within a tile of TJ targets, then the energy in FP64 and the
// gradient moments in a second FP32 level per item, FP64 across items.
#include <cmath>
#include <mutex>

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
                const float q00 = d0 * d0, q11 = d1 * d1, q22 = d2 * d2;
                const float q01 = d0 * d1, q02 = d0 * d2, q12 = d1 * d2;
                const float t2 =
                    fmaf(B[5], q12, fmaf(B[4], q02, fmaf(B[3], q01, fmaf(B[2], q22, fmaf(B[1], q11, fmaf(B[0], q00, v0.w))))));
                const float e1 = ex2(t1), e2 = ex2(t2);
                e[ii] += e1;
                e[ii] += e2;
                S1[ii][0] = fmaf(e1, u0, S1[ii][0]);
                S1[ii][1] = fmaf(e1, u1, S1[ii][1]);
                S1[ii][2] = fmaf(e1, u2, S1[ii][2]);
                D2[ii][0] = fmaf(e2, d0, D2[ii][0]);
                D2[ii][1] = fmaf(e2, d1, D2[ii][1]);
                D2[ii][2] = fmaf(e2, d2, D2[ii][2]);
                Q2[ii][0] = fmaf(e2, q00, Q2[ii][0]);
                Q2[ii][1] = fmaf(e2, q11, Q2[ii][1]);
                Q2[ii][2] = fmaf(e2, q22, Q2[ii][2]);
                Q2[ii][3] = fmaf(e2, q01, Q2[ii][3]);
                Q2[ii][4] = fmaf(e2, q02, Q2[ii][4]);
                Q2[ii][5] = fmaf(e2, q12, Q2[ii][5]);
            } else {
                const float d0 = (x[ii][0] - v0.x) - v1.x, d1 = (x[ii][1] - v0.y) - v1.y;
                // C' packed (c00, c11, c01)
                const float u0 = fmaf(v2.z, d1, v2.x * d0);
                const float u1 = fmaf(v2.y, d1, v2.z * d0);
                const float t1 = fmaf(d1, u1, fmaf(d0, u0, v0.w));
                const float q00 = d0 * d0, q11 = d1 * d1, q01 = d0 * d1;
                const float t2 = fmaf(B[2], q01, fmaf(B[1], q11, fmaf(B[0], q00, v0.w)));
                const float e1 = ex2(t1), e2 = ex2(t2);
                e[ii] += e1;
                e[ii] += e2;
                S1[ii][0] = fmaf(e1, u0, S1[ii][0]);
                S1[ii][1] = fmaf(e1, u1, S1[ii][1]);
                D2[ii][0] = fmaf(e2, d0, D2[ii][0]);
                D2[ii][1] = fmaf(e2, d1, D2[ii][1]);
                Q2[ii][0] = fmaf(e2, q00, Q2[ii][0]);
                Q2[ii][1] = fmaf(e2, q11, Q2[ii][1]);
                Q2[ii][2] = fmaf(e2, q01, Q2[ii][2]);
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

template <int D, int IPT_, bool GRAD>
struct PackedBody {
    using StreamRec = YRec2;
    static constexpr int IPT = IPT_;
    static constexpr int NS = Sym<D>::N;
    static constexpr int NR = Sym<D>::NR;
    static constexpr int NV = GRAD ? 1 + NR + D : 1;
    float2 X[IPT][D], B[IPT][NS];                 // source coordinates and k B_i, duplicated in both halves
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
#pragma unroll
        for (int k = 0; k < NS; ++k) c[k] = fld(r, 7 + k);
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            float2 d[3];
#pragma unroll
            for (int q = 0; q < D; ++q) d[q] = fadd2(fadd2(X[ii][q], ny[q]), nl[q]);
            const float2* b = B[ii];
            float2 t1, t2;
            float2 u[3], qq[6];
            if (!GRAD) {
                // Horner forms (off-diagonals doubled in both matrices)
                if (D == 3) {
                    const float2 g0 = ffma2(c[4], d[2], ffma2(c[3], d[1], fmul2(c[0], d[0])));
                    const float2 g1 = ffma2(c[5], d[2], fmul2(c[1], d[1]));
                    const float2 g2 = fmul2(c[2], d[2]);
                    t1 = ffma2(d[0], g0, ffma2(d[1], g1, ffma2(d[2], g2, lv)));
                    const float2 h0 = ffma2(b[4], d[2], ffma2(b[3], d[1], fmul2(b[0], d[0])));
                    const float2 h1 = ffma2(b[5], d[2], fmul2(b[1], d[1]));
                    const float2 h2 = fmul2(b[2], d[2]);
                    t2 = ffma2(d[0], h0, ffma2(d[1], h1, ffma2(d[2], h2, lv)));
                } else {
                    const float2 g0 = ffma2(c[2], d[1], fmul2(c[0], d[0]));
                    const float2 g1 = fmul2(c[1], d[1]);
                    t1 = ffma2(d[0], g0, ffma2(d[1], g1, lv));
                    const float2 h0 = ffma2(b[2], d[1], fmul2(b[0], d[0]));
                    const float2 h1 = fmul2(b[1], d[1]);
                    t2 = ffma2(d[0], h0, ffma2(d[1], h1, lv));
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
#pragma unroll
                for (int k = 0; k < NS; ++k) qq[k] = fmul2(d[Sym<D>::a(k)], d[Sym<D>::b(k)]);
                t2 = lv;
#pragma unroll
                for (int k = 0; k < NS; ++k) t2 = ffma2(b[k], qq[k], t2);
            }
            const float2 e1 = make_float2(ex2(t1.x), ex2(t1.y));
            const float2 e2 = make_float2(ex2(t2.x), ex2(t2.y));
            e[ii] = fadd2(fadd2(e[ii], e1), e2);
            if (GRAD) {
#pragma unroll
                for (int q = 0; q < D; ++q) {
                    S1[ii][q] = ffma2(e1, u[q], S1[ii][q]);
                    D2[ii][q] = ffma2(e2, d[q], D2[ii][q]);
                }
#pragma unroll
                for (int k = 0; k < NS; ++k) Q2[ii][k] = ffma2(e2, qq[k], Q2[ii][k]);
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

template <class Body, int NT, int TJ>
__global__ void __launch_bounds__(NT) pair_kernel(PairArgs a)
{
    Body body;
    run_pairs<Body, NT, TJ, 4>(a, body);
}

// deterministic reduction of per-item partials: out[v] = sum_items partials[item][v];
// block v sums value v in a fixed order (strided per thread, then a fixed tree)
__global__ void __launch_bounds__(1024) reduce_items_kernel(const double* __restrict__ part, int n_items, int nv,
                                                             double* __restrict__ out)
{
    __shared__ double red[1024];
    const int v = blockIdx.x;
    if (v >= nv) return;
    double s = 0;
    for (int it = threadIdx.x; it < n_items; it += blockDim.x) s += part[(size_t)it * 8 + v];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[v] = red[0];
}

__global__ void reduce_chunks_kernel(const double* __restrict__ part, int n_jc, size_t n, double* __restrict__ out)
{
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        double s = 0;
        for (int c = 0; c < n_jc; ++c) s += part[(size_t)c * n + e];
        out[e] = s;
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
using KernelFn = void (*)(PairArgs);

struct Variant {
    KernelShape shape;
    KernelFn fn;
};

template <int D>
static const std::vector<Variant>& adjoint_variants()
{
    // packed gradient variants keep their moment sums in FP32 over one item: at most 512 pair
    // records (1024 targets) per item bounds that sum's rounding error
    static const std::vector<Variant> v = {
        {{2, 128, 64}, pair_kernel<RefAdjointBody<D, 2>, 128, 64>},
        {{1, 128, 64}, pair_kernel<RefAdjointBody<D, 1>, 128, 64>},
        {{1, 256, 64}, pair_kernel<RefAdjointBody<D, 1>, 256, 64>},
        {{2, 256, 32}, pair_kernel<RefAdjointBody<D, 2>, 256, 32>},
        {{1, 128, 32, 2, 512}, pair_kernel<PackedBody<D, 1, true>, 128, 32>},
        {{2, 128, 32, 2, 512}, pair_kernel<PackedBody<D, 2, true>, 128, 32>},
        {{1, 256, 32, 2, 512}, pair_kernel<PackedBody<D, 1, true>, 256, 32>},
    };
    return v;
}

template <int D>
static const std::vector<Variant>& energy_variants()
{
    static const std::vector<Variant> v = {
        {{4, 128, 64}, pair_kernel<RefEnergyBody<D, 4>, 128, 64>},
        {{2, 128, 64}, pair_kernel<RefEnergyBody<D, 2>, 128, 64>},
        {{2, 256, 64}, pair_kernel<RefEnergyBody<D, 2>, 256, 64>},
        {{4, 256, 32}, pair_kernel<RefEnergyBody<D, 4>, 256, 32>},
        {{2, 128, 32, 2}, pair_kernel<PackedBody<D, 2, false>, 128, 32>},
        {{4, 128, 32, 2}, pair_kernel<PackedBody<D, 4, false>, 128, 32>},
        {{2, 256, 32, 2}, pair_kernel<PackedBody<D, 2, false>, 256, 32>},
    };
    return v;
}

std::vector<KernelShape> adjoint_shapes()
{
    std::vector<KernelShape> s;
    for (auto& v : adjoint_variants<3>()) s.push_back(v.shape);
    return s;
}
std::vector<KernelShape> energy_shapes()
{
    std::vector<KernelShape> s;
    for (auto& v : energy_variants<3>()) s.push_back(v.shape);
    return s;
}

int conv_launch(Context& c, const double* pose_dev, bool grad, int i0, int i1, double* out_dev, double* dEdx_dev,
                cudaStream_t s, const KernelShape* force);   // conv.cu

static int occupancy_blocks(KernelFn fn, int nt)
{
    static std::mutex mu;
    static std::vector<std::pair<KernelFn, int>> cache;
    std::lock_guard<std::mutex> lk(mu);
    for (auto& e : cache)
        if (e.first == fn) return e.second;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, nt, 0) != cudaSuccess || nb < 1) nb = 1;
    cache.push_back({fn, nb});
    return nb;
}

// Splits [i0, i1) x targets into items and launches `fn`, then the reductions.
int launch_pair_variant(Context& c, KernelFn fn, const KernelShape& sh, const void* xrec, const void* yrec,
                        size_t yrec_size, int nv, double Lmax, const double* pose_dev, int i0, int i1,
                        double* out_dev, double* dEdx_dev, double** h_part, int h_width, int* n_jc_out,
                        cudaStream_t s)
{
    const int rows = i1 - i0;
    const int BI = sh.ipt * sh.nt;
    const int n_ib = (rows + BI - 1) / BI;
    const int total_tiles = (int)(yrec_size / sh.tj);
    const int resident = c.num_sms * occupancy_blocks(fn, sh.nt);
    const int target = 4 * resident;
    int n_jc = std::max(1, std::min(total_tiles, (target + n_ib - 1) / n_ib));
    if (sh.max_chunk > 0) n_jc = std::max(n_jc, (total_tiles * sh.tj + sh.max_chunk - 1) / sh.max_chunk);
    n_jc = std::min(n_jc, total_tiles);
    const int jc_tiles = (total_tiles + n_jc - 1) / n_jc;
    n_jc = (total_tiles + jc_tiles - 1) / jc_tiles;
    const int n_items = n_ib * n_jc;
    size_t need = sizeof(double) * (size_t)n_items * 8;
    const size_t dx_off = need;
    if (dEdx_dev) need += sizeof(double) * (size_t)n_jc * rows * c.D;
    const size_t h_off = need;
    if (h_part) need += sizeof(double) * (size_t)n_jc * rows * h_width;
    DUGMA_RET(c.ensure_scratch(need));
    PairArgs a{};
    a.xrec = xrec;
    a.yrec = yrec;
    a.wx = c.wx;
    a.wy = c.wy;
    a.xcov = c.xcov;
    a.ycov = c.ycov;
    a.pose = pose_dev;
    a.Lmax = Lmax;
    a.N = c.N;
    a.i0 = i0;
    a.i_end = i1;
    a.n_ib = n_ib;
    a.n_jc = n_jc;
    a.jc_tiles = jc_tiles;
    a.total_tiles = total_tiles;
    a.partials = c.scratch;
    a.dx_part = dEdx_dev ? reinterpret_cast<double*>(reinterpret_cast<char*>(c.scratch) + dx_off) : nullptr;
    a.h_part = h_part ? reinterpret_cast<double*>(reinterpret_cast<char*>(c.scratch) + h_off) : nullptr;
    a.counter = c.counter;
    a.err = c.err;
    if (h_part) *h_part = a.h_part;
    if (n_jc_out) *n_jc_out = n_jc;
    DUGMA_CK(cudaMemsetAsync(c.counter, 0, sizeof(int), s));
    const int grid = std::min(resident, n_items);
    cudaEvent_t ev1 = nullptr;
    if (c.timing) {
        if (c.tused == c.tevents.size()) {
            cudaEvent_t e0, e1;
            DUGMA_CK(cudaEventCreate(&e0));
            DUGMA_CK(cudaEventCreate(&e1));
            c.tevents.push_back({e0, e1});
        }
        DUGMA_CK(cudaEventRecord(c.tevents[c.tused].first, s));
        ev1 = c.tevents[c.tused].second;
        ++c.tused;
    }
    fn<<<grid, sh.nt, 0, s>>>(a);
    DUGMA_CK(cudaGetLastError());
    if (ev1) DUGMA_CK(cudaEventRecord(ev1, s));
    if (out_dev) {
        reduce_items_kernel<<<nv, 1024, 0, s>>>(a.partials, n_items, nv, out_dev);
        DUGMA_CK(cudaGetLastError());
    }
    if (dEdx_dev) {
        const size_t n = (size_t)rows * c.D;
        const int g = (int)std::min<size_t>((n + 255) / 256, (size_t)c.num_sms * 8);
        reduce_chunks_kernel<<<g, 256, 0, s>>>(a.dx_part, n_jc, n, dEdx_dev);
        DUGMA_CK(cudaGetLastError());
    }
    return DUGMA_OK;
}

int launch_pairs(Context& c, const double* pose_dev, int model, bool grad, int i0, int i1, double* out_dev,
                 double* dEdx_dev, cudaStream_t s, const KernelShape* force)
{
    if (i0 < 0 || i1 > c.N || i0 >= i1) return set_error(DUGMA_ERR_ARG, "bad source row range [%d, %d)", i0, i1);
    if (model == DUGMA_MODEL_CONV) return conv_launch(c, pose_dev, grad, i0, i1, out_dev, dEdx_dev, s, force);
    if (model != DUGMA_MODEL_REF) return set_error(DUGMA_ERR_ARG, "unknown model %d", model);
    const KernelShape want = force ? *force : (grad ? c.shape_adj : c.shape_energy);
    const std::vector<Variant>& vars =
        c.D == 3 ? (grad ? adjoint_variants<3>() : energy_variants<3>()) : (grad ? adjoint_variants<2>() : energy_variants<2>());
    const Variant* v = &vars[0];
    for (auto& cand : vars)
        if (cand.shape.same(want)) v = &cand;
    // record layout: 0 scalar adjoint, 1 scalar Horner energy, 2 / 3 their packed-pair forms
    const int layout = (grad ? 0 : 1) + (v->shape.pack == 2 ? 2 : 0);
    DUGMA_RET(launch_prologue(c, pose_dev, layout, s));
    const int nv = grad ? 1 + (c.D == 3 ? 6 : 3) : 1;
    return launch_pair_variant(c, v->fn, v->shape, c.xrec, c.yrec, (size_t)c.M_pad / v->shape.pack, nv, c.Lmax_y,
                               pose_dev, i0, i1, out_dev, grad ? dEdx_dev : nullptr, nullptr, 0, nullptr, s);
}

// ---------------------------------------------------------------------------
// Allocation-free fused adjoint.
//
// For callers that cannot allocate device memory while they evaluate: code that runs
// while a CUDA graph is being captured (allocation calls are not allowed there), loops
// with a latency budget that must never enter an allocator, and host applications that
// own every device allocation themselves.  They pass the six input arrays and the
// output buffer; everything the evaluation needs besides them (per-pose records,
// normalised weights, work-queue counter, per-item partial sums) lives in one
// file-scope device array of kNoAllocScratchBytes, which every GPU that loads this
// library holds until the process exits.
// ---------------------------------------------------------------------------
constexpr size_t kNoAllocScratchBytes = (size_t)4 << 20;   // 4 MiB
constexpr int kNoAllocMaxPadded = 16384;                     // N and M, after padding to 1024 / 128

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// max_j log2(w_j) over positive weights into *out (one block, fixed order)
__global__ void noalloc_max_log2_kernel(const float* __restrict__ w, int n, double* out)
{
    __shared__ double red[256];
    double m = -INFINITY;
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if (w[i] > 0.0f) m = fmax(m, log2((double)w[i]));
    red[threadIdx.x] = m;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + h]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = isfinite(red[0]) ? red[0] : 0.0;
}

__global__ void noalloc_norm_log2_kernel(const float* __restrict__ w, int n, const double* Lmax, float* __restrict__ lw)
{
    const double L = *Lmax;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        lw[i] = w[i] > 0.0f ? __double2float_rn(log2((double)w[i]) - L) : -INFINITY;
}

// the pair kernel ran with a zero weight offset: restore the 2^Lmax_y factor of every output
__global__ void noalloc_scale_kernel(double* out, int n, const double* Lmax)
{
    if (threadIdx.x < n) out[threadIdx.x] *= exp2(*Lmax);
}

static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[64];

}  // namespace dugma

extern "C" int dugma_energy_grad_noalloc(const float* x, const float* x_cov_inv, const float* y, const float* y_cov_inv,
                                         const float* det_x, const float* det_y, int N, int M, int D,
                                         const double* pose_dev, double* out_dev, void* stream)
{
    using namespace dugma;
    if (!x || !x_cov_inv || !det_x || !y || !y_cov_inv || !det_y || !pose_dev || !out_dev)
        return set_error(DUGMA_ERR_ARG, "energy_grad_noalloc: null argument");
    if (D != 2 && D != 3) return set_error(DUGMA_ERR_ARG, "energy_grad_noalloc: D must be 2 or 3 (got %d)", D);
    const int N_pad = (N + kPadI - 1) / kPadI * kPadI, M_pad = (M + kPadJ - 1) / kPadJ * kPadJ;
    if (N < 1 || M < 1 || N_pad > kNoAllocMaxPadded || M_pad > kNoAllocMaxPadded)
        return set_error(DUGMA_ERR_ARG,
                         "energy_grad_noalloc: N = %d, M = %d; this entry point takes 1 <= N, M <= %d (its scratch is "
                         "a fixed %zu-byte device array); use dugma_energy_grad for larger clouds",
                         N, M, kNoAllocMaxPadded, kNoAllocScratchBytes);
    int dev = 0;
    DUGMA_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return set_error(DUGMA_ERR_ARG, "energy_grad_noalloc: device %d out of range", dev);
    const Variant& var = D == 3 ? adjoint_variants<3>()[0] : adjoint_variants<2>()[0];
    unsigned char* base = nullptr;
    {
        // once per device: the device address of the scratch array (a host-side name is not one)
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_addr[dev]) {
            void* p = nullptr;
            DUGMA_CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
            occupancy_blocks(var.fn, var.shape.nt);   // fills the launch-shape cache before any capture
            g_noalloc_addr[dev] = p;
        }
        base = static_cast<unsigned char*>(g_noalloc_addr[dev]);
    }
    // carve: records, normalised log weights, offsets, counters, then partial sums
    size_t off = 0;
    auto take = [&](size_t bytes) {
        unsigned char* p = base + off;
        off += (bytes + 255) / 256 * 256;
        return p;
    };
    Context c;   // a view of the caller's arrays and the static scratch; owns nothing
    c.N = N;
    c.M = M;
    c.D = D;
    c.N_pad = N_pad;
    c.M_pad = M_pad;
    c.dev = dev;
    cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, dev);
    c.x = const_cast<float*>(x);
    c.xinv = const_cast<float*>(x_cov_inv);
    c.wx = const_cast<float*>(det_x);
    c.y = const_cast<float*>(y);
    c.yinv = const_cast<float*>(y_cov_inv);
    c.wy = const_cast<float*>(det_y);
    c.xrec = reinterpret_cast<XRec*>(take(sizeof(XRec) * (size_t)N_pad));
    c.yrec = reinterpret_cast<YRec*>(take(sizeof(YRec) * (size_t)M_pad));
    c.lwx = reinterpret_cast<float*>(take(sizeof(float) * (size_t)N));
    c.lwy = reinterpret_cast<float*>(take(sizeof(float) * (size_t)M));
    double* Lm = reinterpret_cast<double*>(take(2 * sizeof(double)));
    c.counter = reinterpret_cast<int*>(take(8 * sizeof(int)));
    c.err = reinterpret_cast<int*>(take(4 * sizeof(int)));
    c.scratch = c.arena_scratch = reinterpret_cast<double*>(base + off);
    c.scratch_bytes = c.arena_scratch_bytes = kNoAllocScratchBytes - off;
    // partial sums: at most (source blocks + 4 items per resident block) x 8 doubles; check the
    // worst case (32 resident blocks per SM) so the launch below can never ask for more
    const int BI = var.shape.ipt * var.shape.nt;
    const size_t worst_items = (size_t)(N_pad / BI + 1) + (size_t)4 * c.num_sms * 32;
    if (worst_items * 8 * sizeof(double) > c.scratch_bytes)
        return set_error(DUGMA_ERR_STATE, "energy_grad_noalloc: scratch layout does not fit");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DUGMA_CK(cudaMemsetAsync(c.err, 0, 4 * sizeof(int), s));   // the error word must start at zero
    noalloc_max_log2_kernel<<<1, 256, 0, s>>>(det_x, N, Lm);
    noalloc_max_log2_kernel<<<1, 256, 0, s>>>(det_y, M, Lm + 1);
    const int g = std::min((std::max(N, M) + 255) / 256, c.num_sms * 4);
    noalloc_norm_log2_kernel<<<g, 256, 0, s>>>(det_x, N, Lm, c.lwx);
    noalloc_norm_log2_kernel<<<g, 256, 0, s>>>(det_y, M, Lm + 1, c.lwy);
    DUGMA_CK(cudaGetLastError());
    DUGMA_RET(launch_prologue(c, pose_dev, 0, s));   // c.yp32 is null: no nearest-neighbour records
    const int nv = 1 + (D == 3 ? 6 : 3);
    DUGMA_RET(launch_pair_variant(c, var.fn, var.shape, c.xrec, c.yrec, (size_t)M_pad, nv, 0.0, pose_dev, 0, N,
                                  out_dev, nullptr, nullptr, 0, nullptr, s));
    noalloc_scale_kernel<<<1, 32, 0, s>>>(out_dev, nv, Lm + 1);
    DUGMA_CK(cudaGetLastError());
    return DUGMA_OK;
}

namespace dugma {
}  // namespace dugma

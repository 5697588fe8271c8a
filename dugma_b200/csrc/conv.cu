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
// and contracts them with St_x once per source.  Per pair (3D): 44 FP32 for N~ and 20 for
// the moments, 2 SFU (rsqrt, ex2).
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
__device__ __noinline__ bool conv_pair_f64(const float* xi, const float* sxi, float4 v0, float4 v1,
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
            acc[0] += c0 * E64[ii];
            if (!GRAD) continue;
            double S[3][3] = {}, UUm[3][3] = {}, Am[3][3] = {};
#pragma unroll
            for (int q = 0; q < NS; ++q) {
                const int ra = Sym<D>::a(q), rb = Sym<D>::b(q);
                S[ra][rb] = S[rb][ra] = (double)sx[ii][q];
                UUm[ra][rb] = UUm[rb][ra] = UUr[ii][q];
                Am[ra][rb] = Am[rb][ra] = Ar[ii][q];
            }
            double u[3], p[3];
#pragma unroll
            for (int q = 0; q < D; ++q) {
                u[q] = Ur[ii][q] / lam;        // sum N~ S^-1 d
                p[q] = (double)x[ii][q] - t[q];
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
                for (int q = 0; q < D; ++q)
                    a.dx_part[((size_t)jc * rows + (row[ii] - a.i0)) * D + q] = -c0 * u[q];
            }
        }
    }
};

template <class Body, int NT, int TJ>
__global__ void __launch_bounds__(NT) conv_kernel(PairArgs a)
{
    Body body;
    run_pairs<Body, NT, TJ, 4>(a, body);
}

using KernelFn = void (*)(PairArgs);
int launch_pair_variant(Context& c, KernelFn fn, const KernelShape& sh, const void* xrec, const void* yrec,
                        size_t yrec_size, int nv, double Lmax, const double* pose_dev, int i0, int i1,
                        double* out_dev, double* dEdx_dev, double** h_part, int h_width, int* n_jc_out,
                        cudaStream_t s);

int conv_launch(Context& c, const double* pose_dev, bool grad, int i0, int i1, double* out_dev, double* dEdx_dev,
                cudaStream_t s, const KernelShape*)
{
    const int n = std::max(c.M_pad, c.N_pad);
    const int g = std::min((n + 255) / 256, c.num_sms * 4);
    if (c.D == 3)
        conv_prologue_kernel<3><<<g, 256, 0, s>>>(pose_dev, c.y, c.ycov, c.M, c.M_pad, c.yrec, c.x, c.xcov, c.N,
                                                  c.N_pad, c.xrec);
    else
        conv_prologue_kernel<2><<<g, 256, 0, s>>>(pose_dev, c.y, c.ycov, c.M, c.M_pad, c.yrec, c.x, c.xcov, c.N,
                                                  c.N_pad, c.xrec);
    DUGMA_CK(cudaGetLastError());
    const KernelShape sh{grad ? 1 : 2, 128, 64};
    KernelFn fn;
    if (c.D == 3)
        fn = grad ? conv_kernel<ConvBody<3, 1, true>, 128, 64> : conv_kernel<ConvBody<3, 2, false>, 128, 64>;
    else
        fn = grad ? conv_kernel<ConvBody<2, 1, true>, 128, 64> : conv_kernel<ConvBody<2, 2, false>, 128, 64>;
    const int nv = grad ? 1 + (c.D == 3 ? 6 : 3) : 1;
    return launch_pair_variant(c, fn, sh, c.xrec, c.yrec, (size_t)c.M_pad, nv, c.cscale, pose_dev, i0, i1, out_dev,
                               grad ? dEdx_dev : nullptr, nullptr, 0, nullptr, s);
}

}  // namespace dugma

// coef.cu -- surrogate coefficients (the compi plugin) by moment accumulation.
//
// The reference accumulates 637 (3D) / 45 (2D) per-pair coefficient terms with FP64
// shared-memory atomics (compi.cu:632-3407, 96-460).  Every one of those terms is a
// product of a source-side factor and a target-side factor (see gen/gen_coef.py), so
//   A_k = sum_ij P_ij c_k(x_i, B_i, y'_j, C'_j)
// is a fixed linear combination of the moments
//   M2[m,a,b] = sum_i B_i[m] f_i[a] H2_i[b],   H2_i = sum_j P_ij g(y'_j)   (pass A, source-stationary)
//   M1[m,a,b] = sum_j C'_j[m] g_j[a] H1_j[b],  H1_j = sum_i P_ij f(x_i)    (pass B, target-stationary)
// with f, g the degree <= 2 monomials of a point (10 in 3D, 6 in 2D).  Per pair this is
// the P computation plus 10 multiply-adds in each pass instead of 637 atomics.
#include <cmath>

#include <mutex>
#include <vector>

#include "coef_map.h"
#include "context.hpp"
#include "pairs.cuh"
#include "umma.cuh"

namespace dugma {

template <int D> struct Feat { static constexpr int N = 1 + D + Sym<D>::N; };

template <int D>
__host__ __device__ inline void monomials(const double* p, double* f)
{
    f[0] = 1.0;
    for (int a = 0; a < D; ++a) f[1 + a] = p[a];
    for (int k = 0; k < Sym<D>::N; ++k) f[1 + D + k] = p[Sym<D>::a(k)] * p[Sym<D>::b(k)];
}

// ---------------------------------------------------------------------------
// Packed form: the streamed side as pair records (256 B, two points per f32x2 operation).
// Field f (0..31) of a Rec256 is the float2 (field f of point 2p, field f of point 2p+1) of
// the Rec128 layout read as 32 floats, with the coordinates (fields 0-2 hi, 4-6 lo) negated
// so that d = (hi_s + f0) + (lo_s + f4) needs only packed adds; field 3 is the log2 weight,
// 8..13 the matrix, 16.. the monomials.  The prologue writes each point's half of its pair
// record next to its Rec128.
// ---------------------------------------------------------------------------
struct __align__(16) Rec256 {
    float4 q[16];   // q[k] = (field 2k even, field 2k odd, field 2k+1 even, field 2k+1 odd)
};

// point j's record r into its half (j & 1) of pair record j / 2
__device__ __forceinline__ void write_pair_half(Rec256* __restrict__ out, int j, const Rec128& r)
{
    const float* a = reinterpret_cast<const float*>(&r);
    float* o = reinterpret_cast<float*>(out + (j >> 1));
    const int h = j & 1;
#pragma unroll
    for (int f = 0; f < 32; ++f) {
        const bool neg = f <= 2 || (f >= 4 && f <= 6);
        o[(f >> 1) * 4 + (f & 1) * 2 + h] = neg ? -a[f] : a[f];
    }
}

// ---------------------------------------------------------------------------
// Records: y side (v0 = y'hi, lv; v1 = y'lo; v2/v3 = k C'_j Horner-packed; g = monomials of y')
//          x side (v0 = x, lw; v1 = 0;     v2/v3 = k B_i Horner-packed;  g = monomials of x)
// ---------------------------------------------------------------------------
// One thread per point: indices [0, M_pad) are the targets, [M_pad, M_pad + N_pad) the sources.
// The pose is pv when use_pv (block 0 then writes it to `pose` for the kernels that follow), else
// read from `pose`.  reset_counter and reset_err (each optional) are zeroed for those kernels.
// CHOL: each matrix as the upper Cholesky factor U' of |k| B (U'^T U' = |k| B; the sources' from
// init's FP64 factor ux of sym(Sigma_x^-1), the targets' of C'_j in FP64 here), so that an exponent is
// lv - |U' d|^2, a sum of squares whose FP32 rounding grows with sqrt(cond B) instead of cond B; the
// records then carry -lv.  !CHOL: k B in the Horner form (off-diagonals doubled) and lv.
template <int D, bool CHOL>
__global__ void coef_prologue_kernel(const PoseBlock pv, int use_pv, double* __restrict__ pose,
                                     const float* __restrict__ y,
                                     const float* __restrict__ yinv, const float* __restrict__ lwy, int M, int M_pad,
                                     Rec128* __restrict__ yr, Rec256* __restrict__ yr2, const float* __restrict__ x,
                                     const float* __restrict__ xinv, const float* __restrict__ lwx, int N, int N_pad,
                                     Rec128* __restrict__ xr, Rec256* __restrict__ xr2, int* __restrict__ reset_counter,
                                     int* __restrict__ reset_err, const double* __restrict__ ux)
{
    pdl_trigger();   // the one-pass kernel may be scheduled now; it waits for this kernel's writes
    constexpr int NS = Sym<D>::N, NF = Feat<D>::N;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (reset_counter) *reset_counter = 0;
        if (reset_err) *reset_err = 0;
        if (use_pv)
#pragma unroll
            for (int k = 0; k < kPoseDoubles; ++k) pose[k] = pv.v[k];
    }
    double R[9], t[3];
#pragma unroll
    for (int k = 0; k < D * D; ++k) R[k] = use_pv ? pv.v[k] : pose[k];
#pragma unroll
    for (int a = 0; a < D; ++a) t[a] = use_pv ? pv.v[kPoseT + a] : pose[kPoseT + a];
    const double s = 1.0 / (use_pv ? pv.v[kPoseSig] : pose[kPoseSig]), ks = K_EXP2 * s, sk = sqrt(-ks);
    const int stride = gridDim.x * blockDim.x;
    for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < M_pad + N_pad; u += stride) {
        if (u >= M_pad) {
            const int i = u - M_pad;
            Rec128 r;
            float xv[3] = {0, 0, 0}, bp[6] = {0, 0, 0, 0, 0, 0};
            double f[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
            float lw = -INFINITY;
            if (i < N) {
                double xd[3] = {0, 0, 0};
                for (int a = 0; a < D; ++a) {
                    xv[a] = x[(size_t)i * D + a];
                    xd[a] = xv[a];
                }
                monomials<D>(xd, f);
                lw = lwx[i];
                if (lw != -INFINITY)
                    for (int k = 0; k < NS; ++k) {
                        if (CHOL) {
                            bp[k] = __double2float_rn(sk * ux[(size_t)i * NS + k]);
                        } else {
                            const int ra = Sym<D>::a(k), rb = Sym<D>::b(k);
                            const double b = 0.5 * ((double)xinv[(size_t)i * D * D + ra + D * rb] +
                                                    (double)xinv[(size_t)i * D * D + rb + D * ra]);
                            bp[k] = __double2float_rn(ks * b * (ra == rb ? 1.0 : 2.0));
                        }
                    }
            }
            r.v0 = make_float4(xv[0], xv[1], xv[2], CHOL ? -lw : lw);
            r.v1 = make_float4(0.f, 0.f, 0.f, 0.f);
            r.v2 = D == 3 ? make_float4(bp[0], bp[1], bp[2], bp[3]) : make_float4(bp[0], bp[1], bp[2], 0.f);
            r.v3 = D == 3 ? make_float4(bp[4], bp[5], 0.f, 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
            for (int q = 0; q < 16; ++q) r.g[q] = q < NF ? __double2float_rn(f[q]) : 0.f;
            xr[i] = r;
            write_pair_half(xr2, i, r);
            continue;
        }
        const int j = u;
        Rec128 r;
        float hi[3] = {0, 0, 0}, lo[3] = {0, 0, 0}, cp[6] = {0, 0, 0, 0, 0, 0};
        double g[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        float lv = -INFINITY;
        if (j < M) {
            double yp[3] = {0, 0, 0};
            for (int a = 0; a < D; ++a) {
                double v = R[a] * (double)y[(size_t)j * D] + R[a + D] * (double)y[(size_t)j * D + 1];
                if (D == 3) v = v + R[a + 6] * (double)y[(size_t)j * D + 2];
                yp[a] = v + t[a];
                hi[a] = __double2float_rn(yp[a]);
                lo[a] = __double2float_rn(yp[a] - (double)hi[a]);
            }
            monomials<D>(yp, g);
            lv = lwy[j];
            if (lv != -INFINITY) {
                double A[3][3], T[3][3];
                for (int r0 = 0; r0 < D; ++r0)
                    for (int c0 = 0; c0 < D; ++c0)
                        A[r0][c0] = 0.5 * ((double)yinv[(size_t)j * D * D + r0 + D * c0] +
                                           (double)yinv[(size_t)j * D * D + c0 + D * r0]);
                for (int r0 = 0; r0 < D; ++r0)
                    for (int c0 = 0; c0 < D; ++c0) {
                        double acc = 0;
                        for (int k = 0; k < D; ++k) acc += A[r0][k] * R[c0 + D * k];
                        T[r0][c0] = acc;
                    }
                double pk[6];
                for (int k = 0; k < NS; ++k) {
                    const int ra = Sym<D>::a(k), rb = Sym<D>::b(k);
                    double acc = 0;
                    for (int q = 0; q < D; ++q) acc += R[ra + D * q] * T[q][rb];
                    pk[k] = acc;
                    cp[k] = __double2float_rn(ks * acc * (ra == rb ? 1.0 : 2.0));
                }
                if (CHOL) {
                    // C'_j has the eigenvalues of sym(Sigma_y_j^-1), which init found positive definite;
                    // a pivot the rotation's rounding pushed under chol_upper's bound gets 1e-12 of the
                    // trace added
                    double u[6];
                    if (!chol_upper<D>(pk, u)) {
                        const double tr = pk[0] + pk[1] + (D == 3 ? pk[2] : 0.0);
                        for (int a = 0; a < D; ++a) pk[a] += 1e-12 * tr;
                        chol_upper<D>(pk, u);
                    }
                    for (int k = 0; k < NS; ++k) cp[k] = __double2float_rn(sk * u[k]);
                }
            }
        }
        r.v0 = make_float4(hi[0], hi[1], hi[2], CHOL ? -lv : lv);
        r.v1 = make_float4(lo[0], lo[1], lo[2], 0.f);
        r.v2 = D == 3 ? make_float4(cp[0], cp[1], cp[2], cp[3]) : make_float4(cp[0], cp[1], cp[2], 0.f);
        r.v3 = D == 3 ? make_float4(cp[4], cp[5], 0.f, 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
        for (int q = 0; q < 16; ++q) r.g[q] = q < NF ? __double2float_rn(g[q]) : 0.f;
        yr[j] = r;
        write_pair_half(yr2, j, r);
    }
}

__device__ __forceinline__ float2 fld256(const Rec256& r, int f)
{
    const float4 q = r.q[f >> 1];
    return (f & 1) ? make_float2(q.z, q.w) : make_float2(q.x, q.y);
}

// packed Horner quadratic form (k-scaled, off-diagonals doubled) plus an offset
template <int D>
__device__ __forceinline__ float2 qform2(const float2* m, const float2* d, float2 off)
{
    if (D == 3) {
        const float2 g0 = ffma2(m[4], d[2], ffma2(m[3], d[1], fmul2(m[0], d[0])));
        const float2 g1 = ffma2(m[5], d[2], fmul2(m[1], d[1]));
        const float2 g2 = fmul2(m[2], d[2]);
        return ffma2(d[0], g0, ffma2(d[1], g1, ffma2(d[2], g2, off)));
    } else {
        const float2 g0 = ffma2(m[2], d[1], fmul2(m[0], d[0]));
        const float2 g1 = fmul2(m[1], d[1]);
        return ffma2(d[0], g0, ffma2(d[1], g1, off));
    }
}

// 2^(exponent) of a pair for one side's matrix record m: !CHOL the Horner form, exponent
// d^T (k B) d + lv; CHOL the Cholesky form with z = U' d (the same 6 operations as the Horner form's
// first step), exponent -(|z|^2 + nlv) with nlv = -lv from the record (9 FP32 operations either way).
template <int D, bool CHOL>
__device__ __forceinline__ float2 pexp2(const float2* m, const float2* d, float2 lv)
{
    if (!CHOL) {
        const float2 t = qform2<D>(m, d, lv);
        return make_float2(ex2(t.x), ex2(t.y));
    }
    float2 m2;
    if (D == 3) {
        const float2 z0 = ffma2(m[4], d[2], ffma2(m[3], d[1], fmul2(m[0], d[0])));
        const float2 z1 = ffma2(m[5], d[2], fmul2(m[1], d[1]));
        const float2 z2 = fmul2(m[2], d[2]);
        m2 = ffma2(z0, z0, ffma2(z1, z1, ffma2(z2, z2, lv)));
    } else {
        const float2 z0 = ffma2(m[2], d[1], fmul2(m[0], d[0]));
        const float2 z1 = fmul2(m[1], d[1]);
        m2 = ffma2(z0, z0, ffma2(z1, z1, lv));
    }
    return make_float2(ex2(-m2.x), ex2(-m2.y));
}

// One body for both passes.  The stationary side keeps (position hi, lo, matrix) in registers,
// duplicated in both halves; the streamed pair record supplies two points' positions,
// matrices, log2 weights and monomials.  H accumulates P * (streamed monomials); the sign of
// d does not matter to the quadratic forms.
// STREAM_LO: the streamed side carries the y' low parts (targets streamed, sources stationary);
// otherwise the stationary side does.  The other side's low part is zero (x is FP32), so d
// needs two packed adds per coordinate instead of three.
template <int D, int IPT_, bool STREAM_LO, bool CHOL>
struct PackedCoefBody {
    using StreamRec = Rec256;
    static constexpr int IPT = IPT_;
    static constexpr int NV = 1;
    static constexpr int NS = Sym<D>::N, NF = Feat<D>::N;
    float2 PH[IPT][D], PL[IPT][D], Mx[IPT][NS];   // stationary point, duplicated in both halves
    float2 h[IPT][NF];
    double H[IPT][NF];
    int row[IPT];
    double G;

    __device__ void setup(const PairArgs& a)
    {
        const double s = 1.0 / a.pose[kPoseSig];
        G = pow(s, (double)D) * exp2(a.Lmax);
    }
    __device__ void load_src(const PairArgs& a, int ii, int i)
    {
        const Rec128* rr = static_cast<const Rec128*>(a.xrec);
        row[ii] = i < a.i_end ? i : -1;
        const Rec128 r = rr[i < a.i_end ? i : 0];
        const bool ok = i < a.i_end;
        const float hv[3] = {r.v0.x, r.v0.y, r.v0.z}, lv[3] = {r.v1.x, r.v1.y, r.v1.z};
        const float mv[6] = {r.v2.x, r.v2.y, r.v2.z, r.v2.w, r.v3.x, r.v3.y};
#pragma unroll
        for (int q = 0; q < D; ++q) {
            const float a0 = ok ? hv[q] : 0.f, a1 = ok ? lv[q] : 0.f;
            PH[ii][q] = make_float2(a0, a0);
            PL[ii][q] = make_float2(a1, a1);
        }
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            const float v = ok ? mv[q] : 0.f;
            Mx[ii][q] = make_float2(v, v);
        }
    }
    __device__ void zero_all()
    {
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii)
#pragma unroll
            for (int q = 0; q < NF; ++q) { h[ii][q] = make_float2(0.f, 0.f); H[ii][q] = 0.0; }
    }
    __device__ __forceinline__ void consume(const Rec256& r, int)
    {
        float2 nh[3], nl[3], ms[6], g[NF];
#pragma unroll
        for (int q = 0; q < D; ++q) { nh[q] = fld256(r, q); nl[q] = fld256(r, 4 + q); }
        const float2 lv = fld256(r, 3);
#pragma unroll
        for (int k = 0; k < NS; ++k) ms[k] = fld256(r, 8 + k);
#pragma unroll
        for (int q = 0; q < NF; ++q) g[q] = fld256(r, 16 + q);
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            // (hi_s - hi_t) + (lo_s - lo_t); hi_s - hi_t is exact for near pairs
            float2 d[3];
#pragma unroll
            for (int q = 0; q < D; ++q) d[q] = fadd2(fadd2(PH[ii][q], nh[q]), STREAM_LO ? nl[q] : PL[ii][q]);
            const float2 p = fadd2(pexp2<D, CHOL>(Mx[ii], d, lv), pexp2<D, CHOL>(ms, d, lv));
#pragma unroll
            for (int q = 0; q < NF; ++q) h[ii][q] = ffma2(p, g[q], h[ii][q]);
        }
    }
    __device__ void fold()
    {
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii)
#pragma unroll
            for (int q = 0; q < NF; ++q) {
                H[ii][q] += (double)h[ii][q].x + (double)h[ii][q].y;
                h[ii][q] = make_float2(0.f, 0.f);
            }
    }
    __device__ void finish(const PairArgs& a, int jc, double (&)[NV])
    {
        const int rows = a.i_end - a.i0;
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            if (row[ii] < 0) continue;
            const double w = (double)a.wx[row[ii]] * G;   // wx: the stationary side's |Sigma|^-1/2
            double* o = a.h_part + ((size_t)jc * rows + (row[ii] - a.i0)) * 16;
#pragma unroll
            for (int q = 0; q < NF; ++q) o[q] = w * H[ii][q];
        }
    }
};

template <class Body, int NT, int TJ, int MINB = 1>
__global__ void __launch_bounds__(NT, MINB) coef_pass_kernel(PairArgs a)
{
    Body body;
    run_pairs<Body, NT, TJ, 4>(a, body);
}

// ---------------------------------------------------------------------------
// Single pass over the pairs for both sides.  A work item is (group of SB source blocks,
// chunk of target tiles); for each source block of its group the block streams the chunk's
// pair records through the bulk-copy ring and, per tile:
//   phase 1: every pair's p = 2^t1 + 2^t2 (target log weight folded in) once, accumulated into
//            the sources' H2 = sum_j p g_j in registers, and written to a shared tile sP;
//   phase 2: warp w sums its quarter of the sources against the tile's targets,
//            T_j = sum_i fw_i p_ij with fw_i = (w_i / 2^Lmax_x) f(x_i), and the warps' partial
//            sums are added in fixed order into the group's H1 rows in FP64.
// H2 is written per (chunk, source), H1 per (group, target), and the moments kernel sums those
// copies in fixed order: the same moments as the two passes, each pair's exponentials computed
// once, and no atomics.
// ---------------------------------------------------------------------------
struct FusedCoefArgs {
    const Rec128* xrec;    // sources: x, lw, k B (Horner), monomials f(x)
    const Rec256* yrec;    // target pair records
    const float* wx;       // |Sigma_x|^-1/2
    const double* pose;
    double Lmax_x, Lmax_y;
    int N, M, n_ib, SB, n_grp, n_jc, jc_tiles, total_tiles;
    double* h2_part;       // [n_jc][N][16]
    double* h1_part;       // [n_grp][M][16]
    int* counter;
    int* err;
};

template <int D>
struct FusedCoefShape {
    static constexpr int IPT = 2, NT = 128, TJ = 16, STAGES = 4;
    static constexpr int FOLD = 4;       // tiles summed in FP32 before each FP64 fold of the sources' sums
    static constexpr int BI = IPT * NT, NW = NT / 32, TT = 2 * TJ;
    static constexpr int NF = Feat<D>::N;          // 10 in 3D, 6 in 2D
    static constexpr int NP = NF / 2;              // monomial pairs (one f32x2 operand each)
    static constexpr int SF = (NF + 3) / 4 * 4;    // sF row: the monomials padded to whole float4s
    static constexpr int SPS = TT + 2;   // sP row stride in floats: even (float2 stores), rows skewed across banks
    static constexpr size_t kOffBars = (size_t)STAGES * TJ * sizeof(Rec256);
    static constexpr size_t kOffP = kOffBars + 128;
    static constexpr size_t kOffF = kOffP + sizeof(float) * BI * SPS;
    static constexpr size_t kOffT = kOffF + sizeof(float) * BI * SF;
    static constexpr size_t kBytes = kOffT + sizeof(float) * NW * TT * (NF + 1) + 16;
};

template <int D, bool CHOL>
__global__ void __launch_bounds__(128, 3) coef_fused_kernel(FusedCoefArgs a)
{
    using S = FusedCoefShape<D>;
    constexpr int IPT = S::IPT, NT = S::NT, TJ = S::TJ, STAGES = S::STAGES, BI = S::BI, NW = S::NW, TT = S::TT;
    constexpr int NF = S::NF, NP = S::NP, SF = S::SF, SPS = S::SPS, NS = Sym<D>::N;
    static_assert(TT == 32, "phase 2 maps a lane of each half-warp to two targets of a tile");
    static_assert(BI % (2 * NW) == 0 && NF % 2 == 0, "sources split evenly over the half-warps, monomials in pairs");
    constexpr uint32_t kTileBytes = TJ * sizeof(Rec256);
    extern __shared__ __align__(128) unsigned char smem[];
    Rec256(*ybuf)[TJ] = reinterpret_cast<Rec256(*)[TJ]>(smem);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + S::kOffBars);
    int* s_item = reinterpret_cast<int*>(smem + S::kOffBars + 64);
    float(*sP)[SPS] = reinterpret_cast<float(*)[SPS]>(smem + S::kOffP);
    // fw rows: the NF monomials of a source, padded to whole float4s
    float(*sF)[SF] = reinterpret_cast<float(*)[SF]>(smem + S::kOffF);
    float(*sT)[TT][NF + 1] = reinterpret_cast<float(*)[TT][NF + 1]>(smem + S::kOffT);

    // a dependent of the coefficient prologue (records, pose, zeroed counter), and the moments
    // kernel a dependent of this one
    pdl_trigger();
    pdl_wait();
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        for (int st = 0; st < STAGES; ++st) mbar_init(&bars[st], 1);
        mbar_fence_init();
    }
    __syncthreads();
    const double sgm = 1.0 / a.pose[kPoseSig];
    const double Gs = pow(sgm, (double)D);
    const double G2 = Gs * exp2(a.Lmax_y);               // H2_i = w_i G2 sum_j p g_j
    const double G1 = Gs * exp2(a.Lmax_x + a.Lmax_y);    // H1_j = G1 sum_i fw_i p_ij
    const double inv_wmax = exp2(-a.Lmax_x);
    const Rec256* yg = a.yrec;
    const int n_items = a.n_grp * a.n_jc;
    uint32_t tcount = 0;
    for (;;) {
        if (tid == 0) *s_item = atomicAdd(a.counter, 1);
        __syncthreads();
        const int item = *s_item;
        if (item >= n_items) break;
        const int grp = item % a.n_grp, jc = item / a.n_grp;
        const int tile0 = jc * a.jc_tiles;
        const int ntiles = min(a.jc_tiles, a.total_tiles - tile0);
        for (int sb = 0; sb < a.SB; ++sb) {
            const int ib = grp * a.SB + sb;
            if (ib >= a.n_ib) break;
            if (tid == 0)
                for (int k = 0; k < STAGES && k < ntiles; ++k) {
                    const int st = (tcount + k) % STAGES;
                    mbar_arrive_expect_tx(&bars[st], kTileBytes);
                    bulk_g2s(&ybuf[st][0], yg + (size_t)(tile0 + k) * TJ, kTileBytes, &bars[st]);
                }
            // the block's sources: position, k B (Horner), and fw = (w / 2^Lmax_x) f(x) for phase 2
            float2 PH[IPT][3], Mx[IPT][6], h[IPT][NF];
            double H[IPT][NF];
            int row[IPT];
#pragma unroll
            for (int ii = 0; ii < IPT; ++ii) {
                const int il = ii * NT + tid, i = ib * BI + il;
                const bool ok = i < a.N;
                row[ii] = ok ? i : -1;
                const Rec128 r = a.xrec[ok ? i : 0];
                const float hv[3] = {r.v0.x, r.v0.y, r.v0.z};
                const float mv[6] = {r.v2.x, r.v2.y, r.v2.z, r.v2.w, r.v3.x, r.v3.y};
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    const float v = ok && q < D ? hv[q] : 0.f;
                    PH[ii][q] = make_float2(v, v);
                }
#pragma unroll
                for (int q = 0; q < 6; ++q) {
                    const float v = ok && q < NS ? mv[q] : 0.f;
                    Mx[ii][q] = make_float2(v, v);
                }
                const double ws = ok ? (double)a.wx[i] * inv_wmax : 0.0;
#pragma unroll
                for (int q = 0; q < SF; ++q) sF[il][q] = q < NF ? __double2float_rn(ws * (double)r.g[q]) : 0.f;
#pragma unroll
                for (int q = 0; q < NF; ++q) {
                    h[ii][q] = make_float2(0.f, 0.f);
                    H[ii][q] = 0.0;
                }
            }
            constexpr int NE = (TT * NF + NT - 1) / NT;   // H1 entries of a tile per thread
            for (int k = 0; k < ntiles; ++k) {
                const uint32_t u = tcount + k;
                const int st = u % STAGES;
                const int jt = (tile0 + k) * TT;
                // this thread's H1 entries of the tile as the previous source block left them (the
                // same thread wrote them), loaded now so that the latency hides behind both phases
                double prev[NE];
#pragma unroll
                for (int n = 0; n < NE; ++n) {
                    const int e = tid + n * NT, l2 = e / NF, q = e - l2 * NF;
                    prev[n] = (sb > 0 && e < TT * NF && jt + l2 < a.M)
                                  ? a.h1_part[((size_t)grp * a.M + jt + l2) * 16 + q]
                                  : 0.0;
                }
                const bool ok = mbar_wait_bounded(&bars[st], (u / STAGES) & 1u, a.err);
                const Rec256* yb = ybuf[st];
                // phase 1
#pragma unroll 8
                for (int jj = 0; jj < TJ; ++jj) {
                    const Rec256& r = yb[jj];
                    float2 nh[3], nl[3], ms[6], g[NF];
#pragma unroll
                    for (int q = 0; q < D; ++q) { nh[q] = fld256(r, q); nl[q] = fld256(r, 4 + q); }
                    const float2 lv = fld256(r, 3);
#pragma unroll
                    for (int q = 0; q < NS; ++q) ms[q] = fld256(r, 8 + q);
#pragma unroll
                    for (int q = 0; q < NF; ++q) g[q] = fld256(r, 16 + q);
#pragma unroll
                    for (int ii = 0; ii < IPT; ++ii) {
                        float2 d[3];
#pragma unroll
                        for (int q = 0; q < D; ++q) d[q] = fadd2(fadd2(PH[ii][q], nh[q]), nl[q]);
                        const float2 p = fadd2(pexp2<D, CHOL>(Mx[ii], d, lv), pexp2<D, CHOL>(ms, d, lv));
#pragma unroll
                        for (int q = 0; q < NF; ++q) h[ii][q] = ffma2(p, g[q], h[ii][q]);
                        *reinterpret_cast<float2*>(&sP[ii * NT + tid][2 * jj]) = p;
                    }
                }
                if ((k + 1) % S::FOLD == 0 || k + 1 == ntiles)
#pragma unroll
                    for (int ii = 0; ii < IPT; ++ii)
#pragma unroll
                        for (int q = 0; q < NF; ++q) {
                            H[ii][q] += (double)h[ii][q].x + (double)h[ii][q].y;
                            h[ii][q] = make_float2(0.f, 0.f);
                        }
                if (__syncthreads_or(!ok)) {
                    // a tile never arrived: drain the copies still in flight (bounded), then stop
                    if (tid == 0)
                        for (int q = k; q < ntiles && q < k + STAGES; ++q) {
                            const uint32_t uq = tcount + q;
                            mbar_wait_bounded(&bars[uq % STAGES], (uq / STAGES) & 1u, nullptr);
                        }
                    return;
                }
                if (tid == 0 && k + STAGES < ntiles) {
                    mbar_arrive_expect_tx(&bars[st], kTileBytes);
                    bulk_g2s(&ybuf[st][0], yg + (size_t)(tile0 + k + STAGES) * TJ, kTileBytes, &bars[st]);
                }
                // phase 2: warp `warp` sums its quarter of the sources; lane (sh, tl) owns targets 2 tl and
                // 2 tl + 1 of the tile and takes every other source (parity sh), each f32x2 operation a
                // pair of monomials; the two halves then swap partials so that lane (sh, tl) holds all
                // of the warp's sources for target 2 tl + sh
                {
                    const int sh = lane >> 4, tl = lane & 15;
                    float2 a0[NP], a1[NP];
#pragma unroll
                    for (int q = 0; q < NP; ++q) a0[q] = a1[q] = make_float2(0.f, 0.f);
                    const int ib0 = warp * (BI / NW) + sh;
#pragma unroll 8
                    for (int s2 = 0; s2 < BI / NW / 2; ++s2) {
                        const int i = ib0 + 2 * s2;
                        const float2 pv = *reinterpret_cast<const float2*>(&sP[i][2 * tl]);
                        const float4* f4 = reinterpret_cast<const float4*>(&sF[i][0]);
                        float f[SF];
#pragma unroll
                        for (int v = 0; v < SF / 4; ++v) {
                            const float4 fv = f4[v];
                            f[4 * v] = fv.x;
                            f[4 * v + 1] = fv.y;
                            f[4 * v + 2] = fv.z;
                            f[4 * v + 3] = fv.w;
                        }
                        const float2 p0 = make_float2(pv.x, pv.x), p1 = make_float2(pv.y, pv.y);
#pragma unroll
                        for (int q = 0; q < NP; ++q) {
                            const float2 fq = make_float2(f[2 * q], f[2 * q + 1]);
                            a0[q] = ffma2(p0, fq, a0[q]);
                            a1[q] = ffma2(p1, fq, a1[q]);
                        }
                    }
#pragma unroll
                    for (int q = 0; q < NP; ++q) {
                        const float2 give = sh ? a0[q] : a1[q];
                        float2 keep = sh ? a1[q] : a0[q];
                        keep.x += __shfl_xor_sync(0xffffffffu, give.x, 16);
                        keep.y += __shfl_xor_sync(0xffffffffu, give.y, 16);
                        sT[warp][2 * tl + sh][2 * q] = keep.x;
                        sT[warp][2 * tl + sh][2 * q + 1] = keep.y;
                    }
                }
                __syncthreads();
                // the warps' partials in fixed order, into the group's H1 rows (FP64)
#pragma unroll
                for (int n = 0; n < NE; ++n) {
                    const int e = tid + n * NT, l2 = e / NF, q = e - l2 * NF;
                    if (e >= TT * NF || jt + l2 >= a.M) continue;
                    float sum = sT[0][l2][q];
#pragma unroll
                    for (int w2 = 1; w2 < NW; ++w2) sum += sT[w2][l2][q];
                    a.h1_part[((size_t)grp * a.M + jt + l2) * 16 + q] = prev[n] + G1 * (double)sum;
                }
            }
            tcount += ntiles;
#pragma unroll
            for (int ii = 0; ii < IPT; ++ii) {
                if (row[ii] < 0) continue;
                const double w = (double)a.wx[row[ii]] * G2;
                double* o = a.h2_part + ((size_t)jc * a.N + row[ii]) * 16;
#pragma unroll
                for (int q = 0; q < NF; ++q) o[q] = w * H[ii][q];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// The one pass with the source-side sums on the tensor cores.  H2_i = sum_j p_ij g_j is, per
// tile, the product P (sources x 32 targets) G (32 targets x monomials): each thread writes its
// source's p into tensor memory (TMEM) as the A operand, the block writes the tile's monomials
// into shared memory as the B operand, and one thread issues tcgen05.mma (kind::tf32, M = 128
// sources, K = 8 targets) into FP32 accumulators in TMEM, folded into FP64 every FOLD tiles.
// FP32 accuracy from TF32 operands by the three-term split P G ~ Ph Gh + Pl Gh + Ph Gl (h = the
// value rounded to TF32, l = the remainder rounded to TF32): B = [Gh | Gl] (N = 32 columns) takes
// Ph into D columns 0-15 and 16-31 in one MMA, and Pl x Gh (N = 16) adds into columns 0-15.
// The FP32 pipe keeps the exponents and the target-side sums: 36 of the 45 lane operations a
// pair costs in the FMA-only kernel (coef_fused_kernel).  Measured on the B200 at 64K x 64K it
// is the slower of the two (10.5 ms against 7.8 ms; 11.1 ms with IPT 2, not built), so it is
// the opt-in one: every pair still issues 46 instructions against 35.6 -- the TF32 split (4 integer
// operations and a subtraction), the TMEM stores and MMA synchronisation, and at one source per
// thread (four blocks' TMEM per SM) twice the pair-record loads -- more than the 5 packed FMAs per
// pair it takes off the FP32 pipe, at the same 52 % issue rate.
// IPT sources per thread, 128 threads: M-block ii holds the block's sources 128 ii .. 128 ii + 127,
// thread tid their row tid (warp w reaches TMEM lanes 32 w .. 32 w + 31, its own rows).  TMEM per
// M-block: 32 + 32 A columns (Ph, Pl of the tile) and 32 D columns; 128 (IPT 1) or 256 (IPT 2)
// columns per block, so 4 or 2 blocks share an SM's 512.  The MMAs of k-step s (targets 8s..8s+7)
// commit to mbarrier s: the next tile's p for those targets overwrites the A columns once they
// completed.  Phase 2 (target-side sums) runs per warp over the warp's own sources, so only the
// MMA issuer waits for the block (a named barrier) between the phases.
// ---------------------------------------------------------------------------
template <int D, int IPT_>
struct TcCoefShape {
    static constexpr int IPT = IPT_, NT = 128, TJ = 16, STAGES = 4;
    static constexpr int FOLD = 4;                   // tiles accumulated in TMEM before each FP64 fold
    static constexpr int BI = IPT * NT, NW = NT / 32, TT = 2 * TJ;
    static constexpr int KS = TT / 8;                // MMA k-steps per tile
    static constexpr int NG = 16;                    // the monomials, padded; B holds hi and lo: 2 NG columns
    static constexpr int NF = Feat<D>::N, NP = NF / 2, SF = (NF + 3) / 4 * 4, SPS = TT + 2;
    static constexpr uint32_t kCols = IPT == 1 ? 128 : 256;   // TMEM columns allocated
    static constexpr uint32_t kColD = IPT * 2 * TT;            // first accumulator column
    static constexpr int kPerSM = 512 / kCols;                 // blocks that fit an SM's TMEM
    static constexpr int kGFloats = TT * 2 * NG;               // one B operand buffer
    static constexpr size_t kOffBars = (size_t)STAGES * TJ * sizeof(Rec256);
    static constexpr size_t kOffG = kOffBars + 128;            // [2 buffers][kGFloats]
    static constexpr size_t kOffP = kOffG + sizeof(float) * 2 * kGFloats;
    static constexpr size_t kOffF = kOffP + sizeof(float) * BI * SPS;
    static constexpr size_t kOffT = kOffF + sizeof(float) * BI * SF;
    static constexpr size_t kUsed = kOffT + sizeof(float) * NW * TT * (NF + 1) + 16;
    // shared memory per block such that no more blocks fit an SM than its TMEM holds
    static constexpr size_t kBytes = kUsed > (232448 / (kPerSM + 1) + 1024) ? kUsed : 232448 / (kPerSM + 1) + 1024;
    static_assert(IPT * (2 * TT + 2 * NG) <= (int)kCols, "TMEM columns");
    static_assert(NF <= NG && TT % 8 == 0 && NW == 4, "MMA shape");
    static_assert(kBytes * kPerSM <= 232448, "shared memory");
};

template <int D, int IPT, bool CHOL>
__global__ void __launch_bounds__(128, 4 / IPT) coef_tc_kernel(FusedCoefArgs a)
{
    using S = TcCoefShape<D, IPT>;
    constexpr int NT = S::NT, TJ = S::TJ, STAGES = S::STAGES, BI = S::BI, NW = S::NW, TT = S::TT;
    constexpr int NF = S::NF, NP = S::NP, SF = S::SF, SPS = S::SPS, NS = Sym<D>::N, KS = S::KS, NG = S::NG;
    static_assert(TT == 32, "phase 2 maps a lane of each half-warp to two targets of a tile");
    static_assert(NF % 2 == 0, "monomials in pairs");
    constexpr uint32_t kTileBytes = TJ * sizeof(Rec256);
    constexpr uint32_t kIdescHL = idesc_tf32(128, 2 * NG), kIdescL = idesc_tf32(128, NG);
    extern __shared__ __align__(128) unsigned char smem[];
    Rec256(*ybuf)[TJ] = reinterpret_cast<Rec256(*)[TJ]>(smem);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + S::kOffBars);   // [0, STAGES): ring; then KS MMA bars
    uint64_t* mbars = bars + STAGES;
    int* s_item = reinterpret_cast<int*>(smem + S::kOffBars + 96);
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(smem + S::kOffBars + 100);
    float* sG = reinterpret_cast<float*>(smem + S::kOffG);
    float(*sP)[SPS] = reinterpret_cast<float(*)[SPS]>(smem + S::kOffP);
    float(*sF)[SF] = reinterpret_cast<float(*)[SF]>(smem + S::kOffF);
    float(*sT)[TT][NF + 1] = reinterpret_cast<float(*)[TT][NF + 1]>(smem + S::kOffT);

    pdl_trigger();   // as in coef_fused_kernel
    pdl_wait();
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (warp == 0) tmem_alloc(s_tmem, S::kCols);
    if (tid == 32) {
        for (int st = 0; st < STAGES + KS; ++st) mbar_init(&bars[st], 1);
        mbar_fence_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = *s_tmem;
    const uint32_t tlane = 32u * warp;   // this warp's TMEM lanes (its rows of every M-block)
    const double sgm = 1.0 / a.pose[kPoseSig];
    const double Gs = pow(sgm, (double)D);
    const double G2 = Gs * exp2(a.Lmax_y);
    const double G1 = Gs * exp2(a.Lmax_x + a.Lmax_y);
    const double inv_wmax = exp2(-a.Lmax_x);
    const Rec256* yg = a.yrec;
    const int n_items = a.n_grp * a.n_jc;
    uint32_t tcount = 0;   // tiles this block has run (ring and MMA barrier phases)
    int last_issued = -1;  // the last tile whose MMAs were issued
    bool failed = false;
    for (;;) {
        if (tid == 0) *s_item = atomicAdd(a.counter, 1);
        __syncthreads();
        const int item = *s_item;
        if (item >= n_items) break;
        const int grp = item % a.n_grp, jc = item / a.n_grp;
        const int tile0 = jc * a.jc_tiles;
        const int ntiles = min(a.jc_tiles, a.total_tiles - tile0);
        for (int sb = 0; sb < a.SB; ++sb) {
            const int ib = grp * a.SB + sb;
            if (ib >= a.n_ib) break;
            if (tid == 0)
                for (int k = 0; k < STAGES && k < ntiles; ++k) {
                    const int st = (tcount + k) % STAGES;
                    mbar_arrive_expect_tx(&bars[st], kTileBytes);
                    bulk_g2s(&ybuf[st][0], yg + (size_t)(tile0 + k) * TJ, kTileBytes, &bars[st]);
                }
            float2 PH[IPT][3], Mx[IPT][6];
            double H[IPT][NF];
            int row[IPT];
#pragma unroll
            for (int ii = 0; ii < IPT; ++ii) {
                const int il = ii * NT + tid, i = ib * BI + il;
                const bool ok = i < a.N;
                row[ii] = ok ? i : -1;
                const Rec128 r = a.xrec[ok ? i : 0];
                const float hv[3] = {r.v0.x, r.v0.y, r.v0.z};
                const float mv[6] = {r.v2.x, r.v2.y, r.v2.z, r.v2.w, r.v3.x, r.v3.y};
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    const float v = ok && q < D ? hv[q] : 0.f;
                    PH[ii][q] = make_float2(v, v);
                }
#pragma unroll
                for (int q = 0; q < 6; ++q) {
                    const float v = ok && q < NS ? mv[q] : 0.f;
                    Mx[ii][q] = make_float2(v, v);
                }
                const double ws = ok ? (double)a.wx[i] * inv_wmax : 0.0;
#pragma unroll
                for (int q = 0; q < SF; ++q) sF[il][q] = q < NF ? __double2float_rn(ws * (double)r.g[q]) : 0.f;
#pragma unroll
                for (int q = 0; q < NF; ++q) H[ii][q] = 0.0;
            }
            constexpr int NE = (TT * NF + NT - 1) / NT;   // H1 entries of a tile per thread
            for (int k = 0; k < ntiles; ++k) {
                const uint32_t u = tcount + k;
                const int st = u % STAGES;
                const int jt = (tile0 + k) * TT;
                // this thread's H1 entries of the tile as the previous source block left them
                double prev[NE];
#pragma unroll
                for (int n = 0; n < NE; ++n) {
                    const int e = tid + n * NT, l2 = e / NF, q = e - l2 * NF;
                    prev[n] = (sb > 0 && e < TT * NF && jt + l2 < a.M)
                                  ? a.h1_part[((size_t)grp * a.M + jt + l2) * 16 + q]
                                  : 0.0;
                }
                bool ok = mbar_wait_bounded(&bars[st], (u / STAGES) & 1u, a.err);
                const Rec256* yb = ybuf[st];
                // B operand: the tile's target monomials zero-padded to NG, TF32 hi in columns 0..NG-1
                // and lo in NG..2NG-1, as core matrices of 8 columns x 4 targets (k-step s starts
                // 256 s floats in; LBO 512 B between target quads, SBO 128 B between column
                // octets).  Buffer u & 1: the MMAs that read it two tiles ago completed before the
                // previous tile's p went to TMEM.
                float* gb = sG + (u & 1) * S::kGFloats;
#pragma unroll
                for (int e = tid; e < TT * NG; e += NT) {
                    const int t = e / NG, n = e - t * NG;
                    float v = 0.f;
                    if (n < NF) {
                        const float2 gv = fld256(yb[t >> 1], 16 + n);
                        v = (t & 1) ? gv.y : gv.x;
                    }
                    const float hi = tf32_rna(v);
                    const int base = ((t >> 2) * 4) * 32 + (t & 3);
                    gb[base + (n >> 3) * 32 + (n & 7) * 4] = hi;
                    gb[base + ((n + NG) >> 3) * 32 + (n & 7) * 4] = tf32_rna(v - hi);
                }
                // phase 1: p for every pair, into sP (phase 2) and TMEM (the MMAs), 4 records per k-step
#pragma unroll
                for (int s = 0; s < KS; ++s) {
                    float2 pq[IPT][4];
#pragma unroll
                    for (int r4 = 0; r4 < 4; ++r4) {
                        const int jj = 4 * s + r4;
                        const Rec256& r = yb[jj];
                        float2 nh[3], nl[3], ms[6];
#pragma unroll
                        for (int q = 0; q < D; ++q) { nh[q] = fld256(r, q); nl[q] = fld256(r, 4 + q); }
                        const float2 lv = fld256(r, 3);
#pragma unroll
                        for (int q = 0; q < NS; ++q) ms[q] = fld256(r, 8 + q);
#pragma unroll
                        for (int ii = 0; ii < IPT; ++ii) {
                            float2 d[3];
#pragma unroll
                            for (int q = 0; q < D; ++q) d[q] = fadd2(fadd2(PH[ii][q], nh[q]), nl[q]);
                            const float2 p = fadd2(pexp2<D, CHOL>(Mx[ii], d, lv), pexp2<D, CHOL>(ms, d, lv));
                            pq[ii][r4] = p;
                            *reinterpret_cast<float2*>(&sP[ii * NT + tid][2 * jj]) = p;
                        }
                    }
                    // the previous tile's k-step s read these A columns
                    if (u > 0) {
                        ok = mbar_wait_bounded(&mbars[s], (u - 1) & 1u, a.err) && ok;
                        tc_fence_after();
                    }
#pragma unroll
                    for (int ii = 0; ii < IPT; ++ii) {
                        float hv[8], lv8[8];
#pragma unroll
                        for (int r4 = 0; r4 < 4; ++r4) {
                            hv[2 * r4] = tf32_rna(pq[ii][r4].x);
                            hv[2 * r4 + 1] = tf32_rna(pq[ii][r4].y);
                            lv8[2 * r4] = tf32_rna(pq[ii][r4].x - hv[2 * r4]);
                            lv8[2 * r4 + 1] = tf32_rna(pq[ii][r4].y - hv[2 * r4 + 1]);
                        }
                        const uint32_t c0 = (uint32_t)ii * 2 * TT + 8 * s;
                        tmem_st8(tmem_addr(tbase, tlane, c0), hv);
                        tmem_st8(tmem_addr(tbase, tlane, c0 + TT), lv8);
                    }
                }
                // fold the accumulators of the last FOLD tiles (complete: k-step KS-1 of the previous
                // tile was waited for above) before this tile's MMAs restart them
                if (k > 0 && k % S::FOLD == 0) {
#pragma unroll
                    for (int ii = 0; ii < IPT; ++ii) {
                        float d0[16], d1[16];
                        const uint32_t cd = S::kColD + 2u * NG * ii;
                        tmem_ld16(tmem_addr(tbase, tlane, cd), d0);
                        tmem_ld16(tmem_addr(tbase, tlane, cd + NG), d1);
                        tmem_wait_ld();
#pragma unroll
                        for (int q = 0; q < NF; ++q) H[ii][q] += (double)d0[q] + (double)d1[q];
                    }
                }
                // the block's p and B operand are in place: the MMA issuer (warp 0) waits for the
                // other warps; they go on to phase 2
                tmem_wait_st();
                fence_proxy_async_smem();
                tc_fence_before();
                if (warp == 0) {
                    named_bar_sync(1, NT);
                    last_issued = (int)u;
                    if (lane == 0) {
                        tc_fence_after();
#pragma unroll 1
                        for (int s = 0; s < KS; ++s) {
                            const uint64_t bd = smem_desc_kmajor(gb + 256 * s, 512, 128);
#pragma unroll
                            for (int ii = 0; ii < IPT; ++ii) {
                                const uint32_t dcol = tbase + S::kColD + 2u * NG * ii;
                                const uint32_t acol = tbase + (uint32_t)ii * 2 * TT + 8u * s;
                                umma_tf32_ts(dcol, acol, bd, kIdescHL, s > 0 || k % S::FOLD != 0);
                                umma_tf32_ts(dcol, acol + TT, bd, kIdescL, true);
                            }
                            umma_commit(&mbars[s]);
                        }
                        if (k + STAGES < ntiles) {
                            mbar_arrive_expect_tx(&bars[st], kTileBytes);
                            bulk_g2s(&ybuf[st][0], yg + (size_t)(tile0 + k + STAGES) * TJ, kTileBytes, &bars[st]);
                        }
                    }
                    __syncwarp();
                } else {
                    named_bar_arrive(1, NT);
                    last_issued = (int)u;
                }
                // phase 2 (the FP32 pipe): warp w sums its own sources (rows 32 w + lane of each
                // M-block); lane (sh, tl) owns targets 2 tl and 2 tl + 1 and takes every other source
                // (parity sh), each f32x2 operation a pair of monomials; the two halves then swap
                // partials so that lane (sh, tl) holds all of the warp's sources for target 2 tl + sh
                {
                    const int sh = lane >> 4, tl = lane & 15;
                    float2 a0[NP], a1[NP];
#pragma unroll
                    for (int q = 0; q < NP; ++q) a0[q] = a1[q] = make_float2(0.f, 0.f);
#pragma unroll 8
                    for (int s2 = 0; s2 < 16 * IPT; ++s2) {
                        const int kk = sh + 2 * s2;
                        const int i = (kk >> 5) * NT + 32 * warp + (kk & 31);
                        const float2 pv = *reinterpret_cast<const float2*>(&sP[i][2 * tl]);
                        const float4* f4 = reinterpret_cast<const float4*>(&sF[i][0]);
                        float f[SF];
#pragma unroll
                        for (int v = 0; v < SF / 4; ++v) {
                            const float4 fv = f4[v];
                            f[4 * v] = fv.x;
                            f[4 * v + 1] = fv.y;
                            f[4 * v + 2] = fv.z;
                            f[4 * v + 3] = fv.w;
                        }
                        const float2 p0 = make_float2(pv.x, pv.x), p1 = make_float2(pv.y, pv.y);
#pragma unroll
                        for (int q = 0; q < NP; ++q) {
                            const float2 fq = make_float2(f[2 * q], f[2 * q + 1]);
                            a0[q] = ffma2(p0, fq, a0[q]);
                            a1[q] = ffma2(p1, fq, a1[q]);
                        }
                    }
#pragma unroll
                    for (int q = 0; q < NP; ++q) {
                        const float2 give = sh ? a0[q] : a1[q];
                        float2 keep = sh ? a1[q] : a0[q];
                        keep.x += __shfl_xor_sync(0xffffffffu, give.x, 16);
                        keep.y += __shfl_xor_sync(0xffffffffu, give.y, 16);
                        sT[warp][2 * tl + sh][2 * q] = keep.x;
                        sT[warp][2 * tl + sh][2 * q + 1] = keep.y;
                    }
                }
                if (__syncthreads_or(!ok)) {
                    // a tile or an MMA never completed: drain the copies still in flight (bounded), stop
                    failed = true;
                    if (tid == 0)
                        for (int q = k; q < ntiles && q <= k + STAGES; ++q) {
                            const uint32_t uq = tcount + q;
                            mbar_wait_bounded(&bars[uq % STAGES], (uq / STAGES) & 1u, nullptr);
                        }
                    break;
                }
                // the warps' partials in fixed order, into the group's H1 rows (FP64)
#pragma unroll
                for (int n = 0; n < NE; ++n) {
                    const int e = tid + n * NT, l2 = e / NF, q = e - l2 * NF;
                    if (e >= TT * NF || jt + l2 >= a.M) continue;
                    float sum = sT[0][l2][q];
#pragma unroll
                    for (int w2 = 1; w2 < NW; ++w2) sum += sT[w2][l2][q];
                    a.h1_part[((size_t)grp * a.M + jt + l2) * 16 + q] = prev[n] + G1 * (double)sum;
                }
            }
            if (failed) break;
            // the last tile's MMAs, then its accumulators into H
            const bool ok = mbar_wait_bounded(&mbars[KS - 1], (uint32_t)last_issued & 1u, a.err);
            tc_fence_after();
            if (ok)
#pragma unroll
                for (int ii = 0; ii < IPT; ++ii) {
                    float d0[16], d1[16];
                    const uint32_t cd = S::kColD + 2u * NG * ii;
                    tmem_ld16(tmem_addr(tbase, tlane, cd), d0);
                    tmem_ld16(tmem_addr(tbase, tlane, cd + NG), d1);
                    tmem_wait_ld();
#pragma unroll
                    for (int q = 0; q < NF; ++q) H[ii][q] += (double)d0[q] + (double)d1[q];
                }
            tcount += ntiles;
            tc_fence_before();
            if (__syncthreads_or(!ok)) {
                failed = true;
                break;
            }
#pragma unroll
            for (int ii = 0; ii < IPT; ++ii) {
                if (row[ii] < 0) continue;
                const double w = (double)a.wx[row[ii]] * G2;
                double* o = a.h2_part + ((size_t)jc * a.N + row[ii]) * 16;
#pragma unroll
                for (int q = 0; q < NF; ++q) o[q] = w * H[ii][q];
            }
        }
        if (failed) break;
    }
    // every MMA this block issued has completed (or its wait gave up and the error word is set):
    // give the TMEM back
    if (failed && tid == 0 && last_issued >= 0)
        mbar_wait_bounded(&mbars[KS - 1], (uint32_t)last_issued & 1u, nullptr);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tbase, S::kCols);
    }
}

__constant__ signed char c_moment3[kNumMoments3D][4];
__constant__ signed char c_moment2[kNumMoments2D][4];
// per side, the indices of its moments in the table (kind 2: side 0, kind 1: side 1)
__constant__ short c_side3[2][kNumMoments3D];
__constant__ short c_side2[2][kNumMoments2D];
__constant__ int c_side_n[2][2];   // [D == 3][side]

constexpr int kMomRows = 64;       // rows staged in shared memory per pass
constexpr int kMomThreads = 320;   // >= moments of one side (168 in 3D); 32 rows x 10 monomials

// One side's input to the moments kernel.
struct MomSide {
    const double* h;      // [copies][n][16]: the per-point H rows, one copy per chunk / group
    int copies, n, nblk;  // rows, and the blocks that share them
    int side;             // 0: sources (x, Sigma_x^-1), 1: targets (y, Sigma_y^-1, posed)
    const float* p;       // the side's points, D per row
    const float* cinv;    // its inverse covariances, D x D per row
    double* out;          // [nblk][moments] block partials
};

// Moments from the per-point H: blockIdx.y picks the side (s0 or s1), and the side's nblk blocks
// split its rows.  Each pass stages kMomRows rows -- H summed over its copies (one (row, feature)
// entry per thread, coalesced), the row's matrix and monomials -- in shared memory; each thread
// then owns one moment of the side and sums its products over the staged rows.  Per-block
// partials in fixed order (deterministic).
template <int D>
__global__ void __launch_bounds__(kMomThreads) moments_kernel(const MomSide s0, const MomSide s1,
                                                              const double* __restrict__ pose)
{
    pdl_trigger();   // in one pass: a dependent of the one-pass kernel, and the reduction one of this kernel
    pdl_wait();
    const MomSide ms = blockIdx.y == 0 ? s0 : s1;
    if ((int)blockIdx.x >= ms.nblk) return;
    const double* __restrict__ hpart = ms.h;
    const float* __restrict__ p = ms.p;
    const float* __restrict__ cinv = ms.cinv;
    double* __restrict__ block_out = ms.out;
    const int n_jc = ms.copies, n = ms.n, side = ms.side;
    constexpr int NS = Sym<D>::N, NF = Feat<D>::N;
    constexpr int NM = D == 3 ? kNumMoments3D : kNumMoments2D;
    const signed char(*tab)[4] = D == 3 ? c_moment3 : c_moment2;
    const short* list = D == 3 ? c_side3[side] : c_side2[side];
    const int nlist = c_side_n[D == 3][side];
    __shared__ double sH[kMomRows][NF];
    __shared__ double sM[kMomRows][NS];
    __shared__ double sF[kMomRows][NF];
    const int my = (int)threadIdx.x < nlist ? list[threadIdx.x] : -1;
    int ia = 0, ib = 0, ic = 0;
    if (my >= 0) {
        ia = tab[my][1];
        ib = tab[my][2];
        ic = tab[my][3];
    }
    double R[9], t[3];
    for (int k = 0; k < D * D; ++k) R[k] = pose[k];
    for (int a = 0; a < D; ++a) t[a] = pose[kPoseT + a];
    const double s = 1.0 / pose[kPoseSig];
    const int per_block = (n + ms.nblk - 1) / ms.nblk;
    const int b0 = blockIdx.x * per_block, b1 = min(n, b0 + per_block);
    double acc = 0.0;
    for (int base = b0; base < b1; base += kMomRows) {
        const int nr = min(kMomRows, b1 - base);
        // one (row, monomial) entry per thread; its copies loaded 16 at a time and added in order
        for (int e = threadIdx.x; e < nr * NF; e += blockDim.x) {
            const int r = e / NF, q = e - r * NF;
            const double* h = hpart + (size_t)(base + r) * 16 + q;
            const size_t cs = (size_t)n * 16;
            double v = 0.0;
            for (int c = 0; c < n_jc; c += 16) {
                double u[16];
#pragma unroll
                for (int k = 0; k < 16; ++k) u[k] = c + k < n_jc ? h[(size_t)(c + k) * cs] : 0.0;
#pragma unroll
                for (int k = 0; k < 16; ++k)
                    if (c + k < n_jc) v += u[k];
            }
            sH[r][q] = v;
        }
        if ((int)threadIdx.x < nr) {
            const int i = base + threadIdx.x;
            double pt[3] = {0, 0, 0}, f[10];
            double A[3][3];
            for (int r0 = 0; r0 < D; ++r0)
                for (int c0 = 0; c0 < D; ++c0)
                    A[r0][c0] = 0.5 * s * ((double)cinv[(size_t)i * D * D + r0 + D * c0] +
                                           (double)cinv[(size_t)i * D * D + c0 + D * r0]);
            if (side == 0) {
                for (int a = 0; a < D; ++a) pt[a] = (double)p[(size_t)i * D + a];
                for (int k = 0; k < NS; ++k) sM[threadIdx.x][k] = A[Sym<D>::a(k)][Sym<D>::b(k)];
            } else {
                for (int a = 0; a < D; ++a) {
                    double v = R[a] * (double)p[(size_t)i * D] + R[a + D] * (double)p[(size_t)i * D + 1];
                    if (D == 3) v = v + R[a + 6] * (double)p[(size_t)i * D + 2];
                    pt[a] = v + t[a];
                }
                double T[3][3];
                for (int r0 = 0; r0 < D; ++r0)
                    for (int c0 = 0; c0 < D; ++c0) {
                        double a2 = 0;
                        for (int k = 0; k < D; ++k) a2 += A[r0][k] * R[c0 + D * k];
                        T[r0][c0] = a2;
                    }
                for (int k = 0; k < NS; ++k) {
                    double a2 = 0;
                    for (int q = 0; q < D; ++q) a2 += R[Sym<D>::a(k) + D * q] * T[q][Sym<D>::b(k)];
                    sM[threadIdx.x][k] = a2;
                }
            }
            monomials<D>(pt, f);
            for (int q = 0; q < NF; ++q) sF[threadIdx.x][q] = f[q];
        }
        __syncthreads();
        if (my >= 0)
            for (int r = 0; r < nr; ++r) acc += sM[r][ia] * sF[r][ib] * sH[r][ic];
        __syncthreads();
    }
    const int kind = side == 0 ? 2 : 1;
    for (int mi = threadIdx.x; mi < NM; mi += blockDim.x)
        if (tab[mi][0] != kind) block_out[(size_t)blockIdx.x * NM + mi] = 0.0;
    if (my >= 0) block_out[(size_t)blockIdx.x * NM + my] = acc;
}

// out[mi] = sum over the na + nb block partials of moment mi; one warp per moment, lanes
// strided over the blocks, fixed-order warp sum.  out[nm] = the device error word, so that one
// copy brings back both; host_out (optional, pinned host memory) receives the same nm + 1 values.
__global__ void moments_reduce_kernel(const double* __restrict__ a, int na, const double* __restrict__ b, int nb,
                                      int nm, double* __restrict__ out, const int* __restrict__ err,
                                      double* __restrict__ host_out)
{
    pdl_wait();   // in one pass: a dependent of the moments kernel
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        out[nm] = (double)*err;
        if (host_out) host_out[nm] = (double)*err;
    }
    const int lane = threadIdx.x & 31;
    const int mi = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (mi >= nm) return;
    double v = 0.0;
    for (int k = lane; k < na; k += 32) v += a[(size_t)k * nm + mi];
    for (int k = lane; k < nb; k += 32) v += b[(size_t)k * nm + mi];
    v = warp_sum(v);
    if (lane == 0) {
        out[mi] = v;
        if (host_out) host_out[mi] = v;
    }
}


static_assert(kNumMoments3D <= kNumMomentsMax && kNumMoments2D <= kNumMomentsMax, "moment count bound");
int num_moments(int D) { return D == 3 ? kNumMoments3D : kNumMoments2D; }

int Context::ensure_coef_records()
{
    if (yrec128) return DUGMA_OK;
    DUGMA_CK(cudaMalloc(&yrec128, sizeof(Rec128) * (size_t)M_pad));
    DUGMA_CK(cudaMalloc(&xrec128, sizeof(Rec128) * (size_t)N_pad));
    // the same records paired for the packed passes (Rec256: two points, same bytes)
    DUGMA_CK(cudaMalloc(&yrec256, sizeof(Rec128) * (size_t)M_pad));
    DUGMA_CK(cudaMalloc(&xrec256, sizeof(Rec128) * (size_t)N_pad));
    // per-block moment partials of both sides: 2 x (2 blocks per SM) x the 3D moment count
    DUGMA_CK(cudaMalloc(&mom_part, sizeof(double) * 2 * (size_t)(2 * num_sms) * kNumMoments3D));
    return DUGMA_OK;
}

// The moment tables and per-side moment lists in constant memory, once per device.
static int upload_moment_tables(int dev)
{
    static std::mutex mu;
    static std::vector<char> done;
    std::lock_guard<std::mutex> lock(mu);
    if (dev < (int)done.size() && done[dev]) return DUGMA_OK;
    short side3[2][kNumMoments3D] = {}, side2[2][kNumMoments2D] = {};
    int cnt[2][2] = {{0, 0}, {0, 0}};
    for (int mi = 0; mi < kNumMoments3D; ++mi)
        for (int sd = 0; sd < 2; ++sd)
            if (kMoment3D[mi][0] == (sd == 0 ? 2 : 1)) side3[sd][cnt[1][sd]++] = (short)mi;
    for (int mi = 0; mi < kNumMoments2D; ++mi)
        for (int sd = 0; sd < 2; ++sd)
            if (kMoment2D[mi][0] == (sd == 0 ? 2 : 1)) side2[sd][cnt[0][sd]++] = (short)mi;
    for (int d = 0; d < 2; ++d)
        for (int sd = 0; sd < 2; ++sd)
            if (cnt[d][sd] > kMomThreads) return set_error(DUGMA_ERR_STATE, "moment table larger than a block");
    DUGMA_CK(cudaMemcpyToSymbol(c_moment3, kMoment3D, sizeof(kMoment3D)));
    DUGMA_CK(cudaMemcpyToSymbol(c_moment2, kMoment2D, sizeof(kMoment2D)));
    DUGMA_CK(cudaMemcpyToSymbol(c_side3, side3, sizeof(side3)));
    DUGMA_CK(cudaMemcpyToSymbol(c_side2, side2, sizeof(side2)));
    DUGMA_CK(cudaMemcpyToSymbol(c_side_n, cnt, sizeof(cnt)));
    if (dev >= (int)done.size()) done.resize(dev + 1, 0);
    done[dev] = 1;
    return DUGMA_OK;
}

// the one-pass kernel's dynamic shared memory limit, once per device; its resident blocks per SM
// (KIND 0: coef_fused_kernel; 1: coef_tc_kernel)
template <int D, int KIND, bool CHOL>
static int fused_coef_setup(int dev, int* per_sm)
{
    static std::mutex mu;
    static std::vector<int> blocks;
    std::lock_guard<std::mutex> lock(mu);
    if (dev < (int)blocks.size() && blocks[dev] > 0) {
        *per_sm = blocks[dev];
        return DUGMA_OK;
    }
    using T = TcCoefShape<D, 1>;
    const void* fn =
        KIND == 0 ? (const void*)coef_fused_kernel<D, CHOL> : (const void*)coef_tc_kernel<D, T::IPT, CHOL>;
    const int nt = KIND == 0 ? FusedCoefShape<D>::NT : T::NT;
    const size_t bytes = KIND == 0 ? FusedCoefShape<D>::kBytes : T::kBytes;
    DUGMA_CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    int nb = 0;
    if (KIND == 0) {
        DUGMA_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, nt, bytes));
    } else {
        // The occupancy query answers 1 for every kernel that allocates TMEM (measured on the B200
        // with driver 580), while the SM runs as many such blocks as their TMEM columns, registers
        // and shared memory allow; the shared memory per block is sized so that no more blocks fit
        // than TMEM holds (a block beyond them would wait in tcgen05.alloc until another exits).
        cudaFuncAttributes fa{};
        DUGMA_CK(cudaFuncGetAttributes(&fa, fn));
        int smem_sm = 0, regs_sm = 0;
        DUGMA_CK(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
        DUGMA_CK(cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev));
        const int regs_warp = (fa.numRegs * 32 + 255) / 256 * 256;   // allocated per warp in units of 256
        const int by_regs = regs_sm / (regs_warp * (nt / 32));
        const int by_smem = smem_sm / (int)(bytes + 1024);            // 1 KB reserved per block
        nb = std::min(T::kPerSM, std::min(by_regs, by_smem));
        if (nb < 1 || by_smem > T::kPerSM)
            return set_error(DUGMA_ERR_STATE,
                             "compi: the tensor-core kernel fits %d blocks per SM by registers and %d by shared "
                             "memory; TMEM holds %d",
                             by_regs, by_smem, T::kPerSM);
    }
    if (dev >= (int)blocks.size()) blocks.resize(dev + 1, 0);
    blocks[dev] = std::max(nb, 1);
    *per_sm = blocks[dev];
    return DUGMA_OK;
}

// Work grid of the one-pass kernel: an item is a group of SB source blocks x a chunk of jc_tiles
// target tiles, and `resident` blocks take items from a counter.  The grid minimises a model of the
// time in units of one block's tile, fitted to B200 timings at 4K, 6K, 16K and 64K points:
//   an item costs its SB * jc_tiles tiles plus 2 per source block (loading the sources, refilling
//   the ring, writing the H2 rows);
//   items <= resident: one round, 1.1 x an item (no balancing: the slowest block decides);
//   more items: items / resident x an item, plus a quarter of an item's tiles for the tail;
//   plus the H2 / H1 copies the moments kernel reads, 128 B a row, at 54 MB per tile unit (HBM
//   bytes in one block's tile time).
// Up to 64 copies of either side and at most 16 GB of them (a full round of items at 3M points
// needs ~42 copies, 16 GB; the model's copy term keeps smaller problems far below).  Against the
// grid it replaced (at most 24 x 24 copies): 64K x 64K 9.5 -> 7.9 ms, 16K 0.58 -> 0.53 ms,
// 4096 x 4096 0.060 -> 0.054 ms.
struct FusedGrid {
    int SB, n_grp, jc_tiles, n_jc;
};

static FusedGrid fused_grid(int n_ib, int total_tiles, int resident, int N, int M)
{
    FusedGrid best{n_ib, 1, total_tiles, 1};
    double best_cost = INFINITY;
    for (int g = 1; g <= std::min(n_ib, 64); ++g) {
        const int SB = (n_ib + g - 1) / g;
        if ((n_ib + SB - 1) / SB != g) continue;   // this grouping is met at another g
        for (int jc = 1; jc <= std::min(total_tiles, 64); ++jc) {
            const int jt = (total_tiles + jc - 1) / jc;
            if ((total_tiles + jt - 1) / jt != jc) continue;
            const double copies = ((double)jc * N + (double)g * M) * 128.0;
            if (copies > 16e9 && (g > 1 || jc > 1)) continue;
            const double items = (double)g * jc, tiles = (double)SB * jt, item = tiles + 2.0 * SB;
            const double cost = (items <= resident ? 1.1 * item : items / resident * item + 0.25 * tiles) + copies / 54e6;
            if (cost < best_cost) {
                best_cost = cost;
                best = {SB, g, jt, jc};
            }
        }
    }
    return best;
}

}  // namespace dugma

extern "C" int dugma_coef_work_grid(int N, int M, int resident, int grid[4])
{
    using dugma::FusedCoefShape;
    if (N < 1 || M < 1 || resident < 1 || !grid)
        return dugma::set_error(DUGMA_ERR_ARG, "coef_work_grid: N, M, resident must be positive");
    const int n_ib = (N + FusedCoefShape<3>::BI - 1) / FusedCoefShape<3>::BI;
    const int M_pad = (M + dugma::kPadJ - 1) / dugma::kPadJ * dugma::kPadJ;
    const int total_tiles = M_pad / 2 / FusedCoefShape<3>::TJ;
    const dugma::FusedGrid g = dugma::fused_grid(n_ib, total_tiles, resident, N, M);
    grid[0] = g.SB;
    grid[1] = g.n_grp;
    grid[2] = g.jc_tiles;
    grid[3] = g.n_jc;
    return DUGMA_OK;
}

namespace dugma {

// Every source row against every target row in one pass (coef_fused_kernel), then the moments
// of both sides from the H2 copies (one per target chunk) and the H1 copies (one per source group).
template <int D, bool CHOL>
static int coef_fused_launch(Context& c, const double* pose_dev, double* moments_dev, cudaStream_t s,
                             double* host_moments)
{
    constexpr int NM = D == 3 ? kNumMoments3D : kNumMoments2D;
    const int kind = c.coef_kernel;
    int per_sm = 1;
    if (kind == 1)
        DUGMA_RET((fused_coef_setup<D, 1, CHOL>(c.dev, &per_sm)));
    else
        DUGMA_RET((fused_coef_setup<D, 0, CHOL>(c.dev, &per_sm)));
    const int resident = c.num_sms * per_sm;
    const int BI = kind == 1 ? TcCoefShape<D, 1>::BI : FusedCoefShape<D>::BI;
    const int n_ib = (c.N + BI - 1) / BI;
    static_assert(TcCoefShape<D, 1>::TJ == FusedCoefShape<D>::TJ, "the kernels stream tiles of the same records");
    const int total_tiles = c.M_pad / 2 / FusedCoefShape<D>::TJ;
    if (c.coef_grid[0] == 0) {
        const FusedGrid fg = fused_grid(n_ib, total_tiles, resident, c.N, c.M);
        c.coef_grid[0] = fg.SB;
        c.coef_grid[1] = fg.n_grp;
        c.coef_grid[2] = fg.jc_tiles;
        c.coef_grid[3] = fg.n_jc;
    }
    const int SB = c.coef_grid[0], n_grp = c.coef_grid[1], jc_tiles = c.coef_grid[2], n_jc = c.coef_grid[3];
    const size_t h2_doubles = (size_t)n_jc * c.N * 16, h1_doubles = (size_t)n_grp * c.M * 16;
    DUGMA_RET(c.ensure_scratch(sizeof(double) * (h2_doubles + h1_doubles)));
    FusedCoefArgs a{};
    a.xrec = c.xrec128;
    a.yrec = static_cast<const Rec256*>(c.yrec256);
    a.wx = c.wx;
    a.pose = pose_dev;
    a.Lmax_x = c.Lmax_x;
    a.Lmax_y = c.Lmax_y;
    a.N = c.N;
    a.M = c.M;
    a.n_ib = n_ib;
    a.SB = SB;
    a.n_grp = n_grp;
    a.n_jc = n_jc;
    a.jc_tiles = jc_tiles;
    a.total_tiles = total_tiles;
    a.h2_part = c.scratch;
    a.h1_part = c.scratch + h2_doubles;
    a.counter = c.counter;
    a.err = c.err;
    // (the coefficient prologue zeroed c.counter)
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
    const int grid = std::min(resident, n_grp * n_jc);
    if (kind == 1)
        DUGMA_CK(launch_dependent(c.pdl, coef_tc_kernel<D, 1, CHOL>, grid, TcCoefShape<D, 1>::NT,
                                  TcCoefShape<D, 1>::kBytes, s, a));
    else
        DUGMA_CK(launch_dependent(c.pdl, coef_fused_kernel<D, CHOL>, grid, FusedCoefShape<D>::NT,
                                  FusedCoefShape<D>::kBytes, s, a));
    DUGMA_CK(cudaGetLastError());
    if (ev1) DUGMA_CK(cudaEventRecord(ev1, s));
    const int nblk = std::max(1, std::min(2 * c.num_sms, (std::max(c.N, c.M) + 31) / 32));
    const int nb0 = std::min(nblk, c.N), nb1 = std::min(nblk, c.M);
    const MomSide m0{a.h2_part, n_jc, c.N, nb0, 0, c.x, c.xinv, c.mom_part};
    const MomSide m1{a.h1_part, n_grp, c.M, nb1, 1, c.y, c.yinv, c.mom_part + (size_t)nblk * NM};
    DUGMA_CK(launch_dependent(c.pdl, moments_kernel<D>, dim3(std::max(nb0, nb1), 2), kMomThreads, 0, s, m0, m1,
                              (const double*)pose_dev));
    DUGMA_CK(launch_dependent(c.pdl, moments_reduce_kernel, (NM + 7) / 8, 256, 0, s, (const double*)c.mom_part, nb0,
                              (const double*)(c.mom_part + (size_t)nblk * NM), nb1, NM, moments_dev,
                              (const int*)c.err, host_moments));
    return DUGMA_OK;
}

template <int D>
static int coef_impl(Context& c, double* pose_dev, double* moments_dev, cudaStream_t s, int i0, int i1, int j0,
                     int j1, const CoefOpts& o)
{
    DUGMA_RET(upload_moment_tables(c.dev));
    DUGMA_RET(c.ensure_coef_records());
    // all rows on both sides: one pass over the pairs; row ranges (sharding): one pass per side
    const bool fused = i0 == 0 && i1 == c.N && j0 == 0 && j1 == c.M && c.fused_coef;
    const int n = c.M_pad + c.N_pad;
    PoseBlock pb{};
    if (o.pose_value)
        for (int k = 0; k < kPoseDoubles; ++k) pb.v[k] = o.pose_value[k];
    // the Cholesky form of every matrix when every weighted point's inverse covariance has a factor,
    // else the Horner form throughout
    const bool chol = c.ux && c.x_indef == 0 && c.y_indef == 0;
    const int pg = std::min((n + 127) / 128, c.num_sms * 8);
    auto prologue = chol ? coef_prologue_kernel<D, true> : coef_prologue_kernel<D, false>;
    prologue<<<pg, 128, 0, s>>>(pb, o.pose_value ? 1 : 0, pose_dev, c.y, c.yinv, c.lwy, c.M, c.M_pad, c.yrec128,
                                static_cast<Rec256*>(c.yrec256), c.x, c.xinv, c.lwx, c.N, c.N_pad, c.xrec128,
                                static_cast<Rec256*>(c.xrec256), fused ? c.counter : nullptr,
                                o.reset_err ? c.err : nullptr, (const double*)c.ux);
    DUGMA_CK(cudaGetLastError());
    if (fused)
        return chol ? coef_fused_launch<D, true>(c, pose_dev, moments_dev, s, o.host_moments)
                    : coef_fused_launch<D, false>(c, pose_dev, moments_dev, s, o.host_moments);
    constexpr int NM = D == 3 ? kNumMoments3D : kNumMoments2D;
    // per side: 2 sources per thread x 128 threads when there are rows enough for two blocks
    // per SM, else 1 x 64 (more blocks for small clouds); items cover at least rows / 8
    // streamed records (128 .. 512), which bounds the per-chunk H partials the moments
    // kernel has to sum to about 8 copies of the rows' H
    // (the packed passes stream pair records: min_chunk counts records of two points)
    auto pass_shape = [&](int rows, int side, KernelFn* fn) {
        const int min_chunk = std::max(64, std::min(256, rows / 16));
        const bool big = rows >= 2 * 256 * c.num_sms;
        if (big)
            *fn = side == 0 ? (chol ? coef_pass_kernel<PackedCoefBody<D, 2, true, true>, 128, 16, 2>
                                    : coef_pass_kernel<PackedCoefBody<D, 2, true, false>, 128, 16, 2>)
                            : (chol ? coef_pass_kernel<PackedCoefBody<D, 2, false, true>, 128, 16, 2>
                                    : coef_pass_kernel<PackedCoefBody<D, 2, false, false>, 128, 16, 2>);
        else
            *fn = side == 0 ? (chol ? coef_pass_kernel<PackedCoefBody<D, 2, true, true>, 64, 16, 6>
                                    : coef_pass_kernel<PackedCoefBody<D, 2, true, false>, 64, 16, 6>)
                            : (chol ? coef_pass_kernel<PackedCoefBody<D, 2, false, true>, 64, 16, 6>
                                    : coef_pass_kernel<PackedCoefBody<D, 2, false, false>, 64, 16, 6>);
        return big ? KernelShape{2, 128, 16, 2, 0, min_chunk} : KernelShape{2, 64, 16, 2, 0, min_chunk};
    };
    // blocks of the moments kernel: about 32 rows each, at most 2 per SM (the partial buffer's size)
    const int nblk = std::max(1, std::min(2 * c.num_sms, (std::max(i1 - i0, j1 - j0) + 31) / 32));
    double* mom = c.mom_part;
    int rc = DUGMA_OK;
    int nb_side[2] = {0, 0};
    for (int side = 0; side < 2 && rc == DUGMA_OK; ++side) {
        // side 0: sources stationary over streamed targets; side 1: the reverse
        double* hp = nullptr;
        int n_jc = 0;
        const Rec128* src = side == 0 ? c.xrec128 : c.yrec128;
        const void* str = side == 0 ? c.yrec256 : c.xrec256;
        const int r0 = side == 0 ? i0 : j0, r1 = side == 0 ? i1 : j1, rows = r1 - r0;
        if (rows <= 0) continue;   // an empty range contributes nothing
        const size_t nstr = (side == 0 ? (size_t)c.M_pad : (size_t)c.N_pad) / 2;
        const double Lmax = side == 0 ? c.Lmax_y : c.Lmax_x;
        KernelFn fn;
        const KernelShape sh = pass_shape(rows, side, &fn);
        // the stationary weights: sources in pass A, targets in pass B
        rc = launch_pair_variant(c, fn, sh, src, str, nstr, 1, Lmax, pose_dev, r0, r1, nullptr, nullptr, &hp, 16,
                                 &n_jc, s, side == 1 ? c.wy : nullptr);
        if (rc != DUGMA_OK) break;
        const int nb = std::min(nblk, rows);
        nb_side[side] = nb;
        const size_t o1 = (size_t)r0 * c.D, o2 = (size_t)r0 * c.D * c.D;
        const MomSide ms = side == 0 ? MomSide{hp, n_jc, rows, nb, 0, c.x + o1, c.xinv + o2, mom}
                                     : MomSide{hp, n_jc, rows, nb, 1, c.y + o1, c.yinv + o2, mom + (size_t)nblk * NM};
        moments_kernel<D><<<dim3(nb, 1), kMomThreads, 0, s>>>(ms, ms, pose_dev);
        if (cudaGetLastError() != cudaSuccess) rc = set_error(DUGMA_ERR_CUDA, "moments kernel launch failed");
    }
    if (rc == DUGMA_OK) {
        moments_reduce_kernel<<<(NM + 7) / 8, 256, 0, s>>>(mom, nb_side[0], mom + (size_t)nblk * NM, nb_side[1], NM,
                                                           moments_dev, c.err, o.host_moments);
        if (cudaGetLastError() != cudaSuccess) rc = set_error(DUGMA_ERR_CUDA, "moment reduction launch failed");
    }
    return rc;
}

int launch_coef(Context& c, double* pose_dev, double* moments_dev, cudaStream_t s, int i0, int i1, int j0, int j1,
                const CoefOpts& opts)
{
    if (i1 < 0) i1 = c.N;
    if (j1 < 0) j1 = c.M;
    return c.D == 3 ? coef_impl<3>(c, pose_dev, moments_dev, s, i0, i1, j0, j1, opts)
                    : coef_impl<2>(c, pose_dev, moments_dev, s, i0, i1, j0, j1, opts);
}

int coef_from_moments(int D, const double* mom, double* out640)
{
    for (int k = 0; k < 640; ++k) out640[k] = 0.0;
    const int K = D == 3 ? kNumCoef3D : kNumCoef2D;
    const int* start = D == 3 ? kCoefStart3D : kCoefStart2D;
    const int* mi = D == 3 ? kCoefMoment3D : kCoefMoment2D;
    const double* wt = D == 3 ? kCoefWeight3D : kCoefWeight2D;
    for (int k = 0; k < K; ++k) {
        double v = 0;
        for (int e = start[k]; e < start[k + 1]; ++e) v += wt[e] * mom[mi[e]];
        out640[k] = v;
    }
    return DUGMA_OK;
}

}  // namespace dugma

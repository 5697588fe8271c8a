// prepare.cu -- init-time and per-evaluation prologue kernels.
//
// This file is compiled with -fmad=false: every FP64 expression below is evaluated
// as written (no fused multiply-add), so the FP32 state written by init and the
// FP32 rounding of y' match the CPU oracle bit for bit.
#include <cmath>
#include <cstdio>
#include <cstring>

#include "context.hpp"

namespace dugma {

// ---------------------------------------------------------------------------
// init: FP64 -> FP32 conversion (init.cu:192-234) fused with the per-point inverse
// covariance and |Sigma|^-1/2 (init.cu:22-190).  The inverse is evaluated in FP64 from
// the FP32-rounded covariance by the adjugate, in the order of the reference's formula,
// and rounded to FP32.  det <= 0: all entries 1e5, weight 0 (init.cu:48-57, 86-100).
// Also writes the packed symmetric FP32 covariance used by the CONV model.
// ---------------------------------------------------------------------------
// ufac (nullable): the upper Cholesky factor of sym(cinv) per point (packed, FP64) for the
// Cholesky-form source records; zero for neglected points, and zero with a count in *indef for
// weighted points whose sym(cinv) is not positive definite.  With ufac null and indef given, only
// the count.
template <int D>
__global__ void init_points_kernel(const double* __restrict__ P, const double* __restrict__ C, int n,
                                   float* __restrict__ p32, float* __restrict__ cinv,
                                   float* __restrict__ w, float* __restrict__ cpack, const double* __restrict__ scale,
                                   int* nonpd, double* __restrict__ ufac, int* indef)
{
    constexpr int NS = Sym<D>::N;
    const double inv_scale = scale[1];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
        for (int a = 0; a < D; ++a) p32[(size_t)i * D + a] = __double2float_rn(P[(size_t)i * D + a]);
        double a_[D * D];
#pragma unroll
        for (int k = 0; k < D * D; ++k) a_[k] = (double)__double2float_rn(C[(size_t)i * D * D + k]);
#pragma unroll
        for (int k = 0; k < NS; ++k) {
            const int ra = Sym<D>::a(k), rb = Sym<D>::b(k);
            cpack[(size_t)i * NS + k] = __double2float_rn(0.5 * (a_[ra + D * rb] + a_[rb + D * ra]) * inv_scale);
        }
        float* o = cinv + (size_t)i * D * D;
        if (D == 3) {
            const double a11 = a_[0], a21 = a_[1], a31 = a_[2], a12 = a_[3], a22 = a_[4], a32 = a_[5],
                         a13 = a_[6], a23 = a_[7], a33 = a_[8];
            const double d = a11 * a22 * a33 - a11 * a23 * a32 - a12 * a21 * a33 + a12 * a23 * a31 +
                             a13 * a21 * a32 - a13 * a22 * a31;
            if (d > 0) {
                o[0] = __double2float_rn((a22 * a33 - a23 * a32) / d);
                o[1] = __double2float_rn(-(a21 * a33 - a23 * a31) / d);
                o[2] = __double2float_rn((a21 * a32 - a22 * a31) / d);
                o[3] = __double2float_rn(-(a12 * a33 - a13 * a32) / d);
                o[4] = __double2float_rn((a11 * a33 - a13 * a31) / d);
                o[5] = __double2float_rn(-(a11 * a32 - a12 * a31) / d);
                o[6] = __double2float_rn((a12 * a23 - a13 * a22) / d);
                o[7] = __double2float_rn(-(a11 * a23 - a13 * a21) / d);
                o[8] = __double2float_rn((a11 * a22 - a12 * a21) / d);
                w[i] = __double2float_rn(sqrt(1.0 / d));
            } else {
#pragma unroll
                for (int k = 0; k < 9; ++k) o[k] = 100000.0f;
                w[i] = 0.0f;
                atomicAdd(nonpd, 1);
            }
        } else {
            const double a1 = a_[0], a2 = a_[1], a3 = a_[2], a4 = a_[3];
            const double d = a1 * a4 - a2 * a3;
            if (d > 0) {
                o[0] = __double2float_rn(a4 / d);
                o[1] = __double2float_rn(-a2 / d);
                o[2] = __double2float_rn(-a3 / d);
                o[3] = __double2float_rn(a1 / d);
                w[i] = __double2float_rn(sqrt(1.0 / d));
            } else {
#pragma unroll
                for (int k = 0; k < 4; ++k) o[k] = 100000.0f;
                w[i] = 0.0f;
                atomicAdd(nonpd, 1);
            }
        }
        if (ufac || indef) {
            double pk[NS], u[NS];
#pragma unroll
            for (int k = 0; k < NS; ++k) {
                const int ra = Sym<D>::a(k), rb = Sym<D>::b(k);
                pk[k] = 0.5 * ((double)o[ra + D * rb] + (double)o[rb + D * ra]);
            }
            const bool ok = chol_upper<D>(pk, u);
            if (w[i] > 0.0f && !ok && indef) atomicAdd(indef, 1);
            if (ufac)
#pragma unroll
                for (int k = 0; k < NS; ++k) ufac[(size_t)i * NS + k] = w[i] > 0.0f ? u[k] : 0.0;
        }
    }
}

// max over the positive weights as float bits (positive floats order like their bit patterns),
// combined across blocks with atomicMax on an int slot zeroed beforehand: order-independent and
// so deterministic.  log2 is monotonic, so log2 of the largest weight is the largest log2.
__global__ void max_weight_kernel(const float* __restrict__ w, int n, int* __restrict__ maxbits)
{
    __shared__ int red[256];
    int m = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (w[i] > 0.0f) m = max(m, __float_as_int(w[i]));
    red[threadIdx.x] = m;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] = max(red[threadIdx.x], red[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0 && red[0] > 0) atomicMax(maxbits, red[0]);
}

// lw_i = log2(w_i) - Lmax with Lmax = log2(largest weight) (-inf when no weight is positive);
// thread 0 also stores Lmax for the host
__global__ void norm_log2_kernel(const float* __restrict__ w, int n, const int* __restrict__ maxbits,
                                 double* __restrict__ Lmax, float* __restrict__ lw)
{
    const int mb = *maxbits;
    const double L = mb > 0 ? log2((double)__int_as_float(mb)) : -INFINITY;
    if (blockIdx.x == 0 && threadIdx.x == 0) *Lmax = L;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        lw[i] = w[i] > 0.0f ? __double2float_rn(log2((double)w[i]) - L) : -INFINITY;
}

// CONV covariance scale: the mean of trace / D over both clouds' covariances (the FP64 staged
// inputs), rounded to a power of two so that dividing by it is exact in FP32.  Per-block sums
// over contiguous slices, then one block over the partials, both in fixed order
// (deterministic).  scale[0] = the scale, scale[1] = its inverse.
__global__ void cov_trace_partial_kernel(const double* __restrict__ XC, int n, const double* __restrict__ YC, int m,
                                         int D, double* __restrict__ part)
{
    __shared__ double red[256];
    const int tot = n + m;
    const int per = (tot + gridDim.x - 1) / gridDim.x;
    const int b0 = blockIdx.x * per, b1 = min(tot, b0 + per);
    double s = 0;
    for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
        const double* C = i < n ? XC + (size_t)i * D * D : YC + (size_t)(i - n) * D * D;
        for (int a = 0; a < D; ++a) s += C[a * (D + 1)];
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void cov_scale_kernel(const double* __restrict__ part, int nb, int tot, int D, double* __restrict__ scale)
{
    __shared__ double red[256];
    double s = 0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) s += part[b];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double tr = red[0] / ((double)D * tot);
        const double c = (isfinite(tr) && tr > 0) ? exp2(round(log2(tr))) : 1.0;
        scale[0] = c;
        scale[1] = 1.0 / c;
    }
}

int launch_init(Context& c, const double* X, const double* XC, const double* Y, const double* YC)
{
    const int D = c.D, N = c.N, M = c.M;
    const size_t nd = (size_t)N * D, md = (size_t)M * D;
    const size_t bytes = sizeof(double) * (nd + nd * D + md + md * D);
    if (bytes > c.scratch_bytes) return set_error(DUGMA_ERR_STATE, "init: staging does not fit the scratch region");
    double* tmp = c.scratch;   // the FP64 inputs are staged in the (still unused) scratch region
    double *tX = tmp, *tXC = tX + nd, *tY = tXC + nd * D, *tYC = tY + md;
    cudaStream_t s = c.stream;
    int rc = DUGMA_OK;
    auto ck = [&](cudaError_t e, const char* what) {
        if (e != cudaSuccess && rc == DUGMA_OK)
            rc = set_error(DUGMA_ERR_CUDA, "init: %s failed: %s", what, cudaGetErrorString(e));
    };
    // pageable sources: the driver pipelines these through its own pinned buffers (a
    // host-side copy into a pinned ring of ours measured slower on the B200 host)
    ck(cudaMemcpyAsync(tX, X, sizeof(double) * nd, cudaMemcpyHostToDevice, s), "copy X");
    ck(cudaMemcpyAsync(tXC, XC, sizeof(double) * nd * D, cudaMemcpyHostToDevice, s), "copy X_C");
    ck(cudaMemcpyAsync(tY, Y, sizeof(double) * md, cudaMemcpyHostToDevice, s), "copy Y");
    ck(cudaMemcpyAsync(tYC, YC, sizeof(double) * md * D, cudaMemcpyHostToDevice, s), "copy Y_C");
    ck(cudaMemsetAsync(c.counter, 0, sizeof(int) * 8, s), "memset");
    const int bs = 256;
    const int gx = std::min((N + bs - 1) / bs, c.num_sms * 8), gy = std::min((M + bs - 1) / bs, c.num_sms * 8);
    double* Lm = c.out;   // scratch: out[0], out[1] max log2 weights; out[2], out[3] the covariance scale
    // CONV covariances are kept divided by the mean of trace / D over both clouds
    const int nb = std::min(kMomSlots, std::max(1, (N + M + 2047) / 2048));
    cov_trace_partial_kernel<<<nb, 256, 0, s>>>(tXC, N, tYC, M, D, c.mom);
    cov_scale_kernel<<<1, 256, 0, s>>>(c.mom, nb, N + M, D, Lm + 2);
    // counter[4], counter[5]: weighted sources / targets without a Cholesky factor
    if (D == 3) {
        init_points_kernel<3><<<gx, bs, 0, s>>>(tX, tXC, N, c.x, c.xinv, c.wx, c.xcov, Lm + 2, c.counter, c.ux,
                                                c.counter + 4);
        init_points_kernel<3><<<gy, bs, 0, s>>>(tY, tYC, M, c.y, c.yinv, c.wy, c.ycov, Lm + 2, c.counter, nullptr,
                                                c.counter + 5);
    } else {
        init_points_kernel<2><<<gx, bs, 0, s>>>(tX, tXC, N, c.x, c.xinv, c.wx, c.xcov, Lm + 2, c.counter, c.ux,
                                                c.counter + 4);
        init_points_kernel<2><<<gy, bs, 0, s>>>(tY, tYC, M, c.y, c.yinv, c.wy, c.ycov, Lm + 2, c.counter, nullptr,
                                                c.counter + 5);
    }
    // counter[2], counter[3]: the largest weight of each cloud as float bits (zeroed above)
    max_weight_kernel<<<std::min(gx, 4 * c.num_sms), bs, 0, s>>>(c.wx, N, c.counter + 2);
    max_weight_kernel<<<std::min(gy, 4 * c.num_sms), bs, 0, s>>>(c.wy, M, c.counter + 3);
    norm_log2_kernel<<<gx, bs, 0, s>>>(c.wx, N, c.counter + 2, Lm, c.lwx);
    norm_log2_kernel<<<gy, bs, 0, s>>>(c.wy, M, c.counter + 3, Lm + 1, c.lwy);
    ck(cudaGetLastError(), "init kernels");
    ck(cudaMemcpyAsync(c.host, Lm, 3 * sizeof(double), cudaMemcpyDeviceToHost, s), "copy Lmax, scale");
    ck(cudaMemcpyAsync(c.host + 3, c.counter, sizeof(int), cudaMemcpyDeviceToHost, s), "copy nonpd");
    ck(cudaMemcpyAsync(c.host + 4, c.counter + 4, 2 * sizeof(int), cudaMemcpyDeviceToHost, s),
       "copy indefinite counts");
    ck(cudaStreamSynchronize(s), "sync");
    if (rc != DUGMA_OK) return rc;
    c.Lmax_x = std::isfinite(c.host[0]) ? c.host[0] : 0.0;
    c.Lmax_y = std::isfinite(c.host[1]) ? c.host[1] : 0.0;
    c.cscale = c.host[2];
    int nonpd = 0;
    memcpy(&nonpd, c.host + 3, sizeof(int));
    c.nonpd = nonpd;
    int indef[2] = {0, 0};
    memcpy(indef, c.host + 4, 2 * sizeof(int));
    c.x_indef = c.ux ? indef[0] : N;
    c.y_indef = indef[1];
    return DUGMA_OK;
}

// ---------------------------------------------------------------------------
// Per-evaluation prologue.
//   y records: y' = R y + t in FP64 in the order of update_sig.cu:247-249 / compi.cu:784-786,
//              split into y'hi = float(y'), y'lo = float(y' - y'hi);
//              C'_j = R (s sym(Sigma_y_j^-1)) R^T (compi.cu:757-765) scaled by k = -1/2 log2 e
//              (layout 0: packed as is; layout 1: off-diagonals doubled for the Horner form);
//              lv_j = log2(w_j) - Lmax_y.
//   x records: x_i, lw_i and either k * s * sym(Sigma_x_i^-1) with doubled off-diagonals (Horner
//              form) or, when ux is given, sqrt(|k| s) U_i from the init-time Cholesky factor U_i
//              of sym(Sigma_x_i^-1) (Cholesky form: (sqrt(|k| s) U_i)^T (sqrt(|k| s) U_i) = |k| B_i).
// Rows past N / M are null records (lw = -inf, zero matrices): they contribute exactly 0.
// ---------------------------------------------------------------------------
// source i's record: x, the log2 weight and its matrix, either the Cholesky factor scaled by
// sqrt(-ks) (ux given) or k B in the Horner layout
template <int D>
__device__ __forceinline__ void source_record(int i, const float* __restrict__ x, const float* __restrict__ xinv,
                                              const float* __restrict__ lwx, int N, XRec* __restrict__ xrec,
                                              const double* __restrict__ ux, double ks)
{
    constexpr int NS = Sym<D>::N;
    XRec r;
    float xv[3] = {0, 0, 0}, bp[6] = {0, 0, 0, 0, 0, 0};
    float lw = -INFINITY;
    if (i < N) {
#pragma unroll
        for (int a = 0; a < D; ++a) xv[a] = x[(size_t)i * D + a];
        lw = lwx[i];
        if (lw != -INFINITY && ux) {
            const double r = sqrt(-ks);
#pragma unroll
            for (int k = 0; k < NS; ++k) bp[k] = __double2float_rn(r * ux[(size_t)i * NS + k]);
        } else if (lw != -INFINITY) {
#pragma unroll
            for (int k = 0; k < NS; ++k) {
                const int ra = Sym<D>::a(k), rb = Sym<D>::b(k);
                double b = 0.5 * ((double)xinv[(size_t)i * D * D + ra + D * rb] +
                                  (double)xinv[(size_t)i * D * D + rb + D * ra]);
                double v = ks * b;
                if (ra != rb) v = 2.0 * v;
                bp[k] = __double2float_rn(v);
            }
        }
    }
    r.v0 = make_float4(xv[0], xv[1], xv[2], lw);
    r.v1 = make_float4(0.f, 0.f, 0.f, 0.f);
    if (D == 3) {
        r.v2 = make_float4(bp[0], bp[1], bp[2], bp[3]);
        r.v3 = make_float4(bp[4], bp[5], 0.f, 0.f);
    } else {
        r.v2 = make_float4(bp[0], bp[1], bp[2], 0.f);
        r.v3 = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    xrec[i] = r;
}

template <int D>
__global__ void prologue_kernel(const double* __restrict__ pose, const float* __restrict__ y,
                                const float* __restrict__ yinv, const float* __restrict__ lwy, int M, int M_pad,
                                int ylayout, YRec* __restrict__ yrec, float4* __restrict__ yp32,
                                const float* __restrict__ x, const float* __restrict__ xinv,
                                const float* __restrict__ lwx, int N, int N_pad, XRec* __restrict__ xrec,
                                const double* __restrict__ ux, int* __restrict__ reset_counter, const PoseBlock pv,
                                int use_pv, double* __restrict__ pose_out, int* __restrict__ reset_err)
{
    pdl_trigger();   // the pair kernel may be scheduled now; it waits for this kernel's writes
    constexpr int NS = Sym<D>::N;
    // the pose pv by value (use_pv; block 0 also writes it to pose_out, if given, for the kernels
    // that follow) or from pose
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (reset_counter) *reset_counter = 0;
        if (reset_err) *reset_err = 0;
        if (use_pv && pose_out)
#pragma unroll
            for (int k = 0; k < kPoseDoubles; ++k) pose_out[k] = pv.v[k];
    }
    double R[9], t[3];
#pragma unroll
    for (int k = 0; k < D * D; ++k) R[k] = use_pv ? pv.v[k] : pose[k];
#pragma unroll
    for (int a = 0; a < D; ++a) t[a] = use_pv ? pv.v[kPoseT + a] : pose[kPoseT + a];
    const double s = 1.0 / (use_pv ? pv.v[kPoseSig] : pose[kPoseSig]);
    const double ks = K_EXP2 * s;
    const int stride = gridDim.x * blockDim.x;
    // one thread per point: [0, M_pad) the targets, [M_pad, M_pad + N_pad) the sources
    for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < M_pad + N_pad; u += stride) {
        if (u >= M_pad) {
            source_record<D>(u - M_pad, x, xinv, lwx, N, xrec, ux, ks);
            continue;
        }
        const int j = u;
        YRec r;
        float hi[3] = {0, 0, 0}, lo[3] = {0, 0, 0}, cp[6] = {0, 0, 0, 0, 0, 0};
        float lv = -INFINITY;
        if (j < M) {
            double yj[3];
#pragma unroll
            for (int a = 0; a < D; ++a) yj[a] = (double)y[(size_t)j * D + a];
#pragma unroll
            for (int a = 0; a < D; ++a) {
                double v = R[a] * yj[0] + R[a + D] * yj[1];
                if (D == 3) v = v + R[a + 6] * yj[2];
                v = v + t[a];
                hi[a] = __double2float_rn(v);
                lo[a] = __double2float_rn(v - (double)hi[a]);
            }
            lv = lwy[j];
            if (lv != -INFINITY) {
                double A[D][D];
#pragma unroll
                for (int r0 = 0; r0 < D; ++r0)
#pragma unroll
                    for (int c0 = 0; c0 < D; ++c0)
                        A[r0][c0] = 0.5 * ((double)yinv[(size_t)j * D * D + r0 + D * c0] +
                                           (double)yinv[(size_t)j * D * D + c0 + D * r0]);
                double T[D][D];   // A R^T
#pragma unroll
                for (int r0 = 0; r0 < D; ++r0)
#pragma unroll
                    for (int c0 = 0; c0 < D; ++c0) {
                        double acc = 0;
#pragma unroll
                        for (int k = 0; k < D; ++k) acc = acc + A[r0][k] * R[c0 + D * k];
                        T[r0][c0] = acc;
                    }
#pragma unroll
                for (int k = 0; k < NS; ++k) {
                    const int ra = Sym<D>::a(k), rb = Sym<D>::b(k);
                    double acc = 0;
#pragma unroll
                    for (int q = 0; q < D; ++q) acc = acc + R[ra + D * q] * T[q][rb];
                    double v = ks * acc;
                    if ((ylayout & 1) && ra != rb) v = 2.0 * v;   // Horner layouts (1, 3)
                    cp[k] = __double2float_rn(v);
                }
            }
        }
        if (ylayout >= 2) {
            // paired layout: this target fills its half of pair record j / 2
            float f[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) f[q] = 0.f;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                f[a] = -hi[a];
                f[4 + a] = -lo[a];
            }
            f[3] = lv;
            f[13] = -lv;
#pragma unroll
            for (int k = 0; k < NS; ++k) f[7 + k] = cp[k];
            float* base = reinterpret_cast<float*>(yrec) + (size_t)(j >> 1) * 32 + (j & 1);
#pragma unroll
            for (int q = 0; q < 16; ++q) base[(q >> 1) * 4 + (q & 1) * 2] = f[q];
        } else {
            r.v0 = make_float4(hi[0], hi[1], hi[2], lv);
            r.v1 = make_float4(lo[0], lo[1], lo[2], 0.f);
            if (D == 3) {
                r.v2 = make_float4(cp[0], cp[1], cp[2], cp[3]);
                r.v3 = make_float4(cp[4], cp[5], 0.f, 0.f);
            } else {
                r.v2 = make_float4(cp[0], cp[1], cp[2], 0.f);
                r.v3 = make_float4(0.f, 0.f, 0.f, 0.f);
            }
            yrec[j] = r;
        }
        // nearest-neighbour records, two targets per 32 bytes with negated coordinates:
        // (-y0 2p, -y0 2p+1, -y1 2p, -y1 2p+1), (-y2 2p, -y2 2p+1, 0, 0); padding targets sit
        // at +inf so that no source ever picks them as a neighbour
        if (yp32) {
            float* pr = reinterpret_cast<float*>(yp32 + 2 * (j / 2));
            const int h = j & 1;
            for (int q = 0; q < 3; ++q) pr[2 * q + h] = j < M ? (q < D ? -hi[q] : 0.f) : -INFINITY;
            pr[6 + h] = 0.f;
        }
    }
}

// the search records of target j (the yp32 layout of prologue_kernel): two targets per 32 bytes,
// coordinates negated, padding targets at +inf
// The pose: pv by value (use_pv; block 0 also writes it to pose), else read from pose.
template <int D>
__global__ void nn_prologue_kernel(const PoseBlock pv, int use_pv, double* __restrict__ pose,
                                   const float* __restrict__ y, int M, int M_pad, float4* __restrict__ yp32,
                                   int* __restrict__ reset_counter, int* __restrict__ reset_err)
{
    pdl_trigger();   // the search kernel may be scheduled now; it waits for this kernel's writes
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
    const int stride = gridDim.x * blockDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < M_pad; j += stride) {
        float hi[3] = {0, 0, 0};
        if (j < M) {
            double yj[3];
#pragma unroll
            for (int a = 0; a < D; ++a) yj[a] = (double)y[(size_t)j * D + a];
#pragma unroll
            for (int a = 0; a < D; ++a) {
                double v = R[a] * yj[0] + R[a + D] * yj[1];
                if (D == 3) v = v + R[a + 6] * yj[2];
                v = v + t[a];
                hi[a] = __double2float_rn(v);
            }
        }
        float* pr = reinterpret_cast<float*>(yp32 + 2 * (j / 2));
        const int h = j & 1;
        for (int q = 0; q < 3; ++q) pr[2 * q + h] = j < M ? (q < D ? -hi[q] : 0.f) : -INFINITY;
        pr[6 + h] = 0.f;
    }
}

// One block: the pose block from src (device-visible memory: the mapped pinned staging a captured
// graph reads at each launch) into pose, the error word zeroed.  The kernels that follow read the
// pose from device memory (every block reading the staging over the host link costs more).
__global__ void pose_in_kernel(const double* __restrict__ src, double* __restrict__ pose, int* __restrict__ err)
{
    if (threadIdx.x < kPoseDoubles) pose[threadIdx.x] = src[threadIdx.x];
    if (threadIdx.x == 0 && err) *err = 0;
}

int launch_pose_in(Context& c, const double* src, double* pose_dev, cudaStream_t s, bool reset_err)
{
    pose_in_kernel<<<1, 32, 0, s>>>(src, pose_dev, reset_err ? c.err : nullptr);
    DUGMA_CK(cudaGetLastError());
    return DUGMA_OK;
}

int launch_nn_prologue(Context& c, double* pose_dev, cudaStream_t s, const PoseBlock* pv, int* reset_counter,
                       int* reset_err)
{
    PoseBlock pb{};
    if (pv) pb = *pv;
    const int g = std::min((c.M_pad + 127) / 128, c.num_sms * 8);
    if (c.D == 3)
        nn_prologue_kernel<3><<<g, 128, 0, s>>>(pb, pv ? 1 : 0, pose_dev, c.y, c.M, c.M_pad, c.yp32, reset_counter,
                                                reset_err);
    else
        nn_prologue_kernel<2><<<g, 128, 0, s>>>(pb, pv ? 1 : 0, pose_dev, c.y, c.M, c.M_pad, c.yp32, reset_counter,
                                                reset_err);
    DUGMA_CK(cudaGetLastError());
    return DUGMA_OK;
}

int launch_prologue(Context& c, const double* pose_dev, int ylayout, cudaStream_t s, bool xchol, int* reset_counter,
                    const PoseBlock* pv, double* pose_out, int* reset_err)
{
    PoseBlock pb{};
    if (pv) pb = *pv;
    if (xchol && (!c.ux || c.x_indef > 0))
        return set_error(DUGMA_ERR_STATE, "Cholesky-form source records need a positive definite factor per source");
    const double* ux = xchol ? c.ux : nullptr;
    const int n = c.M_pad + c.N_pad;
    const int bs = 128;
    const int g = std::min((n + bs - 1) / bs, c.num_sms * 8);
    if (c.D == 3)
        prologue_kernel<3><<<g, bs, 0, s>>>(pose_dev, c.y, c.yinv, c.lwy, c.M, c.M_pad, ylayout, c.yrec, nullptr,
                                            c.x, c.xinv, c.lwx, c.N, c.N_pad, c.xrec, ux, reset_counter, pb,
                                            pv ? 1 : 0, pose_out, reset_err);
    else
        prologue_kernel<2><<<g, bs, 0, s>>>(pose_dev, c.y, c.yinv, c.lwy, c.M, c.M_pad, ylayout, c.yrec, nullptr,
                                            c.x, c.xinv, c.lwx, c.N, c.N_pad, c.xrec, ux, reset_counter, pb,
                                            pv ? 1 : 0, pose_out, reset_err);
    DUGMA_CK(cudaGetLastError());
    return DUGMA_OK;
}

}  // namespace dugma

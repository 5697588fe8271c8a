// nn.cu -- brute-force nearest neighbours and sigma (the update_sig plugin).
//
// The reference computes, for every x_i, min_j |x_i - (R y_j + t)|^2 / D quantised to
// 1e-6 as an unsigned int with shared and global atomicMin, then a FP32 tree sum
// (update_sig.cu:181-269, 272-315, 384-385).  Here:
//   y'_j = float(FP64(R y_j + t))               (update_sig.cu:247-252, written by the prologue)
//   d    = x_i - y'_j in FP32,  d2 = fmaf(dz,dz, fmaf(dy,dy, dx*dx))
// Target records hold two targets each, coordinates negated (d = x + (-y') is the same FP32
// value), interleaved so that the search kernels evaluate both with f32x2 operations.
//   the k smallest (d2, j) in lexicographic order are kept in registers (ties -> lowest j)
// Targets are streamed by bulk copy like the energy kernels; target chunks are merged in
// index order afterwards, so the result is exact and deterministic.  sigma is then
//   exact:      sum_i d2min_i / (D N) in FP64
//   quantised:  sum_i rn_u32(fl32(d2min_i / D) * 1e6) / 1e6 / N   (the reference's value)
#include <cmath>

#include "context.hpp"
#include "pairs.cuh"

namespace dugma {

// two nearest-neighbour targets (see the prologue): a = (-y0, -y0', -y1, -y1'), b = (-y2, -y2', 0, 0)
struct __align__(16) NNRec2 {
    float4 a, b;
};

template <int D, int IPT_, int K>
struct NNBody {
    using StreamRec = NNRec2;
    static constexpr int IPT = IPT_;
    static constexpr int NV = 1;
    float2 X[IPT][D];   // source coordinates, duplicated in both halves
    float bd[IPT][K];
    int bi[IPT][K];
    int row[IPT];

    __device__ void setup(const PairArgs&) {}
    __device__ void load_src(const PairArgs& a, int ii, int i)
    {
        const float* xs = static_cast<const float*>(a.xrec);
        row[ii] = i < a.i_end ? i : -1;
#pragma unroll
        for (int q = 0; q < D; ++q) {
            const float v = i < a.i_end ? xs[(size_t)i * D + q] : 0.f;
            X[ii][q] = make_float2(v, v);
        }
    }
    __device__ void zero_all()
    {
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii)
#pragma unroll
            for (int q = 0; q < K; ++q) { bd[ii][q] = INFINITY; bi[ii][q] = 0x7fffffff; }
    }
    // both targets of a record in one f32x2 sequence (per half the FP32 operations of the
    // reference: d = x + (-y'), d2 = fmaf(dz,dz, fmaf(dy,dy, dx*dx))), then one test per source
    // of the nearer of the two against its k-th distance; the rare insertions take the targets
    // in index order, so ties keep the lower j
    __device__ __forceinline__ void consume(const NNRec2& r, int jp)
    {
        const float2 n0 = make_float2(r.a.x, r.a.y), n1 = make_float2(r.a.z, r.a.w), n2 = make_float2(r.b.x, r.b.y);
        float2 dd[IPT];
        bool hit = false;
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            const float2 d0 = fadd2(X[ii][0], n0), d1 = fadd2(X[ii][1], n1);
            if (D == 3) {
                const float2 d2 = fadd2(X[ii][2], n2);
                dd[ii] = ffma2(d2, d2, ffma2(d1, d1, fmul2(d0, d0)));
            } else {
                dd[ii] = ffma2(d1, d1, fmul2(d0, d0));
            }
            hit |= fminf(dd[ii].x, dd[ii].y) < bd[ii][K - 1];
        }
        // one branch per record for all the sources: the distance arithmetic above stays
        // branch-free and schedules like the distance-only kernel
        if (hit) {
#pragma unroll
            for (int ii = 0; ii < IPT; ++ii) {
                insert(ii, dd[ii].x, 2 * jp);
                insert(ii, dd[ii].y, 2 * jp + 1);
            }
        }
    }
    __device__ __forceinline__ void insert(int ii, float dd, int j)
    {
        if (!(dd < bd[ii][K - 1])) return;
        // sorted insertion; strict comparisons keep the earlier index first on ties
#pragma unroll
        for (int q = K - 1; q > 0; --q) {
            const bool shift = dd < bd[ii][q - 1];
            const bool place = !shift && dd < bd[ii][q];
            bd[ii][q] = shift ? bd[ii][q - 1] : (place ? dd : bd[ii][q]);
            bi[ii][q] = shift ? bi[ii][q - 1] : (place ? j : bi[ii][q]);
        }
        if (dd < bd[ii][0]) { bd[ii][0] = dd; bi[ii][0] = j; }
    }
    __device__ void fold() {}
    __device__ void finish(const PairArgs& a, int jc, double (&)[NV])
    {
        // partial lists for this target chunk: h_part as [n_jc][rows][K] (d2 float, idx int) pairs
        const int rows = a.i_end - a.i0;
        float2* out = reinterpret_cast<float2*>(a.h_part);
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            if (row[ii] < 0) continue;
            float2* o = out + ((size_t)jc * rows + (row[ii] - a.i0)) * K;
#pragma unroll
            for (int q = 0; q < K; ++q) o[q] = make_float2(bd[ii][q], __int_as_float(bi[ii][q]));
        }
    }
};

// Nearest squared distance only (sigma): both targets of a record in one f32x2 sequence, the
// same FP32 operations as NNBody, a running minimum per half.
template <int D, int IPT_>
struct NNMinBody {
    using StreamRec = NNRec2;
    static constexpr int IPT = IPT_;
    static constexpr int NV = 1;
    float2 X[IPT][D];
    float2 bd[IPT];
    int row[IPT];

    __device__ void setup(const PairArgs&) {}
    __device__ void load_src(const PairArgs& a, int ii, int i)
    {
        const float* xs = static_cast<const float*>(a.xrec);
        row[ii] = i < a.i_end ? i : -1;
#pragma unroll
        for (int q = 0; q < D; ++q) {
            const float v = i < a.i_end ? xs[(size_t)i * D + q] : 0.f;
            X[ii][q] = make_float2(v, v);
        }
    }
    __device__ void zero_all()
    {
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) bd[ii] = make_float2(INFINITY, INFINITY);
    }
    __device__ __forceinline__ void consume(const NNRec2& r, int)
    {
        const float2 n0 = make_float2(r.a.x, r.a.y), n1 = make_float2(r.a.z, r.a.w), n2 = make_float2(r.b.x, r.b.y);
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            const float2 d0 = fadd2(X[ii][0], n0), d1 = fadd2(X[ii][1], n1);
            float2 dd;
            if (D == 3) {
                const float2 d2 = fadd2(X[ii][2], n2);
                dd = ffma2(d2, d2, ffma2(d1, d1, fmul2(d0, d0)));
            } else {
                dd = ffma2(d1, d1, fmul2(d0, d0));
            }
            bd[ii].x = fminf(bd[ii].x, dd.x);
            bd[ii].y = fminf(bd[ii].y, dd.y);
        }
    }
    __device__ void fold() {}
    __device__ void finish(const PairArgs& a, int jc, double (&)[NV])
    {
        const int rows = a.i_end - a.i0;
        float2* out = reinterpret_cast<float2*>(a.h_part);
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            if (row[ii] < 0) continue;
            out[(size_t)jc * rows + (row[ii] - a.i0)] = make_float2(fminf(bd[ii].x, bd[ii].y), __int_as_float(0));
        }
    }
};

// merge the per-chunk sorted lists in chunk (= index) order
template <int K>
__global__ void nn_merge_kernel(const float2* __restrict__ part, int n_jc, int rows, int k_out, int* __restrict__ idx,
                                float* __restrict__ d2, float* __restrict__ dmin)
{
    pdl_trigger();   // a dependent of the search kernel; the sigma sums (if any) dependents of this one
    pdl_wait();
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
        float bd[K];
        int bi[K];
#pragma unroll
        for (int q = 0; q < K; ++q) { bd[q] = INFINITY; bi[q] = 0x7fffffff; }
        for (int c = 0; c < n_jc; ++c) {
            const float2* p = part + ((size_t)c * rows + r) * K;
            for (int e = 0; e < K; ++e) {
                const float dd = p[e].x;
                const int j = __float_as_int(p[e].y);
                if (!(dd < bd[K - 1])) break;   // lists are sorted: nothing further can enter
#pragma unroll
                for (int q = K - 1; q > 0; --q) {
                    const bool shift = dd < bd[q - 1];
                    const bool place = !shift && dd < bd[q];
                    bd[q] = shift ? bd[q - 1] : (place ? dd : bd[q]);
                    bi[q] = shift ? bi[q - 1] : (place ? j : bi[q]);
                }
                if (dd < bd[0]) { bd[0] = dd; bi[0] = j; }
            }
        }
        if (idx)
            for (int q = 0; q < k_out; ++q) {
                idx[(size_t)r * k_out + q] = bi[q];
                d2[(size_t)r * k_out + q] = bd[q];
            }
        if (dmin) dmin[r] = bd[0];
    }
}

// sigma sums over the nearest squared distances: per-block partials over contiguous slices
// (fixed order), then one block over the partials (fixed order), so the result is deterministic
__global__ void sigma_partial_kernel(const float* __restrict__ dmin, int n, int D, double* __restrict__ pe,
                                     unsigned long long* __restrict__ pq)
{
    pdl_trigger();   // a dependent of the merge of the nearest distances; the final sum one of this kernel
    pdl_wait();
    __shared__ double s_exact[256];
    __shared__ unsigned long long s_q[256];
    const int per = (n + gridDim.x - 1) / gridDim.x;
    const int b0 = blockIdx.x * per, b1 = min(n, b0 + per);
    double se = 0;
    unsigned long long sq = 0;
    for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
        const float v = dmin[i];
        se += (double)v;
        const float sv = __fmul_rn(__fdiv_rn(v, (float)D), 1000000.0f);
        sq += (unsigned long long)__float2uint_rn(sv);
    }
    s_exact[threadIdx.x] = se;
    s_q[threadIdx.x] = sq;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            s_exact[threadIdx.x] += s_exact[threadIdx.x + h];
            s_q[threadIdx.x] += s_q[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        pe[blockIdx.x] = s_exact[0];
        pq[blockIdx.x] = s_q[0];
    }
}

// host_out (optional, mapped pinned memory) receives out[0..1] and the error word at [2];
// pose_sig (optional) a device pose block whose sig becomes out[1]
__global__ void sigma_final_kernel(const double* __restrict__ pe, const unsigned long long* __restrict__ pq, int nb,
                                   int n, int D, double* __restrict__ out, double* __restrict__ host_out,
                                   const int* __restrict__ err, double* __restrict__ pose_sig)
{
    pdl_wait();   // a dependent of sigma_partial_kernel
    __shared__ double s_exact[256];
    __shared__ unsigned long long s_q[256];
    double se = 0;
    unsigned long long sq = 0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        se += pe[i];
        sq += pq[i];
    }
    s_exact[threadIdx.x] = se;
    s_q[threadIdx.x] = sq;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            s_exact[threadIdx.x] += s_exact[threadIdx.x + h];
            s_q[threadIdx.x] += s_q[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double o0, o1;
        if (n > 0) {
            o0 = s_exact[0] / ((double)D * n);
            o1 = (double)__double2float_rn((double)s_q[0] / 1e6 / (double)n);
        } else {   // the partial sums of a row range: sum d2min, and the sum of the quantised terms
            o0 = s_exact[0];
            o1 = (double)s_q[0];
        }
        out[0] = o0;
        out[1] = o1;
        if (pose_sig) pose_sig[kPoseSig] = o1;   // the quantised sigma, rounded to float as update_sig returns it
        if (host_out) {
            host_out[0] = o0;
            host_out[1] = o1;
            host_out[2] = (double)*err;
        }
    }
}

template <class Body, int NT, int TJ>
__global__ void __launch_bounds__(NT) nn_kernel(PairArgs a)
{
    Body body;
    run_pairs<Body, NT, TJ, 4>(a, body);
}


struct NNVariant {
    KernelShape shape;   // tj counts records of two targets; ipt is the k = 1 sources per thread
    KernelFn k1;
    KernelFn k8;
    int ipt8;            // sources per thread of the k <= 8 kernel
    KernelFn k16;
    int ipt16;           // sources per thread of the k <= 16 kernel
    KernelFn kmin;       // nearest distance only (sigma)
};

template <int D>
static const std::vector<NNVariant>& nn_variants()
{
    static const std::vector<NNVariant> v = {
        {{4, 128, 64}, nn_kernel<NNBody<D, 4, 1>, 128, 64>, nn_kernel<NNBody<D, 2, 8>, 128, 64>, 2,
         nn_kernel<NNBody<D, 1, 16>, 128, 64>, 1, nn_kernel<NNMinBody<D, 4>, 128, 64>},
        {{8, 128, 64}, nn_kernel<NNBody<D, 8, 1>, 128, 64>, nn_kernel<NNBody<D, 1, 8>, 128, 64>, 1,
         nn_kernel<NNBody<D, 2, 16>, 128, 64>, 2, nn_kernel<NNMinBody<D, 8>, 128, 64>},
        {{4, 256, 64}, nn_kernel<NNBody<D, 4, 1>, 256, 64>, nn_kernel<NNBody<D, 2, 8>, 256, 64>, 2,
         nn_kernel<NNBody<D, 1, 16>, 256, 64>, 1, nn_kernel<NNMinBody<D, 4>, 256, 64>},
    };
    return v;
}

std::vector<KernelShape> nn_shapes()
{
    std::vector<KernelShape> s;
    for (auto& v : nn_variants<3>()) s.push_back(v.shape);
    return s;
}

// Runs the brute-force search; dmin_dev (nullable) receives the nearest squared distance per source.
// Source rows [i0, i1) (i1 < 0: all); idx/d2 rows are relative to i0, dmin is indexed absolutely.
// The search: the targets' search records (the nearest-neighbour prologue, which also zeroes the
// work counter, and the error word when reset_err; the pose by value when pv, or read from
// pose_src), the pair kernel, the merge of its per-chunk lists.
static int nn_run(Context& c, double* pose_dev, int k, int* idx_dev, float* d2_dev, float* dmin_dev,
                  cudaStream_t s, const KernelShape* force, int i0 = 0, int i1 = -1, const PoseBlock* pv = nullptr,
                  const double* pose_src = nullptr, bool reset_err = false)
{
    if (i1 < 0) i1 = c.N;
    const int rows = i1 - i0;
    if (pose_src) {
        DUGMA_RET(launch_pose_in(c, pose_src, pose_dev, s, reset_err));
        reset_err = false;
    }
    DUGMA_RET(launch_nn_prologue(c, pose_dev, s, pv, c.counter, reset_err ? c.err : nullptr));
    const KernelShape want = force ? *force : c.shape_nn;
    const auto& vars = c.D == 3 ? nn_variants<3>() : nn_variants<2>();
    const NNVariant* v = &vars[0];
    for (auto& cand : vars)
        if (cand.shape.ipt == want.ipt && cand.shape.nt == want.nt && cand.shape.tj == want.tj) v = &cand;
    const int K = k <= 1 ? 1 : (k <= 8 ? 8 : 16);
    // only the nearest distance wanted (sigma): the packed distance-only kernel
    const bool min_only = K == 1 && !idx_dev && !d2_dev;
    KernelFn fn = min_only ? v->kmin : (K == 1 ? v->k1 : (K == 8 ? v->k8 : v->k16));
    KernelShape sh = v->shape;
    // the k = 8 / 16 kernels may keep fewer sources per thread (see the variant table)
    if (K == 8) sh.ipt = v->ipt8;
    if (K == 16) sh.ipt = v->ipt16;
    if (K > 1) {
        // every target chunk restarts the sorted lists, and a list insertion (taken by some lane
        // of a warp far more often than by one thread) costs the whole warp ~4K instructions:
        // few long chunks, just enough items to fill the GPU about once
        const int n_ib = (rows + sh.ipt * sh.nt - 1) / (sh.ipt * sh.nt);
        const int want_jc = std::max(1, (4 * c.num_sms + n_ib - 1) / n_ib);
        sh.min_chunk = std::max(1, (c.M_pad / 2 + want_jc - 1) / want_jc);
    }
    double* hp = nullptr;
    int n_jc = 0;
    DUGMA_RET(launch_pair_variant(c, fn, sh, c.x, c.yp32, (size_t)c.M_pad / 2, 1, 0.0, pose_dev, i0, i1, nullptr,
                                  nullptr, &hp, K, &n_jc, s, nullptr, true));
    const int g = std::min((rows + 255) / 256, c.num_sms * 8);
    const float2* part = reinterpret_cast<const float2*>(hp);
    float* dm = dmin_dev ? dmin_dev + i0 : nullptr;
    if (K == 1)
        DUGMA_CK(launch_dependent(c.pdl, nn_merge_kernel<1>, g, 256, 0, s, part, n_jc, rows, k, idx_dev, d2_dev, dm));
    else if (K == 8)
        DUGMA_CK(launch_dependent(c.pdl, nn_merge_kernel<8>, g, 256, 0, s, part, n_jc, rows, k, idx_dev, d2_dev, dm));
    else
        DUGMA_CK(launch_dependent(c.pdl, nn_merge_kernel<16>, g, 256, 0, s, part, n_jc, rows, k, idx_dev, d2_dev, dm));
    return DUGMA_OK;
}

int launch_nn(Context& c, double* pose_dev, int k, int* idx_dev, float* d2_dev, cudaStream_t s,
              const KernelShape* force)
{
    if (k < 1 || k > 16 || k > c.M) return set_error(DUGMA_ERR_ARG, "k = %d must be in [1, min(16, M)]", k);
    return nn_run(c, pose_dev, k, idx_dev, d2_dev, nullptr, s, force);
}

int launch_sigma(Context& c, double* pose_dev, double* out_dev, cudaStream_t s, int i0, int i1, const SigmaOpts& o)
{
    const bool whole = i1 < 0;
    if (whole) i1 = c.N;
    const int rows = i1 - i0;
    DUGMA_RET(nn_run(c, pose_dev, 1, nullptr, nullptr, c.dmin, s, nullptr, i0, i1, o.pose_value, o.pose_src,
                     o.reset_err));
    // partials in the scratch region (the search's chunk lists there are merged by now, in stream order)
    const int nb = std::max(1, std::min(2 * c.num_sms, (rows + 1023) / 1024));
    DUGMA_RET(c.ensure_scratch(sizeof(double) * 2 * (size_t)nb));
    double* pe = c.scratch;
    unsigned long long* pq = reinterpret_cast<unsigned long long*>(c.scratch + nb);
    DUGMA_CK(launch_dependent(c.pdl, sigma_partial_kernel, nb, 256, 0, s, (const float*)(c.dmin + i0), rows, c.D, pe,
                              pq));
    DUGMA_CK(launch_dependent(c.pdl, sigma_final_kernel, 1, 256, 0, s, (const double*)pe,
                              (const unsigned long long*)pq, nb, whole ? c.N : 0, c.D, out_dev, o.host_out,
                              (const int*)c.err, o.pose_sig));
    return DUGMA_OK;
}

}  // namespace dugma

// nn.cu -- brute-force nearest neighbours and sigma (the update_sig plugin).
//
// The reference computes, for every x_i, min_j |x_i - (R y_j + t)|^2 / D quantised to
// 1e-6 as an unsigned int with shared and global atomicMin, then a FP32 tree sum
// (update_sig.cu:181-269, 272-315, 384-385).  Here:
//   y'_j = float(FP64(R y_j + t))               (update_sig.cu:247-252, written by the prologue)
//   d    = x_i - y'_j in FP32,  d2 = fmaf(dz,dz, fmaf(dy,dy, dx*dx))
//   the k smallest (d2, j) in lexicographic order are kept in registers (ties -> lowest j)
// Targets are streamed by bulk copy like the energy kernels; target chunks are merged in
// index order afterwards, so the result is exact and deterministic.  sigma is then
//   exact:      sum_i d2min_i / (D N) in FP64
//   quantised:  sum_i rn_u32(fl32(d2min_i / D) * 1e6) / 1e6 / N   (the reference's value)
#include <cmath>

#include "context.hpp"
#include "pairs.cuh"

namespace dugma {

template <int D, int IPT_, int K>
struct NNBody {
    using StreamRec = float4;
    static constexpr int IPT = IPT_;
    static constexpr int NV = 1;
    float x[IPT][D];
    float bd[IPT][K];
    int bi[IPT][K];
    int row[IPT];

    __device__ void setup(const PairArgs&) {}
    __device__ void load_src(const PairArgs& a, int ii, int i)
    {
        const float* xs = static_cast<const float*>(a.xrec);
        row[ii] = i < a.i_end ? i : -1;
#pragma unroll
        for (int q = 0; q < D; ++q) x[ii][q] = i < a.i_end ? xs[(size_t)i * D + q] : 0.f;
    }
    __device__ void zero_all()
    {
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii)
#pragma unroll
            for (int q = 0; q < K; ++q) { bd[ii][q] = INFINITY; bi[ii][q] = 0x7fffffff; }
    }
    __device__ __forceinline__ void consume(const float4& y, int j)
    {
#pragma unroll
        for (int ii = 0; ii < IPT; ++ii) {
            const float d0 = x[ii][0] - y.x, d1 = x[ii][1] - y.y;
            float dd;
            if (D == 3) {
                const float d2 = x[ii][2] - y.z;
                dd = fmaf(d2, d2, fmaf(d1, d1, d0 * d0));
            } else {
                dd = fmaf(d1, d1, d0 * d0);
            }
            if (K == 1) {
                if (dd < bd[ii][0]) { bd[ii][0] = dd; bi[ii][0] = j; }
            } else if (dd < bd[ii][K - 1]) {
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
        }
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

// merge the per-chunk sorted lists in chunk (= index) order
template <int K>
__global__ void nn_merge_kernel(const float2* __restrict__ part, int n_jc, int rows, int k_out, int* __restrict__ idx,
                                float* __restrict__ d2, float* __restrict__ dmin)
{
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

// sigma sums over the nearest squared distances (single block, fixed order)
__global__ void sigma_kernel(const float* __restrict__ dmin, int n, int D, double* __restrict__ out)
{
    __shared__ double s_exact[256];
    __shared__ unsigned long long s_q[256];
    double se = 0;
    unsigned long long sq = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
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
        out[0] = s_exact[0] / ((double)D * n);
        out[1] = (double)__double2float_rn((double)s_q[0] / 1e6 / (double)n);
    }
}

template <class Body, int NT, int TJ>
__global__ void __launch_bounds__(NT) nn_kernel(PairArgs a)
{
    Body body;
    run_pairs<Body, NT, TJ, 4>(a, body);
}

using KernelFn = void (*)(PairArgs);
int launch_pair_variant(Context& c, KernelFn fn, const KernelShape& sh, const void* xrec, const void* yrec,
                        size_t yrec_size, int nv, double Lmax, const double* pose_dev, int i0, int i1,
                        double* out_dev, double* dEdx_dev, double** h_part, int h_width, int* n_jc_out,
                        cudaStream_t s);

struct NNVariant {
    KernelShape shape;
    KernelFn k1, k8, k16;
};

template <int D>
static const std::vector<NNVariant>& nn_variants()
{
    static const std::vector<NNVariant> v = {
        {{4, 128, 128}, nn_kernel<NNBody<D, 4, 1>, 128, 128>, nn_kernel<NNBody<D, 4, 8>, 128, 128>,
         nn_kernel<NNBody<D, 2, 16>, 128, 128>},
        {{8, 128, 128}, nn_kernel<NNBody<D, 8, 1>, 128, 128>, nn_kernel<NNBody<D, 4, 8>, 128, 128>,
         nn_kernel<NNBody<D, 2, 16>, 128, 128>},
        {{4, 256, 128}, nn_kernel<NNBody<D, 4, 1>, 256, 128>, nn_kernel<NNBody<D, 2, 8>, 256, 128>,
         nn_kernel<NNBody<D, 1, 16>, 256, 128>},
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
static int nn_run(Context& c, const double* pose_dev, int k, int* idx_dev, float* d2_dev, float* dmin_dev,
                  cudaStream_t s, const KernelShape* force)
{
    DUGMA_RET(launch_prologue(c, pose_dev, 0, s));
    const KernelShape want = force ? *force : c.shape_nn;
    const auto& vars = c.D == 3 ? nn_variants<3>() : nn_variants<2>();
    const NNVariant* v = &vars[0];
    for (auto& cand : vars)
        if (cand.shape.ipt == want.ipt && cand.shape.nt == want.nt && cand.shape.tj == want.tj) v = &cand;
    const int K = k <= 1 ? 1 : (k <= 8 ? 8 : 16);
    KernelFn fn = K == 1 ? v->k1 : (K == 8 ? v->k8 : v->k16);
    KernelShape sh = v->shape;
    // the k = 8 / 16 kernels keep fewer sources per thread (see the variant table)
    if (K == 8) sh.ipt = sh.nt == 128 ? 4 : 2;
    if (K == 16) sh.ipt = sh.nt == 128 ? 2 : 1;
    double* hp = nullptr;
    int n_jc = 0;
    DUGMA_RET(launch_pair_variant(c, fn, sh, c.x, c.yp32, (size_t)c.M_pad, 1, 0.0, pose_dev, 0, c.N, nullptr,
                                  nullptr, &hp, K, &n_jc, s));
    const int g = std::min((c.N + 255) / 256, c.num_sms * 8);
    const float2* part = reinterpret_cast<const float2*>(hp);
    if (K == 1)
        nn_merge_kernel<1><<<g, 256, 0, s>>>(part, n_jc, c.N, k, idx_dev, d2_dev, dmin_dev);
    else if (K == 8)
        nn_merge_kernel<8><<<g, 256, 0, s>>>(part, n_jc, c.N, k, idx_dev, d2_dev, dmin_dev);
    else
        nn_merge_kernel<16><<<g, 256, 0, s>>>(part, n_jc, c.N, k, idx_dev, d2_dev, dmin_dev);
    DUGMA_CK(cudaGetLastError());
    return DUGMA_OK;
}

int launch_nn(Context& c, const double* pose_dev, int k, int* idx_dev, float* d2_dev, cudaStream_t s,
              const KernelShape* force)
{
    if (k < 1 || k > 16 || k > c.M) return set_error(DUGMA_ERR_ARG, "k = %d must be in [1, min(16, M)]", k);
    return nn_run(c, pose_dev, k, idx_dev, d2_dev, nullptr, s, force);
}

int launch_sigma(Context& c, const double* pose_dev, double* out_dev, cudaStream_t s)
{
    DUGMA_RET(nn_run(c, pose_dev, 1, nullptr, nullptr, c.dmin, s, nullptr));
    sigma_kernel<<<1, 256, 0, s>>>(c.dmin, c.N, c.D, out_dev);
    DUGMA_CK(cudaGetLastError());
    return DUGMA_OK;
}

}  // namespace dugma

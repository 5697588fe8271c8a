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

#include "bodies.cuh"
#include "context.hpp"
#include "pairs.cuh"

namespace dugma {

template <class Body, int NT, int TJ>
__global__ void __launch_bounds__(NT) pair_kernel(PairArgs a)
{
    Body body;
    run_pairs<Body, NT, TJ, 4>(a, body);
}

// the same with a register budget that keeps MINB blocks resident per SM, and the record loop
// unrolled UNROLL times
template <class Body, int NT, int TJ, int MINB, int UNROLL = 4>
__global__ void __launch_bounds__(NT, MINB) pair_kernel_occ(PairArgs a)
{
    Body body;
    run_pairs<Body, NT, TJ, 4, UNROLL>(a, body);
}

// deterministic reduction of per-item partials: out[v] = sum_items partials[item][v];
// block v sums value v in a fixed order (strided per thread, then a fixed tree)
// host_out (optional, mapped pinned memory) receives out[0..nv) and the error word at [nv]
__global__ void __launch_bounds__(1024) reduce_items_kernel(const double* __restrict__ part, int n_items, int nv,
                                                             double* __restrict__ out, double* __restrict__ host_out,
                                                             const int* __restrict__ err)
{
    pdl_wait();   // a dependent of the pair kernel: its partials
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
    if (threadIdx.x == 0) {
        out[v] = red[0];
        if (host_out) {
            host_out[v] = red[0];
            if (v == 0) host_out[nv] = (double)*err;
        }
    }
}

__global__ void reduce_chunks_kernel(const double* __restrict__ part, int n_jc, size_t n, double* __restrict__ out)
{
    pdl_wait();   // a dependent of the pair kernel (or of reduce_items_kernel after it): its partials
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        double s = 0;
        for (int c = 0; c < n_jc; ++c) s += part[(size_t)c * n + e];
        out[e] = s;
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

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
        {{2, 96, 32, 2, 512}, pair_kernel_occ<PackedBody<D, 2, true>, 96, 32, 5>},
        {{2, 128, 64, 2, 512}, pair_kernel_occ<PackedBody<D, 2, true>, 128, 64, 4>},
        {{4, 64, 64, 2, 512}, pair_kernel_occ<PackedBody<D, 4, true>, 64, 64, 4>},
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

// Problems with a weighted source whose sym(Sigma_x^-1) has no Cholesky factor (an indefinite
// inverse covariance: not a covariance, but the reference evaluates it) run the packed kernels on
// the Horner form of k B_i instead, whatever shape is pinned.
template <int D>
static const Variant& adjoint_fallback()
{
    static const Variant v = {{4, 64, 64, 2, 512}, pair_kernel_occ<PackedBody<D, 4, true, false>, 64, 64, 4>};
    return v;
}
template <int D>
static const Variant& energy_fallback()
{
    static const Variant v = {{4, 128, 32, 2}, pair_kernel<PackedBody<D, 4, false, false>, 128, 32>};
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
                        cudaStream_t s, const float* w_stationary, bool counter_zeroed, double* host_out)
{
    const int rows = i1 - i0;
    const int BI = sh.ipt * sh.nt;
    const int n_ib = (rows + BI - 1) / BI;
    const int total_tiles = (int)(yrec_size / sh.tj);
    const int resident = c.num_sms * occupancy_blocks(fn, sh.nt);
    const int target = 4 * resident;
    int n_jc = std::max(1, std::min(total_tiles, (target + n_ib - 1) / n_ib));
    // small problems: rather than many one-tile items (each pays the per-item set-up, FP64
    // contraction and block reduction), one wave of items that fills the resident blocks,
    // unless that makes items longer than 1/8 of the targets
    n_jc = std::min(n_jc, std::max(std::max(1, resident / n_ib), total_tiles / 8));
    if (sh.max_chunk > 0) n_jc = std::max(n_jc, (total_tiles * sh.tj + sh.max_chunk - 1) / sh.max_chunk);
    if (sh.min_chunk > 0) n_jc = std::min(n_jc, std::max(1, total_tiles * sh.tj / sh.min_chunk));
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
    a.wx = w_stationary ? w_stationary : c.wx;
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
    if (!counter_zeroed) DUGMA_CK(cudaMemsetAsync(c.counter, 0, sizeof(int), s));
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
    DUGMA_CK(launch_dependent(c.pdl, fn, grid, sh.nt, 0, s, a));
    if (ev1) DUGMA_CK(cudaEventRecord(ev1, s));
    if (out_dev)
        DUGMA_CK(launch_dependent(c.pdl, reduce_items_kernel, nv, 1024, 0, s, (const double*)a.partials, n_items, nv,
                                  out_dev, host_out, (const int*)c.err));
    if (dEdx_dev) {
        const size_t n = (size_t)rows * c.D;
        const int g = (int)std::min<size_t>((n + 255) / 256, (size_t)c.num_sms * 8);
        DUGMA_CK(launch_dependent(c.pdl, reduce_chunks_kernel, g, 256, 0, s, (const double*)a.dx_part, n_jc, n,
                                  dEdx_dev));
    }
    return DUGMA_OK;
}

int launch_pairs(Context& c, const double* pose_dev, int model, bool grad, int i0, int i1, double* out_dev,
                 double* dEdx_dev, cudaStream_t s, const KernelShape* force, const EvalIO* io)
{
    if (i0 < 0 || i1 > c.N || i0 >= i1) return set_error(DUGMA_ERR_ARG, "bad source row range [%d, %d)", i0, i1);
    if (model == DUGMA_MODEL_CONV) return conv_launch(c, pose_dev, grad, i0, i1, out_dev, dEdx_dev, s, force);
    if (model == DUGMA_MODEL_REF_F64) {
        if (grad)
            return set_error(DUGMA_ERR_ARG, "the FP64 reference-precision model has no adjoint (use the "
                                            "finite-difference gradient)");
        return ref64_launch(c, pose_dev, i0, i1, out_dev, s);
    }
    if (model != DUGMA_MODEL_REF) return set_error(DUGMA_ERR_ARG, "unknown model %d", model);
    const KernelShape want = force ? *force : (grad ? c.shape_adj : c.shape_energy);
    const std::vector<Variant>& vars =
        c.D == 3 ? (grad ? adjoint_variants<3>() : energy_variants<3>()) : (grad ? adjoint_variants<2>() : energy_variants<2>());
    const Variant* v = &vars[0];
    for (auto& cand : vars)
        if (cand.shape.same(want)) v = &cand;
    // the packed kernels read the Cholesky form of the source records when every weighted source
    // has a factor, else the Horner form
    bool xchol = v->shape.pack == 2;
    if (xchol && c.x_indef > 0) {
        v = c.D == 3 ? (grad ? &adjoint_fallback<3>() : &energy_fallback<3>())
                     : (grad ? &adjoint_fallback<2>() : &energy_fallback<2>());
        xchol = false;
    }
    // record layout: 0 scalar adjoint, 1 scalar Horner energy, 2 / 3 their packed-pair forms
    const int layout = (grad ? 0 : 1) + (v->shape.pack == 2 ? 2 : 0);
    if (io && (io->pv || io->pose_src) && !io->pose_out)
        return set_error(DUGMA_ERR_ARG, "a pose by value or from host memory needs a device pose block");
    if (io && io->pose_src) DUGMA_RET(launch_pose_in(c, io->pose_src, io->pose_out, s, true));
    const double* pose_read = io && io->pose_src ? io->pose_out : pose_dev;
    DUGMA_RET(launch_prologue(c, pose_read, layout, s, xchol, c.counter, io ? io->pv : nullptr,
                              io ? io->pose_out : nullptr, io && io->pv ? c.err : nullptr));
    const int nv = grad ? 1 + (c.D == 3 ? 6 : 3) : 1;
    return launch_pair_variant(c, v->fn, v->shape, c.xrec, c.yrec, (size_t)c.M_pad / v->shape.pack, nv, c.Lmax_y,
                               io && io->pose_out ? io->pose_out : pose_dev, i0, i1, out_dev,
                               grad ? dEdx_dev : nullptr, nullptr, 0, nullptr, s, nullptr, true,
                               io ? io->host_out : nullptr);
}

// ---------------------------------------------------------------------------
// Allocation-free fused adjoint.
//
// For callers that cannot allocate device memory while they evaluate: loops with a
// latency budget that must never enter an allocator, and host applications that own
// every device allocation themselves.  They pass the six input arrays and the output
// buffer; everything the evaluation needs besides them (per-pose records, normalised
// weights, work-queue counter, per-item partial sums, the device error word) lives in
// one file-scope device array of kNoAllocScratchBytes, which every GPU that loads this
// library holds until the process exits.  The context built here is marked no_alloc,
// so a launch that would need more scratch fails instead of allocating.
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

// the pair kernel ran with a zero weight offset: restore the 2^Lmax_y factor of every output;
// if a bounded wait of the pair kernel gave up (error word set), every output becomes NaN
__global__ void noalloc_scale_kernel(double* out, int n, const double* Lmax, const int* err)
{
    if (threadIdx.x < n) out[threadIdx.x] = *err ? (double)NAN : out[threadIdx.x] * exp2(*Lmax);
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
    DUGMA_CK(cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, dev));
    c.no_alloc = true;
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
    noalloc_scale_kernel<<<1, 32, 0, s>>>(out_dev, nv, Lm + 1, c.err);
    DUGMA_CK(cudaGetLastError());
    return DUGMA_OK;
}

// batch.cu -- many registration problems of uneven sizes, each with many multistart poses,
// evaluated (energy + pose gradient, REF model) in one persistent launch.
//
// A batch owns one context per problem (the init state of each cloud pair).  An evaluation
//   1. uploads the poses (problem p, pose q) -> pq = p * n_poses + q;
//   2. runs one prologue over all (pq, target) and (pq, source) pairs, writing paired
//      target records (YRec2) and source records per pq;
//   3. runs one persistent adjoint launch over a global list of work items
//      (pq, source block, target chunk) sorted by cost, largest first, handed out by an
//      atomic counter, each item reducing into its own partial slot;
//   4. sums each pq's item partials in a fixed order.
// Steps 2-4 are captured once as a CUDA graph per pose count and replayed afterwards.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "bodies.cuh"
#include "context.hpp"

namespace dugma {

// Tile shapes of the batched launch: sources per thread, threads per block, pair records per
// shared-memory tile, and pair records per work item (the chunk of a problem's targets one item
// covers).  dugma_batch_autotune times them on the caller's poses and keeps the fastest.
struct BatchShape {
    int ipt, nt, tj, chunk;
};

struct PQDesc {
    const float *x, *xinv, *lwx, *y, *yinv, *lwy, *wx;
    const double* ux;   // the problem's Cholesky factors (Cholesky-form source records) or null
    const double* pose;
    XRec* xrec;
    YRec2* yrec;
    double Lmax;
    int N, M, M_pad;
};

struct BatchItem {
    int pq, ib, tile0, ntiles;
};

// one block row per pq: targets (paired layout, kC' unmodified) then sources (the Cholesky form
// sqrt(|k| s) U_i when the descriptor carries factors, else the Horner form)
template <int D>
__global__ void batch_prologue_kernel(const PQDesc* __restrict__ desc, int max_span)
{
    constexpr int NS = Sym<D>::N;
    const PQDesc pd = desc[blockIdx.y];
    const double* pose = pd.pose;
    double R[9], t[3];
    for (int k = 0; k < D * D; ++k) R[k] = pose[k];
    for (int a = 0; a < D; ++a) t[a] = pose[kPoseT + a];
    const double s = 1.0 / pose[kPoseSig], ks = K_EXP2 * s;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < max_span; idx += gridDim.x * blockDim.x) {
        if (idx < pd.M_pad) {
            const int j = idx;
            float f[16];
            for (int q = 0; q < 16; ++q) f[q] = 0.f;
            f[3] = -INFINITY;
            f[13] = INFINITY;
            if (j < pd.M && pd.lwy[j] != -INFINITY) {
                double A[3][3], T[3][3];
                for (int a = 0; a < D; ++a) {
                    double v = R[a] * (double)pd.y[(size_t)j * D] + R[a + D] * (double)pd.y[(size_t)j * D + 1];
                    if (D == 3) v += R[a + 6] * (double)pd.y[(size_t)j * D + 2];
                    v += t[a];
                    const float hi = __double2float_rn(v);
                    f[a] = -hi;
                    f[4 + a] = -__double2float_rn(v - (double)hi);
                }
                f[3] = pd.lwy[j];
                f[13] = -pd.lwy[j];
                for (int r0 = 0; r0 < D; ++r0)
                    for (int c0 = 0; c0 < D; ++c0)
                        A[r0][c0] = 0.5 * ((double)pd.yinv[(size_t)j * D * D + r0 + D * c0] +
                                           (double)pd.yinv[(size_t)j * D * D + c0 + D * r0]);
                for (int r0 = 0; r0 < D; ++r0)
                    for (int c0 = 0; c0 < D; ++c0) {
                        double acc = 0;
                        for (int k = 0; k < D; ++k) acc += A[r0][k] * R[c0 + D * k];
                        T[r0][c0] = acc;
                    }
                for (int k = 0; k < NS; ++k) {
                    double acc = 0;
                    for (int q = 0; q < D; ++q) acc += R[Sym<D>::a(k) + D * q] * T[q][Sym<D>::b(k)];
                    f[7 + k] = __double2float_rn(ks * acc);
                }
            } else if (j < pd.M) {
                // neglected target: no contribution, but a finite position
                for (int a = 0; a < D; ++a) f[a] = -pd.y[(size_t)j * D + a];
            }
            float* base = reinterpret_cast<float*>(pd.yrec) + (size_t)(j >> 1) * 32 + (j & 1);
            for (int q = 0; q < 16; ++q) base[(q >> 1) * 4 + (q & 1) * 2] = f[q];
        }
        if (idx < pd.N) {
            const int i = idx;
            XRec r;
            float xv[3] = {0, 0, 0}, bp[6] = {0, 0, 0, 0, 0, 0};
            for (int a = 0; a < D; ++a) xv[a] = pd.x[(size_t)i * D + a];
            const float lw = pd.lwx[i];
            if (lw != -INFINITY && pd.ux) {
                const double r = sqrt(-ks);
                for (int k = 0; k < NS; ++k) bp[k] = __double2float_rn(r * pd.ux[(size_t)i * NS + k]);
            } else if (lw != -INFINITY)
                for (int k = 0; k < NS; ++k) {
                    const int ra = Sym<D>::a(k), rb = Sym<D>::b(k);
                    const double b = 0.5 * ((double)pd.xinv[(size_t)i * D * D + ra + D * rb] +
                                            (double)pd.xinv[(size_t)i * D * D + rb + D * ra]);
                    bp[k] = __double2float_rn(ks * b * (ra == rb ? 1.0 : 2.0));
                }
            r.v0 = make_float4(xv[0], xv[1], xv[2], lw);
            r.v1 = make_float4(0.f, 0.f, 0.f, 0.f);
            r.v2 = D == 3 ? make_float4(bp[0], bp[1], bp[2], bp[3]) : make_float4(bp[0], bp[1], bp[2], 0.f);
            r.v3 = D == 3 ? make_float4(bp[4], bp[5], 0.f, 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
            pd.xrec[i] = r;
        }
    }
}

// The persistent skeleton of run_pairs (pairs.cuh) with per-item problem/pose descriptors.
template <class Body, int NT, int TJ, int STAGES>
__global__ void __launch_bounds__(NT) batch_pairs_kernel(const PQDesc* __restrict__ desc,
                                                         const BatchItem* __restrict__ items, int n_items,
                                                         double* __restrict__ partials, int* counter, int* err)
{
    using Rec = typename Body::StreamRec;
    constexpr int NV = Body::NV;
    constexpr int BI = Body::IPT * NT;
    constexpr uint32_t kTileBytes = TJ * sizeof(Rec);
    __shared__ __align__(128) Rec ybuf[STAGES][TJ];
    __shared__ __align__(8) uint64_t bars[STAGES];
    __shared__ double red[NT / 32][NV];
    __shared__ int s_item;
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    __syncthreads();
    Body body;
    uint32_t tcount = 0;
    for (;;) {
        if (tid == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= n_items) break;
        const BatchItem it = items[item];
        const PQDesc pd = desc[it.pq];
        PairArgs a{};
        a.xrec = pd.xrec;
        a.yrec = pd.yrec;
        a.wx = pd.wx;
        a.pose = pd.pose;
        a.Lmax = pd.Lmax;
        a.N = pd.N;
        a.i0 = 0;
        a.i_end = pd.N;
        body.setup(a);
        const Rec* yg = reinterpret_cast<const Rec*>(pd.yrec);
        if (tid == 0)
            for (int k = 0; k < STAGES && k < it.ntiles; ++k) {
                const int st = (tcount + k) % STAGES;
                mbar_arrive_expect_tx(&bars[st], kTileBytes);
                bulk_g2s(&ybuf[st][0], yg + (size_t)(it.tile0 + k) * TJ, kTileBytes, &bars[st]);
            }
        for (int ii = 0; ii < Body::IPT; ++ii) body.load_src(a, ii, it.ib * BI + ii * NT + tid);
        body.zero_all();
        for (int k = 0; k < it.ntiles; ++k) {
            const uint32_t u = tcount + k;
            const int st = u % STAGES;
            const bool ok = mbar_wait_bounded(&bars[st], (u / STAGES) & 1u, err);
            const Rec* yb = ybuf[st];
#pragma unroll 4
            for (int jj = 0; jj < TJ; ++jj) body.consume(yb[jj], (it.tile0 + k) * TJ + jj);
            body.fold();
            if (__syncthreads_or(!ok)) {
                if (tid == 0)
                    for (int q = k; q < it.ntiles && q < k + STAGES; ++q) {
                        const uint32_t uq = tcount + q;
                        mbar_wait_bounded(&bars[uq % STAGES], (uq / STAGES) & 1u, nullptr);
                    }
                return;
            }
            if (tid == 0 && k + STAGES < it.ntiles) {
                mbar_arrive_expect_tx(&bars[st], kTileBytes);
                bulk_g2s(&ybuf[st][0], yg + (size_t)(it.tile0 + k + STAGES) * TJ, kTileBytes, &bars[st]);
            }
        }
        tcount += it.ntiles;
        double acc[NV];
        for (int v = 0; v < NV; ++v) acc[v] = 0.0;
        body.finish(a, 0, acc);
        block_sum<NV, NT>(acc, &red[0][0]);
        if (tid == 0)
            for (int v = 0; v < NV; ++v) partials[(size_t)item * 8 + v] = acc[v];
    }
}

// out[pq][v] = sum of the pq's item partials, in the fixed order of its item index list
__global__ void batch_reduce_kernel(const double* __restrict__ partials, const int* __restrict__ pq_start,
                                    const int* __restrict__ pq_items, int nv, double* __restrict__ out)
{
    __shared__ double red[128];
    const int pq = blockIdx.x;
    const int b = pq_start[pq], e = pq_start[pq + 1];
    for (int v = 0; v < nv; ++v) {
        double s = 0;
        for (int k = b + threadIdx.x; k < e; k += blockDim.x) s += partials[(size_t)pq_items[k] * 8 + v];
        red[threadIdx.x] = s;
        __syncthreads();
        for (int h = blockDim.x / 2; h > 0; h >>= 1) {
            if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[(size_t)pq * nv + v] = red[0];
        __syncthreads();
    }
}

using BatchKernelFn = void (*)(const PQDesc*, const BatchItem*, int, double*, int*, int*);
struct BatchVariant {
    BatchShape sh;
    BatchKernelFn chol, horner;   // Cholesky-form and Horner-form source records
};

template <int D, int IPT, int NT, int TJ>
static BatchVariant batch_variant(int chunk)
{
    return {{IPT, NT, TJ, chunk}, batch_pairs_kernel<PackedBody<D, IPT, true, true>, NT, TJ, 4>,
            batch_pairs_kernel<PackedBody<D, IPT, true, false>, NT, TJ, 4>};
}

template <int D>
static const std::vector<BatchVariant>& batch_variants()
{
    static const std::vector<BatchVariant> v = {
        batch_variant<D, 4, 64, 64>(512),  batch_variant<D, 4, 64, 64>(256), batch_variant<D, 4, 64, 64>(1024),
        batch_variant<D, 4, 64, 32>(256),  batch_variant<D, 2, 128, 64>(512), batch_variant<D, 2, 128, 32>(256),
    };
    return v;
}

static const BatchShape& batch_shape_of(int D, int k)
{
    return D == 3 ? batch_variants<3>()[k].sh : batch_variants<2>()[k].sh;
}

struct Batch {
    int D = 3, P = 0;
    int shape = 0;                    // index into batch_variants<D>()
    int prepared_shape = -1;          // the shape the pose-count state below was built for
    std::vector<float*> ptrs;          // 6 per problem
    std::vector<Context*> ctx;
    cudaStream_t stream = nullptr;
    // per pose-count state
    int n_poses = 0, n_items = 0, nv = 0;
    void* mem = nullptr;              // one allocation: poses, descriptors, records, items, partials, ...
    double* poses = nullptr;
    PQDesc* desc = nullptr;
    BatchItem* items = nullptr;
    int *pq_start = nullptr, *pq_items = nullptr, *counter = nullptr, *err = nullptr;
    double *partials = nullptr, *out = nullptr;
    double* host = nullptr;           // pinned: poses in, results out
    size_t host_doubles = 0;
    // optional device timing of each evaluation (dugma_batch_timing)
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> tevents;
    size_t tused = 0;
    int max_span = 0;
    bool chol = true;                 // every problem's weighted sources have Cholesky factors
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;

    void release_pose_state()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (mem) cudaFree(mem);
        if (host) cudaFreeHost(host);
        exec = nullptr;
        graph = nullptr;
        mem = nullptr;
        host = nullptr;
        n_poses = 0;
    }
};

static int batch_prepare(Batch& b, int n_poses)
{
    if (b.n_poses == n_poses && b.prepared_shape == b.shape) return DUGMA_OK;
    cudaStreamSynchronize(b.stream);
    b.release_pose_state();
    const int D = b.D, NG = D == 3 ? 6 : 3;
    b.nv = 1 + NG;
    const int n_pq = b.P * n_poses;
    const BatchShape& sh = batch_shape_of(D, b.shape);
    const int BI = sh.ipt * sh.nt;
    // sizes and the work list (cost = rows x tiles; largest first)
    std::vector<size_t> yoff(n_pq), xoff(n_pq);
    size_t ybytes = 0, xbytes = 0;
    std::vector<BatchItem> items;
    std::vector<double> cost;
    b.max_span = 0;
    for (int p = 0; p < b.P; ++p) {
        const Context& c = *b.ctx[p];
        const int total_tiles = c.M_pad / 2 / sh.tj;
        const int chunk_tiles = sh.chunk / sh.tj;
        b.max_span = std::max(b.max_span, std::max(c.M_pad, c.N));
        for (int q = 0; q < n_poses; ++q) {
            const int pq = p * n_poses + q;
            yoff[pq] = ybytes;
            ybytes += sizeof(YRec2) * (size_t)(c.M_pad / 2);
            xoff[pq] = xbytes;
            xbytes += sizeof(XRec) * (size_t)((c.N + 3) / 4 * 4);
            for (int ib = 0; ib * BI < c.N; ++ib)
                for (int t0 = 0; t0 < total_tiles; t0 += chunk_tiles) {
                    const int nt = std::min(chunk_tiles, total_tiles - t0);
                    items.push_back({pq, ib, t0, nt});
                    cost.push_back((double)std::min(BI, c.N - ib * BI) * nt);
                }
        }
    }
    std::vector<int> order(items.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b2) { return cost[a] > cost[b2]; });
    std::vector<BatchItem> sorted(items.size());
    for (size_t k = 0; k < order.size(); ++k) sorted[k] = items[order[k]];
    // per-pq item lists in sorted-position order (deterministic reduction order)
    std::vector<int> pq_start(n_pq + 1, 0), pq_items(sorted.size());
    for (const BatchItem& it : sorted) ++pq_start[it.pq + 1];
    for (int k = 0; k < n_pq; ++k) pq_start[k + 1] += pq_start[k];
    {
        std::vector<int> fill(pq_start.begin(), pq_start.end() - 1);
        for (size_t k = 0; k < sorted.size(); ++k) pq_items[fill[sorted[k].pq]++] = (int)k;
    }
    b.n_items = (int)sorted.size();
    // one device allocation for everything pose-dependent
    auto up = [](size_t v) { return (v + 255) / 256 * 256; };
    const size_t s_poses = up(sizeof(double) * 16 * n_pq), s_desc = up(sizeof(PQDesc) * n_pq),
                 s_items = up(sizeof(BatchItem) * sorted.size()), s_start = up(sizeof(int) * (n_pq + 1)),
                 s_list = up(sizeof(int) * sorted.size()), s_ctr = 256, s_part = up(sizeof(double) * 8 * sorted.size()),
                 s_out = up(sizeof(double) * b.nv * n_pq), s_y = up(ybytes), s_x = up(xbytes);
    const size_t total = s_poses + s_desc + s_items + s_start + s_list + s_ctr + s_part + s_out + s_y + s_x;
    if (cudaMalloc(&b.mem, total) != cudaSuccess) {
        cudaGetLastError();
        b.mem = nullptr;
        return set_error(DUGMA_ERR_NOMEM, "batch: cannot allocate %zu bytes", total);
    }
    char* m = static_cast<char*>(b.mem);
    b.poses = reinterpret_cast<double*>(m); m += s_poses;
    b.desc = reinterpret_cast<PQDesc*>(m); m += s_desc;
    b.items = reinterpret_cast<BatchItem*>(m); m += s_items;
    b.pq_start = reinterpret_cast<int*>(m); m += s_start;
    b.pq_items = reinterpret_cast<int*>(m); m += s_list;
    b.counter = reinterpret_cast<int*>(m);
    b.err = b.counter + 4; m += s_ctr;
    b.partials = reinterpret_cast<double*>(m); m += s_part;
    b.out = reinterpret_cast<double*>(m); m += s_out;
    char* ybase = m; m += s_y;
    char* xbase = m;
    std::vector<PQDesc> desc(n_pq);
    for (int p = 0; p < b.P; ++p) {
        const Context& c = *b.ctx[p];
        for (int q = 0; q < n_poses; ++q) {
            const int pq = p * n_poses + q;
            PQDesc& d = desc[pq];
            d.x = c.x;
            d.xinv = c.xinv;
            d.lwx = c.lwx;
            d.y = c.y;
            d.yinv = c.yinv;
            d.lwy = c.lwy;
            d.wx = c.wx;
            d.ux = b.chol ? c.ux : nullptr;
            d.pose = b.poses + 16 * (size_t)pq;
            d.xrec = reinterpret_cast<XRec*>(xbase + xoff[pq]);
            d.yrec = reinterpret_cast<YRec2*>(ybase + yoff[pq]);
            d.Lmax = c.Lmax_y;
            d.N = c.N;
            d.M = c.M;
            d.M_pad = c.M_pad;
        }
    }
    DUGMA_CK(cudaMemcpy(b.desc, desc.data(), sizeof(PQDesc) * n_pq, cudaMemcpyHostToDevice));
    DUGMA_CK(cudaMemcpy(b.items, sorted.data(), sizeof(BatchItem) * sorted.size(), cudaMemcpyHostToDevice));
    DUGMA_CK(cudaMemcpy(b.pq_start, pq_start.data(), sizeof(int) * (n_pq + 1), cudaMemcpyHostToDevice));
    DUGMA_CK(cudaMemcpy(b.pq_items, pq_items.data(), sizeof(int) * sorted.size(), cudaMemcpyHostToDevice));
    b.host_doubles = (size_t)n_pq * 16 + 16;
    if (cudaMallocHost((void**)&b.host, sizeof(double) * b.host_doubles) != cudaSuccess) {
        cudaGetLastError();
        b.host = nullptr;
        return set_error(DUGMA_ERR_NOMEM, "batch: pinned staging allocation failed");
    }
    b.n_poses = n_poses;
    b.prepared_shape = b.shape;
    return DUGMA_OK;
}

template <int D>
static int batch_enqueue(Batch& b, cudaStream_t s)
{
    const BatchVariant& var = batch_variants<D>()[b.shape];
    const BatchKernelFn fn = b.chol ? var.chol : var.horner;
    const int n_pq = b.P * b.n_poses;
    int sms = 148, per_sm = 1;
    DUGMA_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b.ctx[0]->dev));
    DUGMA_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, var.sh.nt, 0));
    const int grid = std::min(std::max(per_sm, 1) * sms, b.n_items);
    const int gx = std::min((b.max_span + 255) / 256, 64);
    batch_prologue_kernel<D><<<dim3(gx, n_pq), 256, 0, s>>>(b.desc, b.max_span);
    DUGMA_CK(cudaGetLastError());
    DUGMA_CK(cudaMemsetAsync(b.counter, 0, 8 * sizeof(int), s));
    fn<<<grid, var.sh.nt, 0, s>>>(b.desc, b.items, b.n_items, b.partials, b.counter, b.err);
    DUGMA_CK(cudaGetLastError());
    batch_reduce_kernel<<<n_pq, 128, 0, s>>>(b.partials, b.pq_start, b.pq_items, b.nv, b.out);
    DUGMA_CK(cudaGetLastError());
    return DUGMA_OK;
}

// Replays (or, the first time at this pose count and shape, runs eagerly and captures) one
// evaluation on the batch stream, with CUDA events around it when timing is on.
static int batch_launch(Batch& b)
{
    cudaEvent_t ev1 = nullptr;
    if (b.timing) {
        if (b.tused == b.tevents.size()) {
            cudaEvent_t e0, e1;
            DUGMA_CK(cudaEventCreate(&e0));
            DUGMA_CK(cudaEventCreate(&e1));
            b.tevents.push_back({e0, e1});
        }
        DUGMA_CK(cudaEventRecord(b.tevents[b.tused].first, b.stream));
        ev1 = b.tevents[b.tused].second;
        ++b.tused;
    }
    if (!b.exec) {
        DUGMA_RET(b.D == 3 ? batch_enqueue<3>(b, b.stream) : batch_enqueue<2>(b, b.stream));
        if (ev1) DUGMA_CK(cudaEventRecord(ev1, b.stream));
        DUGMA_CK(cudaStreamSynchronize(b.stream));
        DUGMA_CK(cudaStreamBeginCapture(b.stream, cudaStreamCaptureModeThreadLocal));
        const int rc = b.D == 3 ? batch_enqueue<3>(b, b.stream) : batch_enqueue<2>(b, b.stream);
        const cudaError_t e = cudaStreamEndCapture(b.stream, &b.graph);
        if (rc != DUGMA_OK || e != cudaSuccess) return rc != DUGMA_OK ? rc : set_error(DUGMA_ERR_CUDA, "batch capture failed");
        DUGMA_CK(cudaGraphInstantiate(&b.exec, b.graph, 0));
        return DUGMA_OK;
    }
    DUGMA_CK(cudaGraphLaunch(b.exec, b.stream));
    if (ev1) DUGMA_CK(cudaEventRecord(ev1, b.stream));
    return DUGMA_OK;
}

static int batch_eval(Batch& b, int n_poses, const double* poses, double* out)
{
    DUGMA_RET(batch_prepare(b, n_poses));
    const int n_pq = b.P * n_poses, D = b.D;
    for (int k = 0; k < n_pq; ++k) {
        double* h = b.host + 16 * (size_t)k;
        for (int q = 0; q < 16; ++q) h[q] = 0.0;
        const double* src = poses + 13 * (size_t)k;
        for (int q = 0; q < D * D; ++q) h[q] = src[q];
        for (int a = 0; a < D; ++a) h[kPoseT + a] = src[9 + a];
        h[kPoseSig] = src[12];
        if (!(src[12] > 0)) return set_error(DUGMA_ERR_ARG, "batch_energy_grad: sig of pose %d is not positive", k);
    }
    DUGMA_CK(cudaMemcpyAsync(b.poses, b.host, sizeof(double) * 16 * n_pq, cudaMemcpyHostToDevice, b.stream));
    DUGMA_RET(batch_launch(b));
    const int nv = b.nv;
    DUGMA_CK(cudaMemcpyAsync(out, b.out, sizeof(double) * nv * n_pq, cudaMemcpyDeviceToHost, b.stream));
    int err = 0;
    DUGMA_CK(cudaMemcpyAsync(b.host + 16 * (size_t)n_pq, b.err, sizeof(int), cudaMemcpyDeviceToHost, b.stream));
    DUGMA_CK(cudaStreamSynchronize(b.stream));
    memcpy(&err, b.host + 16 * (size_t)n_pq, sizeof(int));
    if (err) return set_error(DUGMA_ERR_TIMEOUT, "batch: a device wait gave up (0x%x)", err);
    return DUGMA_OK;
}

}  // namespace dugma

using namespace dugma;

extern "C" {

int dugma_batch_create(int n_problems, int D, const int* N, const int* M, const double* const* X,
                       const double* const* X_C, const double* const* Y, const double* const* Y_C, void** batch)
{
    if (n_problems < 1 || !N || !M || !X || !X_C || !Y || !Y_C || !batch)
        return set_error(DUGMA_ERR_ARG, "batch_create: bad arguments");
    if (D != 2 && D != 3) return set_error(DUGMA_ERR_ARG, "batch_create: D must be 2 or 3");
    Batch* b = new Batch;
    b->D = D;
    b->P = n_problems;
    b->ptrs.resize(6 * (size_t)n_problems);
    for (int p = 0; p < n_problems; ++p) {
        double ok = 0;
        const int rc = dugma_init(X[p], X_C[p], Y[p], Y_C[p], &ok, N[p], M[p], D, &b->ptrs[6 * (size_t)p]);
        if (rc != DUGMA_OK && rc != DUGMA_ERR_NONPD) {
            for (int k = 0; k < p; ++k) dugma_fr_m(&b->ptrs[6 * (size_t)k]);
            delete b;
            return rc;
        }
        b->ctx.push_back(find_context(&b->ptrs[6 * (size_t)p]));
        if (b->ctx.back()->x_indef > 0) b->chol = false;
    }
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
        for (int k = 0; k < n_problems; ++k) dugma_fr_m(&b->ptrs[6 * (size_t)k]);
        delete b;
        return set_error(DUGMA_ERR_CUDA, "batch_create: stream creation failed");
    }
    *batch = b;
    return DUGMA_OK;
}

int dugma_batch_energy_grad(void* batch, int n_poses, const double* poses, int model, double* out)
{
    Batch* b = static_cast<Batch*>(batch);
    if (!b || n_poses < 1 || !poses || !out) return set_error(DUGMA_ERR_ARG, "batch_energy_grad: bad arguments");
    if (model != DUGMA_MODEL_REF) return set_error(DUGMA_ERR_ARG, "batch_energy_grad: the batched path is REF only");
    return batch_eval(*b, n_poses, poses, out);
}

int dugma_batch_shapes(int* shapes, int max)
{
    const std::vector<BatchVariant>& v = batch_variants<3>();
    const int n = (int)v.size();
    for (int k = 0; k < n && k < max && shapes; ++k) {
        shapes[4 * k] = v[k].sh.ipt;
        shapes[4 * k + 1] = v[k].sh.nt;
        shapes[4 * k + 2] = v[k].sh.tj;
        shapes[4 * k + 3] = v[k].sh.chunk;
    }
    return n;
}

int dugma_batch_set_shape(void* batch, int ipt, int nt, int tj, int chunk)
{
    Batch* b = static_cast<Batch*>(batch);
    if (!b) return set_error(DUGMA_ERR_ARG, "batch_set_shape: null batch");
    const int n = (int)batch_variants<3>().size();
    for (int k = 0; k < n; ++k) {
        const BatchShape& sh = batch_shape_of(b->D, k);
        if (sh.ipt == ipt && sh.nt == nt && sh.tj == tj && sh.chunk == chunk) {
            b->shape = k;
            return DUGMA_OK;
        }
    }
    return set_error(DUGMA_ERR_ARG, "batch_set_shape: (%d, %d, %d, %d) is not a compiled shape", ipt, nt, tj, chunk);
}

int dugma_batch_get_shape(void* batch, int shape[4])
{
    Batch* b = static_cast<Batch*>(batch);
    if (!b || !shape) return set_error(DUGMA_ERR_ARG, "batch_get_shape: null argument");
    const BatchShape& sh = batch_shape_of(b->D, b->shape);
    shape[0] = sh.ipt;
    shape[1] = sh.nt;
    shape[2] = sh.tj;
    shape[3] = sh.chunk;
    return DUGMA_OK;
}

int dugma_batch_autotune(void* batch, int n_poses, const double* poses, char* report, size_t report_len)
{
    Batch* b = static_cast<Batch*>(batch);
    if (!b || n_poses < 1 || !poses) return set_error(DUGMA_ERR_ARG, "batch_autotune: bad arguments");
    const int nv = 1 + (b->D == 3 ? 6 : 3);
    std::vector<double> out((size_t)b->P * n_poses * nv);
    const int n = (int)batch_variants<3>().size();
    const bool was_timing = b->timing;
    const size_t was_used = b->tused;
    std::string rep;
    double best = 1e300;
    int best_k = b->shape;
    cudaEvent_t e0, e1;
    DUGMA_CK(cudaEventCreate(&e0));
    DUGMA_CK(cudaEventCreate(&e1));
    b->timing = false;
    int rc = DUGMA_OK;
    for (int k = 0; k < n && rc == DUGMA_OK; ++k) {
        b->shape = k;
        rc = batch_eval(*b, n_poses, poses, out.data());   // first run: prepares and captures
        if (rc != DUGMA_OK) break;
        const int reps = 2;
        float ms = 0;
        cudaEventRecord(e0, b->stream);
        for (int r = 0; r < reps && rc == DUGMA_OK; ++r) rc = batch_launch(*b);
        cudaEventRecord(e1, b->stream);
        if (rc != DUGMA_OK) break;
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
            rc = set_error(DUGMA_ERR_CUDA, "batch_autotune: event timing failed");
        ms /= reps;
        const BatchShape& sh = batch_shape_of(b->D, k);
        char buf[96];
        snprintf(buf, sizeof(buf), "%s(ipt=%d,nt=%d,tj=%d,chunk=%d):%.3fms", rep.empty() ? "" : " ", sh.ipt, sh.nt,
                 sh.tj, sh.chunk, ms);
        rep += buf;
        if (ms < best) {
            best = ms;
            best_k = k;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->timing = was_timing;
    b->tused = was_used;
    b->shape = best_k;
    if (rc != DUGMA_OK) return rc;
    if (report && report_len) snprintf(report, report_len, "%s", rep.c_str());
    return DUGMA_OK;
}

int dugma_batch_timing(void* batch, int mode, double* total_ms, int* launches)
{
    Batch* b = static_cast<Batch*>(batch);
    if (!b) return set_error(DUGMA_ERR_ARG, "batch_timing: null batch");
    if (mode == 1) {
        b->timing = true;
        b->tused = 0;
        return DUGMA_OK;
    }
    if (mode == 0) {
        b->timing = false;
        return DUGMA_OK;
    }
    if (mode != 2) return set_error(DUGMA_ERR_ARG, "batch_timing: mode must be 0, 1 or 2");
    double tot = 0;
    for (size_t k = 0; k < b->tused; ++k) {
        DUGMA_CK(cudaEventSynchronize(b->tevents[k].second));
        float ms = 0;
        DUGMA_CK(cudaEventElapsedTime(&ms, b->tevents[k].first, b->tevents[k].second));
        tot += ms;
    }
    if (total_ms) *total_ms = tot;
    if (launches) *launches = (int)b->tused;
    return DUGMA_OK;
}

int dugma_batch_destroy(void* batch)
{
    Batch* b = static_cast<Batch*>(batch);
    if (!b) return set_error(DUGMA_ERR_ARG, "batch_destroy: null batch");
    if (b->stream) cudaStreamSynchronize(b->stream);
    b->release_pose_state();
    for (int p = 0; p < b->P; ++p) dugma_fr_m(&b->ptrs[6 * (size_t)p]);
    if (b->stream) cudaStreamDestroy(b->stream);
    for (auto& e : b->tevents) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    delete b;
    return DUGMA_OK;
}

}  // extern "C"

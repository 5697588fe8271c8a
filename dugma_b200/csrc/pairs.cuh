// pairs.cuh -- persistent all-pairs skeleton shared by the energy, adjoint, CONV and
// coefficient kernels.
//
// Work is a grid of (source block, target chunk) items handed out by an atomic
// counter.  A block keeps IPT source points per thread in registers and streams the
// chunk's target records through shared memory in tiles of TJ records, moved by the
// bulk-copy (TMA) engine into a STAGES-deep ring completed on mbarriers (bounded
// waits).  Each item's contribution is reduced over the block in FP64 in a fixed order
// and written to its own partial slot, so results do not depend on scheduling.
#pragma once

#include <type_traits>
#include <utility>

#include "common.cuh"

namespace dugma {

struct PairArgs {
    const void* xrec;      // source records (XRec or Rec128), N_pad of them
    const void* yrec;      // target records (YRec or Rec128), M_pad of them
    const float* wx;       // |Sigma_x|^-1/2 per source (FP32 state)
    const float* wy;       // |Sigma_y|^-1/2 per target
    const float* xcov;     // packed FP32 covariances (CONV)
    const float* ycov;
    const double* pose;    // R, t, sig
    double Lmax;           // REF: log2 weight offset of the streamed side; CONV: covariance scale
    int N;                 // number of real source rows
    int i0, i_end;         // source row range [i0, i_end)
    int n_ib, n_jc, jc_tiles, total_tiles;
    double* partials;      // [n_items][8]
    double* dx_part;       // [n_jc][i_end - i0][D] or nullptr
    double* h_part;        // coefficient passes: [n_jc][rows][16] or nullptr
    int* counter;
    int* err;
};

// Bodies with a fold_tile(tile, first record index, records) member finish each tile with the
// tile still in shared memory (work deferred out of the per-record loop); the others have fold().
template <class B, class R, class = void>
struct HasTileFold : std::false_type {};
template <class B, class R>
struct HasTileFold<B, R, std::void_t<decltype(std::declval<B&>().fold_tile(std::declval<const R*>(), 0, 0))>>
    : std::true_type {};

template <class Body, int NT, int TJ, int STAGES, int UNROLL = 4>
__device__ __forceinline__ void run_pairs(const PairArgs& a, Body& body)
{
    using Rec = typename Body::StreamRec;
    constexpr int NV = Body::NV;
    constexpr int BI = Body::IPT * NT;
    constexpr uint32_t kTileBytes = TJ * sizeof(Rec);
    static_assert(kTileBytes % 16 == 0, "bulk copies move multiples of 16 bytes");

    __shared__ __align__(128) Rec ybuf[STAGES][TJ];
    __shared__ __align__(8) uint64_t bars[STAGES];
    __shared__ double red[NT / 32][NV];
    __shared__ int s_item;

    // launched as a dependent of the prologue (and the reductions as dependents of this kernel):
    // let them be scheduled, then wait for the prologue's records, pose and zeroed counter
    pdl_trigger();
    pdl_wait();
    const int tid = threadIdx.x;
    if (tid == 0) {
#pragma unroll
        for (int s = 0; s < STAGES; ++s) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    __syncthreads();
    body.setup(a);

    const Rec* yg = static_cast<const Rec*>(a.yrec);
    const int n_items = a.n_ib * a.n_jc;
    uint32_t tcount = 0;
    for (;;) {
        if (tid == 0) s_item = atomicAdd(a.counter, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= n_items) break;
        const int ib = item % a.n_ib, jc = item / a.n_ib;
        const int tile0 = jc * a.jc_tiles;
        const int ntiles = min(a.jc_tiles, a.total_tiles - tile0);
        if (tid == 0) {
            for (int k = 0; k < STAGES && k < ntiles; ++k) {
                const int st = (tcount + k) % STAGES;
                mbar_arrive_expect_tx(&bars[st], kTileBytes);
                bulk_g2s(&ybuf[st][0], yg + (size_t)(tile0 + k) * TJ, kTileBytes, &bars[st]);
            }
        }
#pragma unroll
        for (int ii = 0; ii < Body::IPT; ++ii) body.load_src(a, ii, a.i0 + ib * BI + ii * NT + tid);
        body.zero_all();
        for (int k = 0; k < ntiles; ++k) {
            const uint32_t u = tcount + k;
            const int st = u % STAGES;
            const bool ok = mbar_wait_bounded(&bars[st], (u / STAGES) & 1u, a.err);
            const Rec* yb = ybuf[st];
#pragma unroll UNROLL
            for (int jj = 0; jj < TJ; ++jj) body.consume(yb[jj], (tile0 + k) * TJ + jj);
            if constexpr (HasTileFold<Body, Rec>::value)
                body.fold_tile(yb, (tile0 + k) * TJ, TJ);
            else
                body.fold();
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
        }
        tcount += ntiles;
        double acc[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) acc[v] = 0.0;
        body.finish(a, jc, acc);
        block_sum<NV, NT>(acc, &red[0][0]);
        if (tid == 0)
#pragma unroll
            for (int v = 0; v < NV; ++v) a.partials[(size_t)item * 8 + v] = acc[v];
    }
}

}  // namespace dugma

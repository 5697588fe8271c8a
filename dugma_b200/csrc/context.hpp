// context.hpp -- per-init device state of the DUGMA library.
//
// The reference keeps N, M, D, R, t and sigma in per-module __constant__ memory and
// is therefore not re-entrant (compi.cu:14-16, update_sig.cu:15-16, init.cu:10).
// Here every dugma_init creates a Context that owns its buffers and a stream; it is
// found again from the Ptr[6] the caller passes back (keyed by Ptr[0]).
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "dugma.h"

namespace dugma {

// Pose block on the device: R (D x D col-major, zero padded to 9), t (3), sig, pad.
constexpr int kPoseDoubles = 16;
constexpr int kMaxPoses = 16;     // device pose slots of a context (the finite-difference stencil)
constexpr int kPoseT = 9;
constexpr int kPoseSig = 12;

constexpr int kHostDoubles = 1024;
constexpr int kPadI = 1024;   // source rows padded to a multiple (largest i-block)
constexpr int kPadJ = 128;    // target rows padded to a multiple (largest j-tile)
constexpr int kMomSlots = 512;   // doubles in Context::mom (moments; block partials during init)
constexpr int kNumMomentsMax = 270;   // surrogate moments of the 3D coefficients (the 2D ones: 66)

// A pose block handed to a kernel by value (no copy to the device before the launch).
struct PoseBlock {
    double v[kPoseDoubles];
};

struct KernelShape {
    int ipt = 0;      // source points per thread
    int nt = 0;       // threads per block
    int tj = 0;       // streamed records per shared-memory tile
    int pack = 1;     // targets per streamed record (2: packed f32x2 kernels on pair records)
    int max_chunk = 0;   // most streamed records one work item may cover (0: no limit)
    int min_chunk = 0;   // fewest streamed records per work item (0: no limit); bounds the
                         // per-chunk partial buffers of the coefficient passes
    bool valid() const { return ipt > 0; }
    bool same(const KernelShape& o) const { return ipt == o.ipt && nt == o.nt && tj == o.tj && pack == o.pack; }
};

struct Context {
    int N = 0, M = 0, D = 0, dev = 0;
    int N_pad = 0, M_pad = 0;
    int nonpd = 0;
    // reference state (Ptr[0..5])
    float *x = nullptr, *xinv = nullptr, *y = nullptr, *yinv = nullptr, *wx = nullptr, *wy = nullptr;
    // extra state
    float *xcov = nullptr, *ycov = nullptr;   // packed symmetric FP32 covariances (CONV model)
    float *lwx = nullptr, *lwy = nullptr;     // log2(w) - Lmax, -inf when neglected
    double* ux = nullptr;                     // upper Cholesky factor of sym(Sigma_x^-1) per source (packed,
                                              // FP64); zero for neglected and not positive definite sources
    int x_indef = 0;                          // weighted sources whose sym(Sigma_x^-1) is not positive definite
    int y_indef = 0;                          // weighted targets whose sym(Sigma_y^-1) is not positive definite
    double Lmax_x = 0, Lmax_y = 0;
    double cscale = 1.0;                      // CONV covariances are stored divided by this
    // per-evaluation records
    YRec* yrec = nullptr;
    XRec* xrec = nullptr;
    Rec128* yrec128 = nullptr;
    Rec128* xrec128 = nullptr;
    void* yrec256 = nullptr;                  // the 128-byte records paired (coefficient passes)
    void* xrec256 = nullptr;
    float4* yp32 = nullptr;                   // -float(y') for nearest neighbours, pair-interleaved
    float* dmin = nullptr;                    // nearest squared distance per source (sigma)
    double* pose = nullptr;                   // kPoseDoubles
    double* poses = nullptr;                  // kMaxPoses x kPoseDoubles
    double* out = nullptr;                    // 64 doubles of results
    int* err = nullptr;                       // device error word
    int* counter = nullptr;                   // work-queue counters (8)
    double* dedx = nullptr;                   // dE/dx rows (allocated on first request)
    double* mom = nullptr;                    // surrogate moments (512 doubles)
    double* mom_part = nullptr;               // per-block moment partials (with the 128-byte records)
    // scratch: a region of the arena, replaced by a separate allocation if a launch needs more
    void* arena = nullptr;                    // one allocation for every buffer above
    size_t arena_bytes = 0;
    double* arena_scratch = nullptr;
    size_t arena_scratch_bytes = 0;
    void* scratch_extra = nullptr;
    double* scratch = nullptr;
    size_t scratch_bytes = 0;
    bool no_alloc = false;                    // scratch is fixed: ensure_scratch fails rather than allocating
    bool fused_coef = true;                   // compi over all rows in one pass (false: one pass per side)
    bool pdl = true;                          // a call's dependent kernels launched early (programmatic dependent launch)
    int coef_kernel = 0;                      // the one pass: 0 FP32 pipe only (the fastest); 1 source-side
                                              // sums on the tensor cores
    int coef_grid[4] = {0, 0, 0, 0};          // that pass's work grid (SB, groups, chunk tiles, chunks), set on first use
    // pinned host staging
    // [0,16) pose, [63] error word, [64,128) results, [256,512) multi-pose staging
    double* host = nullptr;                   // kHostDoubles doubles
    double* host_dev = nullptr;               // the same memory as the device addresses it (null: not mapped)
    cudaStream_t stream = nullptr;
    int num_sms = 148;
    KernelShape shape_adj, shape_energy, shape_nn, shape_conv_adj, shape_conv_energy;
    std::mutex mu;                            // one host call at a time per context
    // optional timing of the main pairwise kernel (dugma_timing)
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> tevents;
    size_t tused = 0;

    int ensure_scratch(size_t bytes);
    int ensure_coef_records();
};

// registry
Context* find_context(float* const* Ptr);
void register_context(Context* c);
void unregister_context(Context* c);

// errors (thread-local message)
int set_error(int code, const char* fmt, ...);
const char* last_error();

#define DUGMA_CK(call)                                                                    \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return ::dugma::set_error(DUGMA_ERR_CUDA, "%s failed: %s (%s:%d)", #call,     \
                                      cudaGetErrorString(e_), __FILE__, __LINE__);        \
    } while (0)

#define DUGMA_RET(call)           \
    do {                          \
        int r_ = (call);          \
        if (r_ != DUGMA_OK) return r_; \
    } while (0)

// ---- kernel launchers (energy.cu, nn.cu, coef.cu) ----
struct PairArgs;
using KernelFn = void (*)(PairArgs);
// One persistent all-pairs launch of `fn` (a run_pairs kernel of shape `sh`): source rows
// [i0, i1) of the stationary records `xrec` against `yrec_size` streamed records `yrec`,
// then, if out_dev, the fixed-order sum of the nv per-item partials into out_dev, and, if
// dEdx_dev, the per-row sums over target chunks.  h_part (nullable) receives the per-chunk
// row buffer of h_width doubles per row, n_jc_out the chunk count.  The stationary side's
// weights are c.wx unless w_stationary is given (the coefficient pass over targets).
// counter_zeroed: a kernel before it on the stream zeroed c.counter (no memset issued); host_out
// (optional, mapped pinned memory): also receives out_dev's nv values and, behind them, the
// error word.
int launch_pair_variant(Context& c, KernelFn fn, const KernelShape& sh, const void* xrec, const void* yrec,
                        size_t yrec_size, int nv, double Lmax, const double* pose_dev, int i0, int i1,
                        double* out_dev, double* dEdx_dev, double** h_part, int h_width, int* n_jc_out,
                        cudaStream_t s, const float* w_stationary = nullptr, bool counter_zeroed = false,
                        double* host_out = nullptr);
// Nearest-neighbour prologue: only the target records of the search (c.yp32), y' = R y + t as the
// full prologue rounds it.  The pose is *pv when given (then also written to pose_dev), else read
// from pose_dev; reset_counter / reset_err (optional) are zeroed for the kernels that follow.
int launch_nn_prologue(Context& c, double* pose_dev, cudaStream_t s, const PoseBlock* pv, int* reset_counter,
                       int* reset_err);
// One small kernel: the pose block from src (device-visible memory, e.g. the mapped pinned staging
// a captured graph reads at each launch) into pose_dev, and the error word zeroed if reset_err.
int launch_pose_in(Context& c, const double* src, double* pose_dev, cudaStream_t s, bool reset_err);
// Per-evaluation prologue: y records (layout 0 = adjoint, 1 = Horner energy, 2 / 3 their paired
// forms), x records in the Cholesky form (xchol, from c.ux) or the Horner form; reset_counter and
// reset_err (optional) are zeroed for the kernels that follow; the pose is *pv when given (and then
// also written to pose_out, if given), else read from pose_dev.
int launch_prologue(Context& c, const double* pose_dev, int ylayout, cudaStream_t s, bool xchol = false,
                    int* reset_counter = nullptr, const PoseBlock* pv = nullptr, double* pose_out = nullptr,
                    int* reset_err = nullptr);
// Pairwise energy (grad = false) or fused adjoint (grad = true) over source rows [i0, i1);
// writes {E, g} to out_dev and, if dEdx_dev, dE/dx for rows [i0, i1) (relative index).
// Options of an evaluation that issues no copy or memset (REF model).  The pose: *pv by value to the
// prologue (a single call), or loaded from pose_src (device-visible memory: the mapped pinned
// staging a captured graph reads at each launch) by a one-block kernel first; either way it is
// written to pose_out (the device pose block the pair kernel reads) and the error word is zeroed.
// The results (nv values) and, behind them, the error word are written to host_out (mapped pinned
// memory) as well.
struct EvalIO {
    const PoseBlock* pv = nullptr;
    const double* pose_src = nullptr;
    double* pose_out = nullptr;
    double* host_out = nullptr;
};
int launch_pairs(Context& c, const double* pose_dev, int model, bool grad, int i0, int i1,
                 double* out_dev, double* dEdx_dev, cudaStream_t s, const KernelShape* force = nullptr,
                 const EvalIO* io = nullptr);
// REF energy at the reference's FP64 per-pair precision (ref64.cu), sums to out_dev[0].
int ref64_launch(Context& c, const double* pose_dev, int i0, int i1, double* out_dev, cudaStream_t s);
// Nearest neighbours: writes idx/d2 (device) and optionally the per-point minimum only.
int launch_nn(Context& c, double* pose_dev, int k, int* idx_dev, float* d2_dev, cudaStream_t s,
              const KernelShape* force = nullptr);
// Options of a sigma evaluation, for a call that issues no copy or memset:
struct SigmaOpts {
    const PoseBlock* pose_value = nullptr;   // the pose by value to the first kernel (which also writes
                                             // it to pose_dev), instead of read from pose_dev
    const double* pose_src = nullptr;        // else the pose loaded into pose_dev first from
                                             // device-visible memory (the mapped staging a captured
                                             // graph reads at each launch)
    bool reset_err = false;                  // the first kernel zeroes the device error word
    double* host_out = nullptr;              // mapped pinned memory that also receives out_dev[0..1] and,
                                             // at [2], the error word
    double* pose_sig = nullptr;              // a device pose block whose sig receives out_dev[1]
};
// sigma: out_dev[0] = exact FP64 sigma, out_dev[1] = quantised (reference) sigma.  For a source
// row range [i0, i1) (i1 >= 0) the partial sums instead: out_dev[0] = sum of the nearest squared
// distances, out_dev[1] = sum of the reference's quantised terms (an integer below 2^53).
int launch_sigma(Context& c, double* pose_dev, double* out_dev, cudaStream_t s, int i0 = 0, int i1 = -1,
                 const SigmaOpts& opts = SigmaOpts());
// Surrogate coefficient moments: out_dev receives kNumMoments doubles.
// Source rows [i0, i1) carry the source-side (B) terms, target rows [j0, j1) the target-side
// (C') terms; -1 for i1 / j1 means all rows.  Sums over partitions of both add up to the whole.
struct CoefOpts {
    bool reset_err = false;              // the first kernel zeroes the device error word (no memset issued)
    const double* pose_value = nullptr;  // a host pose block handed to the first kernel by value; that
                                         // kernel writes it to pose_dev for the others (no copy issued)
    double* host_moments = nullptr;      // device-visible pinned host memory that also receives the moments
                                         // and, after them, the error word (no copy back issued)
};
int launch_coef(Context& c, double* pose_dev, double* moments_dev, cudaStream_t s, int i0 = 0, int i1 = -1,
                int j0 = 0, int j1 = -1, const CoefOpts& opts = CoefOpts());
int coef_from_moments(int D, const double* moments, double* coef640);
int num_moments(int D);

// init kernels
int launch_init(Context& c, const double* X, const double* XC, const double* Y, const double* YC);

// candidate kernel shapes for the autotuner
std::vector<KernelShape> adjoint_shapes();
std::vector<KernelShape> energy_shapes();
std::vector<KernelShape> nn_shapes();
std::vector<KernelShape> conv_shapes(bool grad);

}  // namespace dugma

/*
 * dugma.h -- C ABI of libdugma_b200.so, the B200 (sm_100a) implementation of the
 * DUGMA registration hot path (Canpu999/DUGMA: init.cu, update_sig.cu, compi.cu,
 * fr_m.cu and their MEX gateways).
 *
 * Data layout (the MATLAB layout the reference's MEX gateways pass through):
 *   X, Y      D x N column-major doubles   = N points, D coordinates each, contiguous
 *   X_C, Y_C  D x (D*N) column-major doubles = one D x D column-major block per point
 *   R         D x D column-major doubles, applied to Y: y' = R y + t
 *   Ptr[6]    device pointers {x, x_cov_inv, y, y_cov_inv, det_x, det_y} (FP32), the
 *             reference's device state after init (init.cu:326-331); Ptr[4], Ptr[5]
 *             hold |Sigma|^-1/2 per point.
 * Every call returns a status (DUGMA_OK = 0) instead of exiting the process;
 * dugma_last_error() describes the last failure on the calling thread.
 * Pose gradients are g = [dE/domega (NR), dE/dt (D)] with the left perturbation
 * R <- exp([omega]x) R, t <- t + dt; NR = 3 in 3D, 1 in 2D.
 */
#ifndef DUGMA_H
#define DUGMA_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  They are also the bit positions of the device error word. */
enum {
    DUGMA_OK = 0,
    DUGMA_ERR_ARG = 1,     /* bad argument: sizes, D, null pointer, unknown context */
    DUGMA_ERR_CUDA = 2,    /* a CUDA runtime call failed */
    DUGMA_ERR_NONPD = 3,   /* warning: some covariances had det <= 0 and were neglected */
    DUGMA_ERR_TIMEOUT = 4, /* a bounded device wait gave up */
    DUGMA_ERR_NOMEM = 5,   /* device allocation failed */
    DUGMA_ERR_NUMERIC = 6, /* non-finite result */
    DUGMA_ERR_STATE = 7    /* call out of order (e.g. graph replay of a released graph) */
};

/* Per-pair models. */
enum {
    DUGMA_MODEL_REF = 0, /* the reference: w_i v_j [exp(-d'C'd/2) + exp(-d'Bd/2)] (compi.cu:753-772) */
    DUGMA_MODEL_CONV = 1, /* convolved GMM: N(d; 0, sig (R Sy R' + Sx)) with its own 3x3 inverse */
    DUGMA_MODEL_REF_F64 = 2 /* REF at the reference's per-pair precision (FP64 d, quadratic forms and exp,
                               compi.cu:732-772); energy only: its gradient is the finite-difference
                               plain form (dugma_energy_fd_grad) */
};

/* Largest supported cloud size (the reference stops at 3e6 points, compi.cu:535). */
#define DUGMA_MAX_POINTS 16777216

/* ---------------- reference entry points (C linkage) ---------------- */

/* Replaces init(X, X_C, Y, Y_C, Coef, N, M, D, Ptr) (init.cu:249-259, bound by init.cpp:9-19):
 * uploads both clouds, inverts each covariance, stores |Sigma|^-1/2; *Coef = 1 on success.
 * A covariance with det <= 0 is neglected exactly as init.cu:48-57 does (entries 1e5, weight 0)
 * and the call returns DUGMA_ERR_NONPD (a warning; the state is usable). */
int dugma_init(const double* X, const double* X_C, const double* Y, const double* Y_C,
               double* Coef, int N, int M, int D, float* Ptr[6]);

/* Replaces cpd(Ptr, R, t, N, M, D, float sig[1]) of update_sig.cu:319-321 (update_sig.cpp:7):
 * sig = mean_i min_j |x_i - (R y_j + t)|^2 / D, with the reference's 1e-6 quantisation. */
int dugma_update_sig(float* Ptr[6], const double* R, const double* t, const double* N,
                     const double* M, const double* D, float sig[1]);

/* Replaces cpd(Ptr, R, t, N, M, D, sig, double coefficient[640]) of compi.cu:511-513
 * (compi.cpp:7): the 637 (3D) / 45 (2D) surrogate coefficients in the energy3D.m /
 * energy2D.m monomial order; the remaining slots of the 640 are zero. */
int dugma_compi(float* Ptr[6], const double* R, const double* t, const double* N,
                const double* M, const double* D, const double* sig, double coefficient[640]);

/* Replaces fr_m(Ptr) (fr_m.cu:14-16): frees the six buffers and the context behind them.
 * Unlike the reference it does not call cudaDeviceReset (that would destroy every other
 * allocation of the process). */
int dugma_fr_m(float* Ptr[6]);

/* Message for the last non-OK status on this thread. */
const char* dugma_last_error(void);

/* ---------------- energy, adjoint, nearest neighbours ---------------- */

/* E(R, t) = sum_ij P_ij for `model`; sig is sigma-bar (update_sig output). */
int dugma_energy(float* Ptr[6], const double* R, const double* t, double sig, int model, double* E);

/* Fused adjoint: E and g (NR + D doubles) in one pass; dEdx (N*D doubles, nullable) = dE/dx_i. */
int dugma_energy_grad(float* Ptr[6], const double* R, const double* t, double sig, int model,
                      double* E, double* g, double* dEdx);

/* Same over source rows [i_begin, i_end) only (partial sums, for sharding the rows across GPUs). */
int dugma_energy_grad_range(float* Ptr[6], const double* R, const double* t, double sig, int model,
                            int i_begin, int i_end, double* E, double* g);

/* Partial surrogate coefficients for sharding compi across GPUs: the source-side terms of
 * source rows [i_begin, i_end) plus the target-side terms of target rows [j_begin, j_end).
 * The coefficients are sums over rows, so the partials of any partition of both ranges add
 * up to dugma_compi's (one all-reduce of 640 doubles).  No counterpart in the reference. */
int dugma_compi_range(float* Ptr[6], const double* R, const double* t, double sig, int i_begin, int i_end,
                      int j_begin, int j_end, double coefficient[640]);

/* The plain form: E plus central finite differences of step h over the NR + D pose
 * coordinates (1 + 2 (NR + D) energy evaluations). */
int dugma_energy_fd_grad(float* Ptr[6], const double* R, const double* t, double sig, int model,
                         double h, double* E, double* g);

/* k (1..16) nearest targets of every source point: idx (N*k, ascending distance, ties to the
 * lowest index) and squared distances d2 (N*k FP32, exactly
 * fmaf(dz,dz, fmaf(dy,dy, dx*dx)) with y' = float(FP64(R y + t))). */
int dugma_nn(float* Ptr[6], const double* R, const double* t, int k, int* idx, float* d2);

/* Data preparation: per-point covariance from the k (1..15) nearest other points (brute-force
 * self-join on the GPU): the sample covariance of the point and its neighbours (divided by k),
 * eigenvalues clamped to [lo, hi].  points: n x D (MATLAB layout); cov: n blocks of D x D. */
int dugma_knn_covariance(const double* points, int n, int D, int k, double lo, double hi, double* cov);

/* Partial sums behind sigma for source rows [i_begin, i_end), for sharding update_sig across
 * GPUs: sums[0] = sum of the nearest squared distances (FP64), sums[1] = sum of the reference's
 * quantised terms round(d2 / D * 1e6) (an exact integer).  Over a partition of the rows,
 * sigma = float(S1 / 1e6 / N) as update_sig returns it, and S0 / (D N) unquantised.
 * No counterpart in the reference. */
int dugma_sigma_range(float* Ptr[6], const double* R, const double* t, int i_begin, int i_end, double sums[2]);

/* sigma without quantisation (FP64 sum of the exact nearest squared distances / (D N)). */
int dugma_sigma(float* Ptr[6], const double* R, const double* t, double* sig);

/* ---------------- asynchronous device-side form (CUDA graphs, torch harness) ---------------- */

/* pose_dev: 16 doubles on the device {R (D*D col-major), pad to 9, t (3, 2D uses 2), sig}
 * laid out as R[0..8], t[9..11], sig[12]; out_dev: 1 + NR + D doubles on the device;
 * dEdx_dev: N*D doubles on the device or NULL.  Work is enqueued on `stream`
 * (a cudaStream_t, NULL = the context's stream) and the call returns without synchronising. */
int dugma_energy_grad_async(float* Ptr[6], const double* pose_dev, int model, double* out_dev,
                            double* dEdx_dev, void* stream);
int dugma_energy_async(float* Ptr[6], const double* pose_dev, int model, double* out_dev, void* stream);

/* Allocation-free fused adjoint.  No counterpart in the reference: it is for callers that
 * cannot allocate device memory while they evaluate — latency-bounded loops that must never
 * enter an allocator, and hosts that own every device allocation themselves.  The caller
 * passes the six input arrays in the order and layout of Ptr[6] after dugma_init (source
 * coordinates, source inverse covariances, target coordinates, target inverse covariances,
 * source |Sigma|^-1/2, target |Sigma|^-1/2; e.g. the Ptr[6] of an init done beforehand), the pose
 * block pose_dev (as dugma_energy_grad_async) and out_dev (1 + NR + D doubles on the
 * device); nothing is allocated.  All other working memory is one 4 MiB file-scope device
 * array that every GPU loading this library holds until exit, which limits N and M to 16384.
 * Larger sizes are rejected with DUGMA_ERR_ARG.  The first call on each device looks up that
 * array's device address (make the first call before any stream capture).  Every call
 * reuses the same array, so calls whose work overlaps on the GPU (other streams, other
 * threads) race; the array keeps the last call's contents and each call re-initialises what
 * it needs.  Work is enqueued on `stream` (a cudaStream_t; NULL = the legacy default stream)
 * and the call returns without synchronising, so device-side failures cannot be returned as
 * a status: if a bounded device wait gives up, every value written to out_dev is NaN. */
int dugma_energy_grad_noalloc(const float* x, const float* x_cov_inv, const float* y, const float* y_cov_inv,
                              const float* det_x, const float* det_y, int N, int M, int D,
                              const double* pose_dev, double* out_dev, void* stream);

/* ---------------- tuning and graphs ---------------- */

/* Times the kernel shapes of `what` (0 = adjoint, 1 = energy, 2 = nearest neighbour, 3 = CONV
 * adjoint, 4 = CONV energy) on this context and keeps the fastest; writes a one-line report
 * into `report` (may be NULL).  `model` selects REF or CONV for what = 0 and 1. */
int dugma_autotune(float* Ptr[6], int what, int model, char* report, size_t report_len);

/* Kernel shapes available for `what` (0 adjoint, 1 energy, 2 nearest neighbour, 3 CONV adjoint,
 * 4 CONV energy): writes up to
 * `max` tuples {source points per thread, threads per block, records per tile, targets per
 * record} into shapes[4 * k] and returns the count (negative status on error). */
int dugma_shapes(int what, int* shapes, int max);

/* The work grid compi's one-pass kernel uses for N sources and M targets when `resident` blocks
 * fit the GPU at once (148 SMs x 3 on a B200): grid = {source blocks of 256 per group, groups,
 * target tiles of 32 per chunk, chunks}; items = groups x chunks.  Host-only (no device work). */
int dugma_coef_work_grid(int N, int M, int resident, int grid[4]);

/* Pins the kernel shape used for `what` on this context (one of dugma_shapes' tuples). */
int dugma_set_shape(float* Ptr[6], int what, int ipt, int nt, int tj, int pack);

/* The kernel shape this context uses for `what`: shape[0..4) = {ipt, nt, tj, pack}. */
int dugma_get_shape(float* Ptr[6], int what, int shape[4]);

/* Captures one energy+gradient evaluation (prologue, pair kernel, reduction) as a CUDA graph
 * reading its pose from the context's pose buffer; dugma_graph_eval replays it for a new
 * pose and returns E and g. */
int dugma_graph_create(float* Ptr[6], int model, void** graph);
int dugma_graph_eval(void* graph, const double* R, const double* t, double sig, double* E, double* g);
int dugma_graph_destroy(void* graph);

/* One iteration of the reference's registration loop on the device as a captured CUDA graph:
 * update_sig at (R, t) (update_sig.cu:319-394, called at DUGMA.m:105), then compi at (R, t) and
 * that sigma (compi.cu:511-628, called at DUGMA.m:60 of the next iteration), with the sigma kept
 * on the device between them and one copy of sigma and the surrogate moments back per step.
 * sig[0] and coefficient[640] are what dugma_update_sig and then dugma_compi would return, bit
 * for bit.  Replaces the host round trip between the two reference calls; no counterpart in the
 * reference.  dugma_em_graph_create runs one step eagerly (at the identity pose) to size the
 * scratch, then captures; the graph reads the context's state, so it must be destroyed before
 * dugma_fr_m of that context. */
int dugma_em_graph_create(float* Ptr[6], void** graph);
int dugma_em_step(void* graph, const double* R, const double* t, float sig[1], double coefficient[640]);
int dugma_em_graph_destroy(void* graph);

/* ---------------- batched problems ---------------- */

/* Many independent registration problems of uneven sizes in one persistent launch.
 * Problem p has N[p] source and M[p] target points; X[p], X_C[p], Y[p], Y_C[p] as in dugma_init. */
int dugma_batch_create(int n_problems, int D, const int* N, const int* M, const double* const* X,
                       const double* const* X_C, const double* const* Y, const double* const* Y_C,
                       void** batch);
/* poses: n_problems * n_poses records of 13 doubles {R (9, col-major), t (3), sig};
 * out: n_problems * n_poses * (1 + NR + D) doubles {E, g}. */
int dugma_batch_energy_grad(void* batch, int n_poses, const double* poses, int model, double* out);
int dugma_batch_destroy(void* batch);

/* Tile shapes of the batched launch: writes up to `max` tuples {sources per thread, threads per
 * block, pair records per tile, pair records per work item} into shapes[4 * k] and returns the
 * count.  No counterpart in the reference (its kernels have one fixed 32 x 32 launch shape). */
int dugma_batch_shapes(int* shapes, int max);
int dugma_batch_set_shape(void* batch, int ipt, int nt, int tj, int chunk);
int dugma_batch_get_shape(void* batch, int shape[4]);
/* Times every batch shape on these poses (as dugma_batch_energy_grad takes them) and keeps the
 * fastest; writes a one-line report into `report` (may be NULL). */
int dugma_batch_autotune(void* batch, int n_poses, const double* poses, char* report, size_t report_len);
/* CUDA events around every batched evaluation on the device (the records' prologue, the
 * persistent pair launch and the per-pose reduction): mode 1 start and clear, 0 stop, 2
 * synchronise and report the summed duration in ms and the number of evaluations. */
int dugma_batch_timing(void* batch, int mode, double* total_ms, int* launches);

/* ---------------- registration driver ---------------- */

enum {
    DUGMA_DRIVE_REFERENCE = 0, /* DUGMA.m loop: compi -> minimise the surrogate on SO(D) -> update sig */
    DUGMA_DRIVE_DIRECT = 1     /* maximise E(R, t) with the fused adjoint, sig annealed by update_sig */
};

/* The registration loop of DUGMA.m:19-137 with a quasi-Newton solver in place of fmincon.
 * Inputs as dugma_init plus the initial pose (R0, t0) and the stopping rules of DUGMA.m:57.
 * Writes the final pose (denormalised, DUGMA.m:122) and stats[8] =
 * {iterations, final sigma, final energy, exit flag, seconds, evaluations, 0, 0}. */
int dugma_register(const double* X, const double* X_C, const double* Y, const double* Y_C, int N,
                   int M, int D, const double* R0, const double* t0, int max_iter,
                   double acc_rot, double acc_trans, double acc_sig, int mode, double* R_out,
                   double* t_out, double* stats);

/* ---------------- measurement ---------------- */

/* Records CUDA events around every launch of the main pairwise kernel on this context
 * (mode 1: start and clear, 0: stop, 2: synchronise and return the summed duration in ms
 * and the number of launches since mode 1). */
int dugma_timing(float* Ptr[6], int mode, double* total_ms, int* launches);

/* Measured peak of a GPU pipe on the current device: what = 0 FP32 fused multiply-add,
 * 1 SFU ex2, 2 packed f32x2 fused multiply-add; returns lane operations per second (and the
 * kernel time in ms). */
int dugma_calibrate(int what, double* lane_ops_per_s, double* ms);

/* Diagnostic of the failure path: every wait of the pair kernels on a shared-memory tile is
 * bounded; when it runs out the kernel sets DUGMA_ERR_TIMEOUT in the context's error word,
 * drains its copies and returns, and the host call reports DUGMA_ERR_TIMEOUT.  This runs one
 * such wait on an mbarrier that nothing completes, with `polls` (1 .. 2^20) polls, and sets
 * *timed_out = 1 when the wait gave up as designed; the device stays usable.  No counterpart
 * in the reference. */
int dugma_wait_selftest(int polls, int* timed_out);

/* The solver the driver uses in place of fmincon (DUGMA.m:73 with energy3D.m / fcontr3D.m;
 * 2D: DUGMA.m:65 with energy2D.m / fcontr2D.m): minimises Q(dR, dt) = sum_k A_k b_k(dR, dt) over
 * dR in SO(D) (dR = exp([w]x), 2D a rotation by theta) and dt, from dR = I, dt = 0.
 * A: the 637 (3D) / 45 (2D) coefficients of dugma_compi.  Writes dR (D x D col-major), dt,
 * the minimum value and an exit flag (> 0 converged, 0 iteration limit, < 0 failed). */
int dugma_minimise_surrogate(int D, const double* A, double* dR, double* dt, double* Qmin, int* exitflag);

/* Library build/version string. */
const char* dugma_version(void);

#ifdef __cplusplus
}
#endif

#endif /* DUGMA_H */

// api.cu -- the C ABI (include/dugma.h), the reference-signature C++ entry points
// (include/dugma_mex.hpp), contexts, CUDA graphs and the kernel-shape autotuner.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "context.hpp"
#include "dugma.h"
#include "dugma_mex.hpp"

namespace dugma {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_last_error;

int set_error(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

const char* last_error() { return g_last_error.c_str(); }

// ---------------------------------------------------------------------------
// registry (keyed by Ptr[0], the device address of the source coordinates)
// ---------------------------------------------------------------------------
static std::mutex g_reg_mu;
static std::unordered_map<const void*, Context*> g_reg;

Context* find_context(float* const* Ptr)
{
    if (!Ptr || !Ptr[0]) return nullptr;
    std::lock_guard<std::mutex> lk(g_reg_mu);
    auto it = g_reg.find(Ptr[0]);
    if (it == g_reg.end()) return nullptr;
    Context* c = it->second;
    // the caller must pass back the same six pointers init returned
    if (Ptr[1] != c->xinv || Ptr[2] != c->y || Ptr[3] != c->yinv || Ptr[4] != c->wx || Ptr[5] != c->wy) return nullptr;
    return c;
}

void register_context(Context* c)
{
    std::lock_guard<std::mutex> lk(g_reg_mu);
    g_reg[c->x] = c;
}

void unregister_context(Context* c)
{
    std::lock_guard<std::mutex> lk(g_reg_mu);
    g_reg.erase(c->x);
}

int Context::ensure_scratch(size_t bytes)
{
    if (bytes <= scratch_bytes) return DUGMA_OK;
    if (no_alloc)
        return set_error(DUGMA_ERR_STATE, "a launch needs %zu bytes of scratch beyond the fixed %zu bytes", bytes,
                         scratch_bytes);
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(stream, &cs);
    if (cs != cudaStreamCaptureStatusNone)
        return set_error(DUGMA_ERR_STATE, "scratch must be sized before graph capture (%zu > %zu bytes)", bytes,
                         scratch_bytes);
    DUGMA_CK(cudaStreamSynchronize(stream));
    if (scratch_extra) cudaFree(scratch_extra);
    scratch_extra = nullptr;
    const size_t want = std::max(bytes, 2 * scratch_bytes);
    if (cudaMalloc(&scratch_extra, want) != cudaSuccess) {
        cudaGetLastError();
        scratch_extra = nullptr;
        scratch = arena_scratch;
        scratch_bytes = arena_scratch_bytes;
        return set_error(DUGMA_ERR_NOMEM, "cannot allocate %zu bytes of scratch", want);
    }
    scratch = reinterpret_cast<double*>(scratch_extra);
    scratch_bytes = want;
    return DUGMA_OK;
}

// ---------------------------------------------------------------------------
// pinned host staging: a process-wide pool of fixed-size blocks, so that creating a
// context does not pay for a pinned allocation every time
// ---------------------------------------------------------------------------
static std::mutex g_pin_mu;
static std::vector<double*> g_pin_free;

static double* pinned_acquire()
{
    std::lock_guard<std::mutex> lk(g_pin_mu);
    if (g_pin_free.empty()) {
        constexpr int kSlab = 16;
        double* slab = nullptr;
        if (cudaMallocHost((void**)&slab, sizeof(double) * kHostDoubles * kSlab) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        for (int k = 0; k < kSlab; ++k) g_pin_free.push_back(slab + (size_t)k * kHostDoubles);
    }
    double* p = g_pin_free.back();
    g_pin_free.pop_back();
    return p;
}

static void pinned_release(double* p)
{
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_pin_mu);
    g_pin_free.push_back(p);
}

// ---------------------------------------------------------------------------
// device arenas of freed contexts are kept (per device, up to kArenaCacheBytes) and
// handed to the next init that fits, the way a caching allocator would
// ---------------------------------------------------------------------------
constexpr size_t kArenaCacheBytes = (size_t)8 << 30;
struct CachedArena {
    int dev;
    size_t bytes;
    void* p;
};
static std::mutex g_arena_mu;
static std::vector<CachedArena> g_arenas;
static size_t g_arena_bytes = 0;

static void* arena_acquire(int dev, size_t bytes, size_t* got)
{
    {
        std::lock_guard<std::mutex> lk(g_arena_mu);
        int best = -1;
        for (int k = 0; k < (int)g_arenas.size(); ++k) {
            const CachedArena& a = g_arenas[k];
            if (a.dev == dev && a.bytes >= bytes && a.bytes <= 2 * bytes + ((size_t)64 << 20) &&
                (best < 0 || a.bytes < g_arenas[best].bytes))
                best = k;
        }
        if (best >= 0) {
            void* p = g_arenas[best].p;
            *got = g_arenas[best].bytes;
            g_arena_bytes -= g_arenas[best].bytes;
            g_arenas.erase(g_arenas.begin() + best);
            return p;
        }
    }
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    *got = bytes;
    return p;
}

static void arena_release(int dev, void* p, size_t bytes)
{
    if (!p) return;
    {
        std::lock_guard<std::mutex> lk(g_arena_mu);
        if (g_arena_bytes + bytes <= kArenaCacheBytes) {
            g_arenas.push_back({dev, bytes, p});
            g_arena_bytes += bytes;
            return;
        }
    }
    cudaFree(p);
}

// streams of freed contexts are kept (per device, up to kStreamCache) for the next init
constexpr size_t kStreamCache = 16;
static std::mutex g_stream_mu;
static std::vector<std::pair<int, cudaStream_t>> g_streams;

static cudaError_t stream_acquire(int dev, cudaStream_t* s)
{
    {
        std::lock_guard<std::mutex> lk(g_stream_mu);
        for (size_t k = 0; k < g_streams.size(); ++k)
            if (g_streams[k].first == dev) {
                *s = g_streams[k].second;
                g_streams.erase(g_streams.begin() + k);
                return cudaSuccess;
            }
    }
    return cudaStreamCreateWithFlags(s, cudaStreamNonBlocking);
}

static void stream_release(int dev, cudaStream_t s)   // s has no pending work
{
    {
        std::lock_guard<std::mutex> lk(g_stream_mu);
        if (g_streams.size() < kStreamCache) {
            g_streams.push_back({dev, s});
            return;
        }
    }
    cudaStreamDestroy(s);
}

static void destroy_context(Context* c)
{
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    arena_release(c->dev, c->arena, c->arena_bytes);
    void* bufs[] = {c->scratch_extra, c->yrec128, c->xrec128, c->yrec256, c->xrec256, c->mom_part, c->dedx};
    for (void* b : bufs)
        if (b) cudaFree(b);
    pinned_release(c->host);
    for (auto& e : c->tevents) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    if (c->stream) stream_release(c->dev, c->stream);
    delete c;
}

// ---------------------------------------------------------------------------
// small host helpers
// ---------------------------------------------------------------------------
static int ng_of(int D) { return D == 3 ? 6 : 3; }

// writes the pose block {R (D x D col-major), t, sig} into host[0..15]
static void pack_pose(const Context& c, const double* R, const double* t, double sig, double* h)
{
    for (int k = 0; k < kPoseDoubles; ++k) h[k] = 0.0;
    for (int k = 0; k < c.D * c.D; ++k) h[k] = R[k];
    for (int a = 0; a < c.D; ++a) h[kPoseT + a] = t[a];
    h[kPoseSig] = sig;
}

static int upload_pose(Context& c, const double* R, const double* t, double sig)
{
    pack_pose(c, R, t, sig, c.host);
    DUGMA_CK(cudaMemcpyAsync(c.pose, c.host, sizeof(double) * kPoseDoubles, cudaMemcpyHostToDevice, c.stream));
    DUGMA_CK(cudaMemsetAsync(c.err, 0, sizeof(int), c.stream));
    return DUGMA_OK;
}

constexpr int kHostMoments = 512;   // c.host[512, 512 + moments): the moments copied back

// copies n doubles of results + the device error word back and checks both
static int fetch(Context& c, const double* dev, int n, double* dst)
{
    if (n > 0) DUGMA_CK(cudaMemcpyAsync(c.host + 64, dev, sizeof(double) * n, cudaMemcpyDeviceToHost, c.stream));
    DUGMA_CK(cudaMemcpyAsync(c.host + 63, c.err, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    DUGMA_CK(cudaStreamSynchronize(c.stream));
    int err = 0;
    memcpy(&err, c.host + 63, sizeof(int));
    if (err) return set_error(DUGMA_ERR_TIMEOUT, "a device wait gave up (error word 0x%x)", err);
    if (dst) memcpy(dst, c.host + 64, sizeof(double) * n);
    return DUGMA_OK;
}

// The surrogate moments for a compi call: the pose goes to the coefficient prologue by value,
// which also zeroes the error word, and the moments with the error word after them (the
// reduction writes it there) come back through the mapped pinned staging, or by one copy when it
// is not mapped.  Then the coefficients from the moments.
static int coef_call(Context& c, const double* R, const double* t, double sig, int i0, int i1, int j0, int j1,
                     double coefficient[640])
{
    pack_pose(c, R, t, sig, c.host);
    CoefOpts o;
    o.reset_err = true;
    o.pose_value = c.host;
    o.host_moments = c.host_dev ? c.host_dev + kHostMoments : nullptr;
    DUGMA_RET(launch_coef(c, c.pose, c.mom, c.stream, i0, i1, j0, j1, o));
    const int nm = num_moments(c.D);
    if (!o.host_moments)
        DUGMA_CK(cudaMemcpyAsync(c.host + kHostMoments, c.mom, sizeof(double) * (nm + 1), cudaMemcpyDeviceToHost,
                                 c.stream));
    DUGMA_CK(cudaStreamSynchronize(c.stream));
    const double err = c.host[kHostMoments + nm];
    if (err != 0.0) return set_error(DUGMA_ERR_TIMEOUT, "a device wait gave up (error word 0x%x)", (int)err);
    return coef_from_moments(c.D, c.host + kHostMoments, coefficient);
}

// The REF model's evaluation options that need no copy or memset (EvalIO), when the pinned
// staging is mapped: the pose by value (pv given: a single call) or loaded from host[0, 16) at
// each launch (a captured graph), the nv results and the error word to host[64, ...).
static bool mapped_io(const Context& c, int model, const PoseBlock* pv, EvalIO* io)
{
    if (!c.host_dev || model != DUGMA_MODEL_REF) return false;
    io->pv = pv;
    io->pose_src = pv ? nullptr : c.host_dev;
    io->pose_out = c.pose;
    io->host_out = c.host_dev + 64;
    return true;
}

// after a launch with mapped_io: the nv results once the stream is done, the error word checked
static int mapped_fetch(Context& c, int nv, double* dst)
{
    DUGMA_CK(cudaStreamSynchronize(c.stream));
    const double err = c.host[64 + nv];
    if (err != 0.0) return set_error(DUGMA_ERR_TIMEOUT, "a device wait gave up (error word 0x%x)", (int)err);
    memcpy(dst, c.host + 64, sizeof(double) * nv);
    return DUGMA_OK;
}

// sigma at a pose without copies or memsets: the pose goes to the search prologue by value (it
// also zeroes the error word), and the result with the error word behind it comes back through
// the mapped pinned staging, or by copies when it is not mapped.  o = (exact, quantised) sigma.
static int sigma_call(Context& c, const double* R, const double* t, double o[2])
{
    pack_pose(c, R, t, 1.0, c.host);
    PoseBlock pb;
    memcpy(pb.v, c.host, sizeof(pb.v));
    SigmaOpts so;
    so.pose_value = &pb;
    so.reset_err = true;
    so.host_out = c.host_dev ? c.host_dev + 64 : nullptr;
    DUGMA_RET(launch_sigma(c, c.pose, c.out, c.stream, 0, -1, so));
    if (!so.host_out) return fetch(c, c.out, 2, o);
    DUGMA_CK(cudaStreamSynchronize(c.stream));
    const double err = c.host[66];
    if (err != 0.0) return set_error(DUGMA_ERR_TIMEOUT, "a device wait gave up (error word 0x%x)", (int)err);
    o[0] = c.host[64];
    o[1] = c.host[65];
    return DUGMA_OK;
}

static bool check_sizes(const Context& c, const double* N, const double* M, const double* D)
{
    if (N && (int)*N != c.N) return false;
    if (M && (int)*M != c.M) return false;
    if (D && (int)*D != c.D) return false;
    return true;
}

static void rodrigues(const double w[3], double Rm[9] /* col-major */)
{
    const double th = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    double K[9] = {0, w[2], -w[1], -w[2], 0, w[0], w[1], -w[0], 0};   // col-major [w]x
    double K2[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += K[r + 3 * k] * K[k + 3 * c];
            K2[r + 3 * c] = s;
        }
    const double a = th < 1e-12 ? 1.0 : std::sin(th) / th;
    const double b = th < 1e-12 ? 0.5 : (1.0 - std::cos(th)) / (th * th);
    for (int k = 0; k < 9; ++k) Rm[k] = (k % 4 == 0 ? 1.0 : 0.0) + a * K[k] + b * K2[k];
}

// left-perturbed pose for finite differences: coordinate q of [omega (NR), t (D)] moved by h
static void perturb(int D, const double* R, const double* t, int q, double h, double* R2, double* t2)
{
    const int NR = D == 3 ? 3 : 1;
    for (int k = 0; k < D * D; ++k) R2[k] = R[k];
    for (int a = 0; a < D; ++a) t2[a] = t[a];
    if (q >= NR) {
        t2[q - NR] += h;
        return;
    }
    if (D == 2) {
        const double c = std::cos(h), s = std::sin(h);
        const double Q[4] = {c, s, -s, c};   // col-major
        for (int r = 0; r < 2; ++r)
            for (int cc = 0; cc < 2; ++cc) R2[r + 2 * cc] = Q[r] * R[2 * cc] + Q[r + 2] * R[1 + 2 * cc];
        return;
    }
    double w[3] = {0, 0, 0}, Q[9];
    w[q] = h;
    rodrigues(w, Q);
    for (int r = 0; r < 3; ++r)
        for (int cc = 0; cc < 3; ++cc) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += Q[r + 3 * k] * R[k + 3 * cc];
            R2[r + 3 * cc] = s;
        }
}

}  // namespace dugma

using namespace dugma;

#define GET_CTX(c, Ptr)                                                               \
    Context* c = find_context(Ptr);                                                   \
    if (!c) return set_error(DUGMA_ERR_ARG, "Ptr does not name a live dugma context"); \
    std::lock_guard<std::mutex> lk_(c->mu)

extern "C" {

const char* dugma_last_error(void) { return last_error(); }

const char* dugma_version(void) { return "dugma_b200 1.0 (sm_100a)"; }

int dugma_init(const double* X, const double* X_C, const double* Y, const double* Y_C, double* Coef, int N, int M,
               int D, float* Ptr[6])
{
    if (Coef) *Coef = 0;
    if (!X || !X_C || !Y || !Y_C || !Ptr) return set_error(DUGMA_ERR_ARG, "init: null argument");
    if (D != 2 && D != 3) return set_error(DUGMA_ERR_ARG, "init: D must be 2 or 3 (got %d)", D);
    if (N < 1 || M < 1 || N > DUGMA_MAX_POINTS || M > DUGMA_MAX_POINTS)
        return set_error(DUGMA_ERR_ARG, "init: N = %d, M = %d outside [1, %d]", N, M, DUGMA_MAX_POINTS);
    Context* c = new Context;
    c->N = N;
    c->M = M;
    c->D = D;
    c->N_pad = (N + kPadI - 1) / kPadI * kPadI;
    c->M_pad = (M + kPadJ - 1) / kPadJ * kPadJ;
    // packed f32x2 pair kernels by default (fastest on B200 in every tuning run so far)
    c->shape_adj = {4, 64, 64, 2, 512};
    c->shape_energy = {4, 128, 32, 2};
    c->shape_nn = {4, 128, 64};
    c->shape_conv_adj = {2, 64, 32, 2, 512};
    c->shape_conv_energy = {1, 128, 32, 2};
    int rc = DUGMA_OK;
    auto fail = [&](int code) {
        destroy_context(c);
        return code;
    };
    if (cudaGetDevice(&c->dev) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return set_error(DUGMA_ERR_CUDA, "init: no CUDA device");
    }
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->dev);
    if (stream_acquire(c->dev, &c->stream) != cudaSuccess)
        return fail(set_error(DUGMA_ERR_CUDA, "init: stream creation failed"));
    // One device arena holds every per-context buffer.  Its scratch region first receives
    // the FP64 host inputs during init and afterwards the kernels' partial sums.
    const int NS = D == 3 ? 6 : 3;
    const size_t staging = sizeof(double) * ((size_t)N * D * (D + 1) + (size_t)M * D * (D + 1));
    const size_t scratch_bytes = std::max(staging, (size_t)4 << 20);
    struct Slot {
        void** p;
        size_t bytes;
    };
    const Slot slots[] = {
        {(void**)&c->x, sizeof(float) * N * D},         {(void**)&c->xinv, sizeof(float) * N * D * D},
        {(void**)&c->y, sizeof(float) * M * D},         {(void**)&c->yinv, sizeof(float) * M * D * D},
        {(void**)&c->wx, sizeof(float) * N},            {(void**)&c->wy, sizeof(float) * M},
        {(void**)&c->xcov, sizeof(float) * N * NS},     {(void**)&c->ycov, sizeof(float) * M * NS},
        {(void**)&c->lwx, sizeof(float) * N},           {(void**)&c->lwy, sizeof(float) * M},
        {(void**)&c->ux, sizeof(double) * N * NS},
        {(void**)&c->yrec, sizeof(YRec) * c->M_pad},    {(void**)&c->xrec, sizeof(XRec) * c->N_pad},
        {(void**)&c->yp32, sizeof(float4) * c->M_pad},  {(void**)&c->dmin, sizeof(float) * N},
        {(void**)&c->pose, sizeof(double) * kPoseDoubles * 2}, {(void**)&c->out, sizeof(double) * 64},
        {(void**)&c->poses, sizeof(double) * kPoseDoubles * kMaxPoses},
        {(void**)&c->err, sizeof(int) * 4},             {(void**)&c->counter, sizeof(int) * 8},
        {(void**)&c->mom, sizeof(double) * kMomSlots},        {(void**)&c->arena_scratch, scratch_bytes},
    };
    auto up = [](size_t v) { return (v + 255) / 256 * 256; };
    size_t total = 0;
    for (const Slot& s : slots) total += up(s.bytes);
    c->arena = arena_acquire(c->dev, total, &c->arena_bytes);
    if (!c->arena) return fail(set_error(DUGMA_ERR_NOMEM, "init: cannot allocate %zu bytes of device memory", total));
    size_t off = 0;
    for (const Slot& s : slots) {
        *s.p = static_cast<char*>(c->arena) + off;
        off += up(s.bytes);
    }
    c->scratch = c->arena_scratch;
    c->scratch_bytes = c->arena_scratch_bytes = scratch_bytes;
    c->host = pinned_acquire();
    if (!c->host) return fail(set_error(DUGMA_ERR_NOMEM, "init: pinned staging allocation failed"));
    // the staging as the device addresses it; without it (not mapped, or DUGMA_NO_MAPPED_STAGING set
    // in the environment) poses and results travel by copies
    // compi's one-pass kernel (DUGMA_COEF_KERNEL = 0, the default: the FP32 pipe alone; 1: the
    // source-side sums on the tensor cores)
    const char* coef_k = getenv("DUGMA_COEF_KERNEL");
    if (coef_k && *coef_k >= '0' && *coef_k <= '1' && !coef_k[1]) c->coef_kernel = *coef_k - '0';
    // the kernels of a call each wait for the one before (DUGMA_NO_PDL set): no early launch
    const char* no_pdl = getenv("DUGMA_NO_PDL");
    c->pdl = !(no_pdl && *no_pdl && *no_pdl != '0');
    const char* no_map = getenv("DUGMA_NO_MAPPED_STAGING");
    if ((no_map && *no_map && *no_map != '0') ||
        cudaHostGetDevicePointer((void**)&c->host_dev, c->host, 0) != cudaSuccess) {
        c->host_dev = nullptr;
        cudaGetLastError();
    }
    if (cudaMemsetAsync(c->err, 0, sizeof(int) * 4, c->stream) != cudaSuccess)
        return fail(set_error(DUGMA_ERR_CUDA, "init: memset failed"));
    rc = launch_init(*c, X, X_C, Y, Y_C);
    if (rc != DUGMA_OK) return fail(rc);
    register_context(c);
    Ptr[0] = c->x;
    Ptr[1] = c->xinv;
    Ptr[2] = c->y;
    Ptr[3] = c->yinv;
    Ptr[4] = c->wx;
    Ptr[5] = c->wy;
    if (Coef) *Coef = 1;
    if (c->nonpd)
        return set_error(DUGMA_ERR_NONPD, "init: %d covariance(s) with det <= 0 were neglected", c->nonpd);
    return DUGMA_OK;
}

int dugma_fr_m(float* Ptr[6])
{
    Context* c = find_context(Ptr);
    if (!c) return set_error(DUGMA_ERR_ARG, "fr_m: Ptr does not name a live dugma context");
    unregister_context(c);
    {
        std::lock_guard<std::mutex> lk(c->mu);
    }
    destroy_context(c);
    return DUGMA_OK;
}

int dugma_update_sig(float* Ptr[6], const double* R, const double* t, const double* N, const double* M,
                     const double* D, float sig[1])
{
    if (!R || !t || !sig) return set_error(DUGMA_ERR_ARG, "update_sig: null argument");
    GET_CTX(c, Ptr);
    if (!check_sizes(*c, N, M, D)) return set_error(DUGMA_ERR_ARG, "update_sig: N, M, D differ from init");
    double o[2];
    DUGMA_RET(sigma_call(*c, R, t, o));
    sig[0] = (float)o[1];
    return DUGMA_OK;
}

int dugma_sigma(float* Ptr[6], const double* R, const double* t, double* sig)
{
    if (!R || !t || !sig) return set_error(DUGMA_ERR_ARG, "sigma: null argument");
    GET_CTX(c, Ptr);
    double o[2];
    DUGMA_RET(sigma_call(*c, R, t, o));
    *sig = o[0];
    return DUGMA_OK;
}

int dugma_sigma_range(float* Ptr[6], const double* R, const double* t, int i_begin, int i_end, double sums[2])
{
    if (!R || !t || !sums) return set_error(DUGMA_ERR_ARG, "sigma_range: null argument");
    GET_CTX(c, Ptr);
    if (i_begin < 0 || i_end > c->N || i_begin > i_end)
        return set_error(DUGMA_ERR_ARG, "sigma_range: bad source row range [%d, %d)", i_begin, i_end);
    if (i_begin == i_end) {
        sums[0] = sums[1] = 0.0;
        return DUGMA_OK;
    }
    DUGMA_RET(upload_pose(*c, R, t, 1.0));
    DUGMA_RET(launch_sigma(*c, c->pose, c->out, c->stream, i_begin, i_end));
    return fetch(*c, c->out, 2, sums);
}

int dugma_compi(float* Ptr[6], const double* R, const double* t, const double* N, const double* M, const double* D,
                const double* sig, double coefficient[640])
{
    if (!R || !t || !sig || !coefficient) return set_error(DUGMA_ERR_ARG, "compi: null argument");
    if (!(*sig > 0)) return set_error(DUGMA_ERR_ARG, "compi: sig must be positive");
    GET_CTX(c, Ptr);
    if (!check_sizes(*c, N, M, D)) return set_error(DUGMA_ERR_ARG, "compi: N, M, D differ from init");
    return coef_call(*c, R, t, *sig, 0, -1, 0, -1, coefficient);
}

int dugma_compi_range(float* Ptr[6], const double* R, const double* t, double sig, int i_begin, int i_end,
                      int j_begin, int j_end, double coefficient[640])
{
    if (!R || !t || !coefficient) return set_error(DUGMA_ERR_ARG, "compi_range: null argument");
    if (!(sig > 0)) return set_error(DUGMA_ERR_ARG, "compi_range: sig must be positive");
    GET_CTX(c, Ptr);
    if (i_begin < 0 || i_end > c->N || i_begin > i_end || j_begin < 0 || j_end > c->M || j_begin > j_end)
        return set_error(DUGMA_ERR_ARG, "compi_range: bad row ranges [%d, %d) x [%d, %d)", i_begin, i_end, j_begin,
                         j_end);
    return coef_call(*c, R, t, sig, i_begin, i_end, j_begin, j_end, coefficient);
}

int dugma_energy(float* Ptr[6], const double* R, const double* t, double sig, int model, double* E)
{
    if (!R || !t || !E) return set_error(DUGMA_ERR_ARG, "energy: null argument");
    if (!(sig > 0)) return set_error(DUGMA_ERR_ARG, "energy: sig must be positive");
    GET_CTX(c, Ptr);
    EvalIO io;
    PoseBlock pb;
    if (mapped_io(*c, model, &pb, &io)) {
        pack_pose(*c, R, t, sig, pb.v);
        DUGMA_RET(launch_pairs(*c, c->pose, model, false, 0, c->N, c->out, nullptr, c->stream, nullptr, &io));
        return mapped_fetch(*c, 1, E);
    }
    DUGMA_RET(upload_pose(*c, R, t, sig));
    DUGMA_RET(launch_pairs(*c, c->pose, model, false, 0, c->N, c->out, nullptr, c->stream));
    return fetch(*c, c->out, 1, E);
}

static int energy_grad_impl(Context* c, const double* R, const double* t, double sig, int model, int i0, int i1,
                            double* E, double* g, double* dEdx)
{
    const int ng = ng_of(c->D);
    double o[8];
    EvalIO io;
    PoseBlock pb;
    if (!dEdx && mapped_io(*c, model, &pb, &io)) {
        pack_pose(*c, R, t, sig, pb.v);
        DUGMA_RET(launch_pairs(*c, c->pose, model, true, i0, i1, c->out, nullptr, c->stream, nullptr, &io));
        DUGMA_RET(mapped_fetch(*c, 1 + ng, o));
    } else {
        DUGMA_RET(upload_pose(*c, R, t, sig));
        if (dEdx && !c->dedx) DUGMA_CK(cudaMalloc(&c->dedx, sizeof(double) * (size_t)c->N * c->D));
        DUGMA_RET(launch_pairs(*c, c->pose, model, true, i0, i1, c->out, dEdx ? c->dedx : nullptr, c->stream));
        if (dEdx)
            DUGMA_CK(cudaMemcpyAsync(dEdx, c->dedx, sizeof(double) * (size_t)(i1 - i0) * c->D, cudaMemcpyDeviceToHost,
                                     c->stream));
        DUGMA_RET(fetch(*c, c->out, 1 + ng, o));
    }
    if (E) *E = o[0];
    if (g) memcpy(g, o + 1, sizeof(double) * ng);
    if (!std::isfinite(o[0])) return set_error(DUGMA_ERR_NUMERIC, "energy is not finite");
    return DUGMA_OK;
}

int dugma_energy_grad(float* Ptr[6], const double* R, const double* t, double sig, int model, double* E, double* g,
                      double* dEdx)
{
    if (!R || !t || !E || !g) return set_error(DUGMA_ERR_ARG, "energy_grad: null argument");
    if (!(sig > 0)) return set_error(DUGMA_ERR_ARG, "energy_grad: sig must be positive");
    GET_CTX(c, Ptr);
    return energy_grad_impl(c, R, t, sig, model, 0, c->N, E, g, dEdx);
}

int dugma_energy_grad_range(float* Ptr[6], const double* R, const double* t, double sig, int model, int i_begin,
                            int i_end, double* E, double* g)
{
    if (!R || !t || !E || !g) return set_error(DUGMA_ERR_ARG, "energy_grad_range: null argument");
    if (!(sig > 0)) return set_error(DUGMA_ERR_ARG, "energy_grad_range: sig must be positive");
    GET_CTX(c, Ptr);
    if (i_begin < 0 || i_end > c->N || i_begin > i_end)
        return set_error(DUGMA_ERR_ARG, "energy_grad_range: [%d, %d) outside [0, %d)", i_begin, i_end, c->N);
    if (i_begin == i_end) {
        *E = 0;
        for (int k = 0; k < ng_of(c->D); ++k) g[k] = 0;
        return DUGMA_OK;
    }
    return energy_grad_impl(c, R, t, sig, model, i_begin, i_end, E, g, nullptr);
}

int dugma_energy_fd_grad(float* Ptr[6], const double* R, const double* t, double sig, int model, double h,
                         double* E, double* g)
{
    if (!R || !t || !E || !g) return set_error(DUGMA_ERR_ARG, "energy_fd_grad: null argument");
    if (!(sig > 0) || !(h > 0)) return set_error(DUGMA_ERR_ARG, "energy_fd_grad: sig and h must be positive");
    GET_CTX(c, Ptr);
    const int D = c->D, ng = ng_of(D), nev = 1 + 2 * ng;
    double* hp = c->host + 256;   // pinned staging for the 1 + 2 NG poses
    for (int k = 0; k < nev; ++k) {
        double R2[9], t2[3];
        if (k == 0) {
            memcpy(R2, R, sizeof(double) * D * D);
            memcpy(t2, t, sizeof(double) * D);
        } else {
            perturb(D, R, t, (k - 1) / 2, (k % 2) ? h : -h, R2, t2);
        }
        pack_pose(*c, R2, t2, sig, hp + 16 * k);
    }
    double* poses = c->poses;   // nev <= 13 <= kMaxPoses
    DUGMA_CK(cudaMemcpyAsync(poses, hp, sizeof(double) * 16 * nev, cudaMemcpyHostToDevice, c->stream));
    DUGMA_CK(cudaMemsetAsync(c->err, 0, sizeof(int), c->stream));
    int rc = DUGMA_OK;
    for (int k = 0; k < nev && rc == DUGMA_OK; ++k)
        rc = launch_pairs(*c, poses + 16 * k, model, false, 0, c->N, c->out + k, nullptr, c->stream);
    double ev[16];
    if (rc == DUGMA_OK) rc = fetch(*c, c->out, nev, ev);
    cudaStreamSynchronize(c->stream);
    if (rc != DUGMA_OK) return rc;
    *E = ev[0];
    for (int q = 0; q < ng; ++q) g[q] = (ev[1 + 2 * q] - ev[2 + 2 * q]) / (2.0 * h);
    return DUGMA_OK;
}

int dugma_nn(float* Ptr[6], const double* R, const double* t, int k, int* idx, float* d2)
{
    if (!R || !t || !idx || !d2) return set_error(DUGMA_ERR_ARG, "nn: null argument");
    GET_CTX(c, Ptr);
    if (k < 1 || k > 16 || k > c->M) return set_error(DUGMA_ERR_ARG, "nn: k = %d must be in [1, min(16, M)]", k);
    DUGMA_RET(upload_pose(*c, R, t, 1.0));
    int* di = nullptr;
    float* dd = nullptr;
    DUGMA_CK(cudaMallocAsync(&di, sizeof(int) * (size_t)c->N * k, c->stream));
    DUGMA_CK(cudaMallocAsync(&dd, sizeof(float) * (size_t)c->N * k, c->stream));
    int rc = launch_nn(*c, c->pose, k, di, dd, c->stream);
    if (rc == DUGMA_OK) {
        cudaMemcpyAsync(idx, di, sizeof(int) * (size_t)c->N * k, cudaMemcpyDeviceToHost, c->stream);
        cudaMemcpyAsync(d2, dd, sizeof(float) * (size_t)c->N * k, cudaMemcpyDeviceToHost, c->stream);
        rc = fetch(*c, c->out, 0, nullptr);
    }
    cudaFreeAsync(di, c->stream);
    cudaFreeAsync(dd, c->stream);
    cudaStreamSynchronize(c->stream);
    return rc;
}

int dugma_energy_grad_async(float* Ptr[6], const double* pose_dev, int model, double* out_dev, double* dEdx_dev,
                            void* stream)
{
    if (!pose_dev || !out_dev) return set_error(DUGMA_ERR_ARG, "energy_grad_async: null argument");
    GET_CTX(c, Ptr);
    cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
    return launch_pairs(*c, pose_dev, model, true, 0, c->N, out_dev, dEdx_dev, s);
}

int dugma_energy_async(float* Ptr[6], const double* pose_dev, int model, double* out_dev, void* stream)
{
    if (!pose_dev || !out_dev) return set_error(DUGMA_ERR_ARG, "energy_async: null argument");
    GET_CTX(c, Ptr);
    cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
    return launch_pairs(*c, pose_dev, model, false, 0, c->N, out_dev, nullptr, s);
}

// ---------------------------------------------------------------------------
// autotuner: time each candidate shape with CUDA events on the context stream
// ---------------------------------------------------------------------------
// kernel families that have tunable shapes: 0 adjoint, 1 energy, 2 nearest neighbour,
// 3 CONV adjoint, 4 CONV energy
static std::vector<KernelShape> shapes_of(int what)
{
    switch (what) {
    case 0: return adjoint_shapes();
    case 1: return energy_shapes();
    case 2: return nn_shapes();
    case 3: return conv_shapes(true);
    default: return conv_shapes(false);
    }
}

static KernelShape& shape_slot(Context& c, int what)
{
    switch (what) {
    case 0: return c.shape_adj;
    case 1: return c.shape_energy;
    case 2: return c.shape_nn;
    case 3: return c.shape_conv_adj;
    default: return c.shape_conv_energy;
    }
}

int dugma_autotune(float* Ptr[6], int what, int model, char* report, size_t report_len)
{
    GET_CTX(c, Ptr);
    if (what < 0 || what > 4) return set_error(DUGMA_ERR_ARG, "autotune: what must be 0 .. 4");
    std::vector<KernelShape> cand = shapes_of(what);
    // use the pose of the last call if there was one, else the identity at sig = 0.01
    DUGMA_CK(cudaMemcpyAsync(c->host, c->pose, sizeof(double) * kPoseDoubles, cudaMemcpyDeviceToHost, c->stream));
    DUGMA_CK(cudaStreamSynchronize(c->stream));
    if (!(c->host[kPoseSig] > 0)) {
        double Rm[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, R2[4] = {1, 0, 0, 1}, t0[3] = {0, 0, 0};
        DUGMA_RET(upload_pose(*c, c->D == 3 ? Rm : R2, t0, 1e-2));
    }
    cudaEvent_t e0, e1;
    DUGMA_CK(cudaEventCreate(&e0));
    DUGMA_CK(cudaEventCreate(&e1));
    std::string rep;
    float best = 1e30f;
    KernelShape best_shape = cand[0];
    int* di = nullptr;
    float* dd = nullptr;
    if (what == 2) {
        DUGMA_CK(cudaMalloc(&di, sizeof(int) * c->N));
        DUGMA_CK(cudaMalloc(&dd, sizeof(float) * c->N));
    }
    int rc = DUGMA_OK;
    for (auto& sh : cand) {
        auto run = [&]() {
            if (what == 2) return launch_nn(*c, c->pose, 1, di, dd, c->stream, &sh);
            if (what >= 3) return launch_pairs(*c, c->pose, DUGMA_MODEL_CONV, what == 3, 0, c->N, c->out, nullptr,
                                               c->stream, &sh);
            return launch_pairs(*c, c->pose, model, what == 0, 0, c->N, c->out, nullptr, c->stream, &sh);
        };
        rc = run();   // warm-up (also sizes scratch)
        if (rc != DUGMA_OK) break;
        const int reps = 3;
        cudaEventRecord(e0, c->stream);
        for (int r = 0; r < reps && rc == DUGMA_OK; ++r) rc = run();
        cudaEventRecord(e1, c->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) rc = set_error(DUGMA_ERR_CUDA, "autotune: sync failed");
        if (rc != DUGMA_OK) break;
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        ms /= reps;
        char buf[96];
        snprintf(buf, sizeof(buf), "%s(ipt=%d,nt=%d,tj=%d,pack=%d):%.3fms", rep.empty() ? "" : " ", sh.ipt, sh.nt,
                 sh.tj, sh.pack, ms);
        rep += buf;
        if (ms < best) {
            best = ms;
            best_shape = sh;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (di) cudaFree(di);
    if (dd) cudaFree(dd);
    if (rc != DUGMA_OK) return rc;
    shape_slot(*c, what) = best_shape;
    if (report && report_len) snprintf(report, report_len, "%s", rep.c_str());
    return DUGMA_OK;
}

int dugma_shapes(int what, int* shapes, int max)
{
    if (what < 0 || what > 4) return -set_error(DUGMA_ERR_ARG, "shapes: what must be 0 .. 4");
    std::vector<KernelShape> cand = shapes_of(what);
    const int n = (int)cand.size();
    for (int k = 0; k < n && k < max && shapes; ++k) {
        shapes[4 * k] = cand[k].ipt;
        shapes[4 * k + 1] = cand[k].nt;
        shapes[4 * k + 2] = cand[k].tj;
        shapes[4 * k + 3] = cand[k].pack;
    }
    return n;
}

int dugma_get_shape(float* Ptr[6], int what, int shape[4])
{
    GET_CTX(c, Ptr);
    if (what < 0 || what > 4 || !shape) return set_error(DUGMA_ERR_ARG, "get_shape: what must be 0 .. 4");
    const KernelShape& k = shape_slot(*c, what);
    shape[0] = k.ipt;
    shape[1] = k.nt;
    shape[2] = k.tj;
    shape[3] = k.pack;
    return DUGMA_OK;
}

int dugma_set_shape(float* Ptr[6], int what, int ipt, int nt, int tj, int pack)
{
    GET_CTX(c, Ptr);
    if (what < 0 || what > 4) return set_error(DUGMA_ERR_ARG, "set_shape: what must be 0 .. 4");
    std::vector<KernelShape> cand = shapes_of(what);
    KernelShape want;
    want.ipt = ipt;
    want.nt = nt;
    want.tj = tj;
    want.pack = pack;
    for (const KernelShape& s : cand)
        if (s.same(want)) {
            shape_slot(*c, what) = s;
            return DUGMA_OK;
        }
    return set_error(DUGMA_ERR_ARG, "set_shape: (%d, %d, %d, %d) is not a compiled shape", ipt, nt, tj, pack);
}

// mode 1: start recording (clears), 0: stop, 2: synchronise and report the total duration
// (ms) and count of the main pairwise-kernel launches recorded since mode 1.
int dugma_timing(float* Ptr[6], int mode, double* total_ms, int* launches)
{
    GET_CTX(c, Ptr);
    if (mode == 1) {
        c->timing = true;
        c->tused = 0;
        return DUGMA_OK;
    }
    if (mode == 0) {
        c->timing = false;
        return DUGMA_OK;
    }
    if (mode != 2) return set_error(DUGMA_ERR_ARG, "timing: mode must be 0, 1 or 2");
    double tot = 0;
    for (size_t k = 0; k < c->tused; ++k) {
        DUGMA_CK(cudaEventSynchronize(c->tevents[k].second));
        float ms = 0;
        DUGMA_CK(cudaEventElapsedTime(&ms, c->tevents[k].first, c->tevents[k].second));
        tot += ms;
    }
    if (total_ms) *total_ms = tot;
    if (launches) *launches = (int)c->tused;
    return DUGMA_OK;
}

// ---------------------------------------------------------------------------
// CUDA graph of one energy+gradient evaluation
// ---------------------------------------------------------------------------
struct Graph {
    Context* c = nullptr;
    float* ptr[6];
    int model = 0;
    bool mapped = false;   // the graph reads its pose from and writes its results to the mapped staging
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

int dugma_graph_create(float* Ptr[6], int model, void** out)
{
    if (!out) return set_error(DUGMA_ERR_ARG, "graph_create: null argument");
    GET_CTX(c, Ptr);
    // one eager run sizes the scratch so that nothing is allocated during capture
    DUGMA_CK(cudaMemcpyAsync(c->host, c->pose, sizeof(double) * kPoseDoubles, cudaMemcpyDeviceToHost, c->stream));
    DUGMA_CK(cudaStreamSynchronize(c->stream));
    if (!(c->host[kPoseSig] > 0)) {
        double Rm[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, R2[4] = {1, 0, 0, 1}, t0[3] = {0, 0, 0};
        DUGMA_RET(upload_pose(*c, c->D == 3 ? Rm : R2, t0, 1e-2));
    }
    DUGMA_RET(launch_pairs(*c, c->pose, model, true, 0, c->N, c->out, nullptr, c->stream));
    DUGMA_CK(cudaStreamSynchronize(c->stream));
    Graph* g = new Graph;
    g->c = c;
    for (int k = 0; k < 6; ++k) g->ptr[k] = Ptr[k];
    g->model = model;
    // REF model with mapped staging: the captured prologue reads the pose the host packs before each
    // launch, and the reduction writes the results back there (no copy or memset in the graph or
    // around it)
    EvalIO io;
    g->mapped = mapped_io(*c, model, nullptr, &io);
    DUGMA_CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int rc = launch_pairs(*c, c->pose, model, true, 0, c->N, c->out, nullptr, c->stream, nullptr,
                          g->mapped ? &io : nullptr);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    if (rc != DUGMA_OK || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        delete g;
        return rc != DUGMA_OK ? rc : set_error(DUGMA_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
    }
    g->graph = graph;
    if (cudaGraphInstantiate(&g->exec, graph, 0) != cudaSuccess) {
        cudaGraphDestroy(graph);
        delete g;
        return set_error(DUGMA_ERR_CUDA, "graph instantiation failed");
    }
    *out = g;
    return DUGMA_OK;
}

int dugma_graph_eval(void* graph, const double* R, const double* t, double sig, double* E, double* gout)
{
    Graph* g = static_cast<Graph*>(graph);
    if (!g || !R || !t || !E || !gout) return set_error(DUGMA_ERR_ARG, "graph_eval: null argument");
    Context* c = find_context(g->ptr);
    if (c != g->c) return set_error(DUGMA_ERR_STATE, "graph_eval: the context of this graph was freed");
    std::lock_guard<std::mutex> lk(c->mu);
    const int ng = ng_of(c->D);
    double o[8];
    if (g->mapped) {
        pack_pose(*c, R, t, sig, c->host);
        DUGMA_CK(cudaGraphLaunch(g->exec, c->stream));
        DUGMA_RET(mapped_fetch(*c, 1 + ng, o));
    } else {
        DUGMA_RET(upload_pose(*c, R, t, sig));
        DUGMA_CK(cudaGraphLaunch(g->exec, c->stream));
        DUGMA_RET(fetch(*c, c->out, 1 + ng, o));
    }
    *E = o[0];
    memcpy(gout, o + 1, sizeof(double) * ng);
    return DUGMA_OK;
}

int dugma_graph_destroy(void* graph)
{
    Graph* g = static_cast<Graph*>(graph);
    if (!g) return set_error(DUGMA_ERR_ARG, "graph_destroy: null graph");
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return DUGMA_OK;
}

// ---------------------------------------------------------------------------
// One EM iteration of the reference loop as a CUDA graph: update_sig at the new pose, its
// sigma written into the device pose block, compi at (R, t, sigma), and one copy of sigma and
// the surrogate moments back (DUGMA.m:60 and :105 without the host round trip between them)
// ---------------------------------------------------------------------------
}  // extern "C"

namespace dugma {

// One EM step on stream s: the pose block from the pinned staging (the search prologue reads it
// there when the staging is mapped, else a copy brings it), sigma there (the search prologue
// zeroes the error word; the sigma kernel puts the quantised sigma into the pose block), compi at
// that pose and sigma.  Sigma, the moments and the error word come back through the mapped
// staging (sigma at [64, 66), the error word behind the moments), or by copies when the staging
// is not mapped (the error word then at [63] as an int).
static int em_enqueue(Context& c, cudaStream_t s)
{
    if (!c.host_dev)
        DUGMA_CK(cudaMemcpyAsync(c.pose, c.host, sizeof(double) * kPoseDoubles, cudaMemcpyHostToDevice, s));
    SigmaOpts so;
    so.pose_src = c.host_dev;
    so.reset_err = true;
    so.pose_sig = c.pose;
    so.host_out = c.host_dev ? c.host_dev + 64 : nullptr;
    DUGMA_RET(launch_sigma(c, c.pose, c.out, s, 0, -1, so));
    CoefOpts co;
    co.host_moments = c.host_dev ? c.host_dev + kHostMoments : nullptr;
    DUGMA_RET(launch_coef(c, c.pose, c.mom, s, 0, -1, 0, -1, co));
    if (!c.host_dev) {
        DUGMA_CK(cudaMemcpyAsync(c.host + kHostMoments, c.mom, sizeof(double) * num_moments(c.D),
                                 cudaMemcpyDeviceToHost, s));
        DUGMA_CK(cudaMemcpyAsync(c.host + 64, c.out, sizeof(double) * 2, cudaMemcpyDeviceToHost, s));
        DUGMA_CK(cudaMemcpyAsync(c.host + 63, c.err, sizeof(int), cudaMemcpyDeviceToHost, s));
    }
    return DUGMA_OK;
}

struct EMGraph {
    Context* c = nullptr;
    float* ptr[6];
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};
}  // namespace dugma

extern "C" {

int dugma_em_graph_create(float* Ptr[6], void** out)
{
    if (!out) return set_error(DUGMA_ERR_ARG, "em_graph_create: null argument");
    GET_CTX(c, Ptr);
    static_assert(kHostMoments + kNumMomentsMax + 1 <= kHostDoubles && kNumMomentsMax + 1 <= kMomSlots,
                  "moment staging exceeds the pinned block");
    // one eager step first: sizes the scratch, allocates the coefficient records and uploads the
    // moment tables, so that nothing allocates or synchronises during the capture
    const double Rm[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, R2[4] = {1, 0, 0, 1}, t0[3] = {0, 0, 0};
    pack_pose(*c, c->D == 3 ? Rm : R2, t0, 0.0, c->host);
    DUGMA_RET(em_enqueue(*c, c->stream));
    DUGMA_CK(cudaStreamSynchronize(c->stream));
    EMGraph* g = new EMGraph;
    g->c = c;
    for (int k = 0; k < 6; ++k) g->ptr[k] = Ptr[k];
    DUGMA_CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = em_enqueue(*c, c->stream);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    if (rc != DUGMA_OK || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        delete g;
        return rc != DUGMA_OK ? rc : set_error(DUGMA_ERR_CUDA, "em graph capture failed: %s", cudaGetErrorString(e));
    }
    g->graph = graph;
    if (cudaGraphInstantiate(&g->exec, graph, 0) != cudaSuccess) {
        cudaGraphDestroy(graph);
        delete g;
        return set_error(DUGMA_ERR_CUDA, "em graph instantiation failed");
    }
    *out = g;
    return DUGMA_OK;
}

int dugma_em_step(void* graph, const double* R, const double* t, float sig[1], double coefficient[640])
{
    EMGraph* g = static_cast<EMGraph*>(graph);
    if (!g || !R || !t || !sig || !coefficient) return set_error(DUGMA_ERR_ARG, "em_step: null argument");
    Context* c = find_context(g->ptr);
    if (c != g->c) return set_error(DUGMA_ERR_STATE, "em_step: the context of this graph was freed");
    std::lock_guard<std::mutex> lk(c->mu);
    pack_pose(*c, R, t, 0.0, c->host);
    DUGMA_CK(cudaGraphLaunch(g->exec, c->stream));
    DUGMA_CK(cudaStreamSynchronize(c->stream));
    int err = 0;
    if (c->host_dev)
        err = (int)c->host[kHostMoments + num_moments(c->D)];
    else
        memcpy(&err, c->host + 63, sizeof(int));
    if (err) return set_error(DUGMA_ERR_TIMEOUT, "a device wait gave up (error word 0x%x)", err);
    sig[0] = (float)c->host[65];
    return coef_from_moments(c->D, c->host + kHostMoments, coefficient);
}

int dugma_em_graph_destroy(void* graph)
{
    EMGraph* g = static_cast<EMGraph*>(graph);
    if (!g) return set_error(DUGMA_ERR_ARG, "em_graph_destroy: null graph");
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return DUGMA_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Reference-signature entry points (C++ linkage): a MEX gateway of the reference links
// against these unchanged (init.cpp:9-19, update_sig.cpp:7, compi.cpp:7, fr_m.cpp:7).
// Errors are printed like the reference does, but never exit the process.
// ---------------------------------------------------------------------------
void init(double* X, double* X_C, double* Y, double* Y_C, double* Coef, int N, int M, int D, float* Ptr[6])
{
    const int rc = dugma_init(X, X_C, Y, Y_C, Coef, N, M, D, Ptr);
    if (rc != DUGMA_OK) fprintf(stderr, "dugma init: %s\n", dugma_last_error());
}

void cpd(float* Ptr[6], double* R, double* t, double* N, double* M, double* D, float sig[1])
{
    if (dugma_update_sig(Ptr, R, t, N, M, D, sig) != DUGMA_OK) {
        fprintf(stderr, "dugma update_sig: %s\n", dugma_last_error());
        sig[0] = NAN;
    }
}

void cpd(float* Ptr[6], double* R, double* t, double* N, double* M, double* D, double* sig,
         double coefficient[640])
{
    if (dugma_compi(Ptr, R, t, N, M, D, sig, coefficient) != DUGMA_OK) {
        fprintf(stderr, "dugma compi: %s\n", dugma_last_error());
        for (int k = 0; k < 640; ++k) coefficient[k] = NAN;
    }
}

void fr_m(float* Ptr[6])
{
    if (dugma_fr_m(Ptr) != DUGMA_OK) fprintf(stderr, "dugma fr_m: %s\n", dugma_last_error());
}

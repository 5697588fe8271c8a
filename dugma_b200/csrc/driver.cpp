// driver.cpp -- the registration loop of DUGMA.m:19-137 with a quasi-Newton solver in
// place of MATLAB's fmincon.
//
// Reference mode (DUGMA_DRIVE_REFERENCE), per iteration (DUGMA.m:57-113):
//   A = compi(R, t, sig)                      the 637 / 45 surrogate coefficients
//   (dR, dt) = argmin Q(dR, dt) = A . b(dR, dt) over dR in SO(D)   (energy3D.m, fcontr3D.m)
//   R <- dR R,  t <- dt + t                   (DUGMA.m:76-78: t is not rotated by dR)
//   stop on the Euler-angle change (rotm2eul ZYX; 2D asind(R21), degrees), |t - t_prev|^2,
//   sig <= acc_sig or the iteration limit; sig <- update_sig(R, t).
// fmincon minimises over a general 3x3 dR with det dR = 1 and dR^T dR = I; here dR =
// exp([w]x) (2D: a rotation by theta), so the constraints hold by construction and the
// minimisation is unconstrained over local coordinates (w, dt) at the current iterate:
// damped Newton steps with the analytic gradient and Hessian of Q (from the monomial
// exponents and the derivatives of R <- exp([w]x) R at w = 0), with backtracking.
// Each iteration's update_sig and the next iteration's compi run as one captured CUDA graph
// (dugma_em_step): the sigma stays on the device between them.
// Direct mode (DUGMA_DRIVE_DIRECT): maximise E(R, t) at the current sig with BFGS on the
// left-perturbation coordinates using the fused adjoint's gradient, then update sig; every
// evaluation replays one captured CUDA graph (pose prologue, adjoint, reduction).
// Both modes normalise the clouds first (normalize.m:3-26) and denormalise the
// translation at the end (DUGMA.m:122).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "dugma.h"
#include "monomials.h"

namespace dugma {
int set_error(int code, const char* fmt, ...);
}

namespace {

using Vec = std::vector<double>;

struct Mat3 {
    double a[9];   // column-major
    double& operator()(int r, int c) { return a[r + 3 * c]; }
    double operator()(int r, int c) const { return a[r + 3 * c]; }
};

Mat3 mul(const Mat3& A, const Mat3& B)
{
    Mat3 C{};
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += A(r, k) * B(k, c);
            C(r, c) = s;
        }
    return C;
}

Mat3 expso3(const double w[3])
{
    const double th = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    Mat3 K{};
    K(0, 1) = -w[2];
    K(0, 2) = w[1];
    K(1, 0) = w[2];
    K(1, 2) = -w[0];
    K(2, 0) = -w[1];
    K(2, 1) = w[0];
    const Mat3 K2 = mul(K, K);
    const double a = th < 1e-10 ? 1.0 - th * th / 6.0 : std::sin(th) / th;
    const double b = th < 1e-10 ? 0.5 - th * th / 24.0 : (1.0 - std::cos(th)) / (th * th);
    Mat3 R{};
    for (int k = 0; k < 9; ++k) R.a[k] = (k % 4 == 0 ? 1.0 : 0.0) + a * K.a[k] + b * K2.a[k];
    return R;
}

// ZYX Euler angles of a rotation (MATLAB rotm2eul default), radians: [z, y, x]
void rotm2eul(const Mat3& R, double e[3])
{
    const double sy = std::max(-1.0, std::min(1.0, -R(2, 0)));
    e[1] = std::asin(sy);
    if (std::fabs(sy) < 1.0 - 1e-12) {
        e[0] = std::atan2(R(1, 0), R(0, 0));
        e[2] = std::atan2(R(2, 1), R(2, 2));
    } else {
        e[0] = std::atan2(-R(0, 1), R(1, 1));
        e[2] = 0.0;
    }
}

// The surrogate's monomials as lists of at most 4 variable indices (a variable appears once
// per unit of its exponent; -1 pads), built once per dimension from the exponent tables.
struct Mono {
    signed char f[4];
};

const std::vector<Mono>& mono_table(int D)
{
    auto build = [](const unsigned char* E, int K, int nv) {
        std::vector<Mono> t(K);
        for (int k = 0; k < K; ++k) {
            int n = 0;
            for (int q = 0; q < 4; ++q) t[k].f[q] = -1;
            for (int q = 0; q < nv; ++q)
                for (int e = 0; e < E[k * nv + q] && n < 4; ++e) t[k].f[n++] = (signed char)q;
        }
        return t;
    };
    static const std::vector<Mono> t3 = build(&dugma::kMonoExp3D[0][0], 637, 12);
    static const std::vector<Mono> t2 = build(&dugma::kMonoExp2D[0][0], 45, 4);
    return D == 3 ? t3 : t2;
}

// Surrogate Q(v) = sum_k A_k prod_q v_q^e_kq, its gradient and Hessian in v.
struct Surrogate {
    int D, K, nv;
    const double* A;
    const unsigned char* E;
    double value(const double* v) const
    {
        const std::vector<Mono>& T = mono_table(D);
        double s = 0;
        for (int k = 0; k < K; ++k) {
            double m = A[k];
            for (int j = 0; j < 4 && T[k].f[j] >= 0; ++j) m *= v[T[k].f[j]];
            s += m;
        }
        return s;
    }
    // Gradient and Hessian in v (nv x nv, row-major) in one pass: for a monomial A x_0 .. x_{n-1}
    // (its factor list; a variable of exponent e appears e times) the gradient gets the product
    // of the other factors at each factor's variable, and every unordered pair of factor
    // positions gets the product of the remaining factors at both off-diagonal entries (a
    // repeated variable so collects e (e - 1) v^(e - 2) on the diagonal).  Written out per
    // factor count (1..4) so that each product is formed once.
    void grad_hess(const double* v, double* g, double* H) const
    {
        const std::vector<Mono>& T = mono_table(D);
        for (int q = 0; q < nv; ++q) g[q] = 0;
        for (int q = 0; q < nv * nv; ++q) H[q] = 0;
        // the upper triangle only (a pair on the diagonal counts twice), mirrored at the end
        auto pair = [&](int a, int b, double m) {
            if (a == b)
                H[a * nv + a] += 2.0 * m;
            else if (a < b)
                H[a * nv + b] += m;
            else
                H[b * nv + a] += m;
        };
        for (int k = 0; k < K; ++k) {
            const signed char* f = T[k].f;
            const double c = A[k];
            if (f[0] < 0) continue;
            const double x0 = v[f[0]];
            if (f[1] < 0) {
                g[f[0]] += c;
                continue;
            }
            const double x1 = v[f[1]];
            if (f[2] < 0) {
                g[f[0]] += c * x1;
                g[f[1]] += c * x0;
                pair(f[0], f[1], c);
                continue;
            }
            const double x2 = v[f[2]];
            if (f[3] < 0) {
                g[f[0]] += c * x1 * x2;
                g[f[1]] += c * x0 * x2;
                g[f[2]] += c * x0 * x1;
                pair(f[0], f[1], c * x2);
                pair(f[0], f[2], c * x1);
                pair(f[1], f[2], c * x0);
                continue;
            }
            const double x3 = v[f[3]];
            const double c01 = c * x0 * x1, c23 = c * x2 * x3;
            g[f[0]] += c23 * x1;
            g[f[1]] += c23 * x0;
            g[f[2]] += c01 * x3;
            g[f[3]] += c01 * x2;
            pair(f[0], f[1], c23);
            pair(f[2], f[3], c01);
            pair(f[0], f[2], c * x1 * x3);
            pair(f[0], f[3], c * x1 * x2);
            pair(f[1], f[2], c * x0 * x3);
            pair(f[1], f[3], c * x0 * x2);
        }
        for (int a = 0; a < nv; ++a)
            for (int b = a + 1; b < nv; ++b) H[b * nv + a] = H[a * nv + b];
    }
};

// The surrogate along the pose: v(R, t) = (t, the rows of R) in 3D, (t, cos, sin) in 2D.  Local
// coordinates p = (dw, dt) at the current pose move it as R <- exp([dw]x) R (2D: a rotation
// by dw) and t <- t + dt; at p = 0 the gradient and Hessian in p follow from those in v:
//   g = J^T gv,  H = J^T Hv J + sum_q gv_q d2v_q/dp2,
// with dR/dw_i = [e_i]x R and d2R/dw_i dw_j = (([e_i]x [e_j]x + [e_j]x [e_i]x) / 2) R.
struct SurrogatePose {
    Surrogate S;
    int D;
    int np() const { return D == 3 ? 6 : 3; }
    void v_of(const Mat3& R, const double* t, double* v) const
    {
        if (D == 3) {
            for (int a = 0; a < 3; ++a) v[a] = t[a];
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) v[3 + 3 * r + c] = R(r, c);   // r11 r12 r13 r21 ... (row-major)
        } else {
            v[0] = t[0];
            v[1] = t[1];
            v[2] = R(0, 0);
            v[3] = R(1, 0);
        }
    }
    double value(const Mat3& R, const double* t) const
    {
        double v[12];
        v_of(R, t, v);
        return S.value(v);
    }
    static Mat3 skew_unit(int i)
    {
        Mat3 K{};
        const int a = (i + 1) % 3, b = (i + 2) % 3;
        K(b, a) = 1.0;
        K(a, b) = -1.0;
        return K;
    }
    void derivs(const Mat3& R, const double* t, double* g, double* H) const
    {
        const int nv = S.nv, n = np();
        double v[12], gv[12], Hv[144], J[12 * 6] = {};
        v_of(R, t, v);
        S.grad_hess(v, gv, Hv);
        if (D == 3) {
            for (int i = 0; i < 3; ++i) {
                const Mat3 G = mul(skew_unit(i), R);
                for (int r = 0; r < 3; ++r)
                    for (int c = 0; c < 3; ++c) J[(3 + 3 * r + c) * n + i] = G(r, c);
                J[i * n + 3 + i] = 1.0;
            }
        } else {
            J[0 * n + 1] = 1.0;
            J[1 * n + 2] = 1.0;
            J[2 * n + 0] = -v[3];   // d cos / d theta
            J[3 * n + 0] = v[2];    // d sin / d theta
        }
        for (int k = 0; k < n; ++k) {
            double s = 0;
            for (int q = 0; q < nv; ++q) s += J[q * n + k] * gv[q];
            g[k] = s;
        }
        double HJ[12 * 6];
        for (int q = 0; q < nv; ++q)
            for (int l = 0; l < n; ++l) {
                double s = 0;
                for (int r = 0; r < nv; ++r) s += Hv[q * nv + r] * J[r * n + l];
                HJ[q * n + l] = s;
            }
        for (int k = 0; k < n; ++k)
            for (int l = 0; l < n; ++l) {
                double s = 0;
                for (int q = 0; q < nv; ++q) s += J[q * n + k] * HJ[q * n + l];
                H[k * n + l] = s;
            }
        if (D == 3) {
            // sum_rc gR_rc (([e_i]x [e_j]x + [e_j]x [e_i]x) / 2 R)_rc with [a]x [b]x = b a^T - (a.b) I:
            // (gR_j . R_i + gR_i . R_j) / 2 - delta_ij <gR, R>, R_i and gR_i the i-th rows
            double dots[3][3], tr = 0;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    double d = 0;
                    for (int c = 0; c < 3; ++c) d += gv[3 + 3 * i + c] * R(j, c);
                    dots[i][j] = d;   // gR_i . R_j
                }
            for (int i = 0; i < 3; ++i) tr += dots[i][i];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) H[i * n + j] += 0.5 * (dots[j][i] + dots[i][j]) - (i == j ? tr : 0.0);
        } else {
            H[0] -= gv[2] * v[2] + gv[3] * v[3];   // d2 cos = -cos, d2 sin = -sin
        }
    }
    void step(const Mat3& R, const double* t, const double* x, Mat3& Rn, double* tn) const
    {
        if (D == 3) {
            Rn = mul(expso3(x), R);
            for (int a = 0; a < 3; ++a) tn[a] = t[a] + x[3 + a];
        } else {
            const double th = std::atan2(R(1, 0), R(0, 0)) + x[0];
            Rn = Mat3{};
            Rn(0, 0) = std::cos(th);
            Rn(1, 0) = std::sin(th);
            Rn(0, 1) = -std::sin(th);
            Rn(1, 1) = std::cos(th);
            Rn(2, 2) = 1.0;
            tn[0] = t[0] + x[1];
            tn[1] = t[1] + x[2];
        }
    }
};

// Solve H x = b for a small system (n <= 6; Gaussian elimination with partial pivoting, in place)
bool solve(int n, double* H, double* b, double* x)
{
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(H[r * n + c]) > std::fabs(H[piv * n + c])) piv = r;
        if (std::fabs(H[piv * n + c]) < 1e-300) return false;
        if (piv != c) {
            for (int k = 0; k < n; ++k) std::swap(H[c * n + k], H[piv * n + k]);
            std::swap(b[c], b[piv]);
        }
        for (int r = c + 1; r < n; ++r) {
            const double f = H[r * n + c] / H[c * n + c];
            for (int k = c; k < n; ++k) H[r * n + k] -= f * H[c * n + k];
            b[r] -= f * b[c];
        }
    }
    for (int r = n - 1; r >= 0; --r) {
        double s = b[r];
        for (int k = r + 1; k < n; ++k) s -= H[r * n + k] * x[k];
        x[r] = s / H[r * n + r];
    }
    return true;
}

// Damped Newton minimisation of the surrogate from dR = I, dt = 0 in local coordinates (analytic
// gradient and Hessian, trust region 0.5, backtracking); returns the exit flag (> 0 converged,
// 0 iteration limit, < 0 failure as fmincon's exitflag).
int minimise_surrogate(const SurrogatePose& F, Mat3& R, double* t, int* evals)
{
    const int n = F.np();
    R = Mat3{};
    R(0, 0) = R(1, 1) = R(2, 2) = 1.0;
    t[0] = t[1] = t[2] = 0.0;
    double f = F.value(R, t);
    if (!std::isfinite(f)) return -1;
    double lam = 0;
    for (int it = 0; it < 100; ++it) {
        double g[6], H[36];
        F.derivs(R, t, g, H);
        double gn = 0;
        for (int k = 0; k < n; ++k) gn += g[k] * g[k];
        gn = std::sqrt(gn);
        for (int r = 0; r < n; ++r)
            for (int c = r + 1; c < n; ++c) H[r * n + c] = H[c * n + r] = 0.5 * (H[r * n + c] + H[c * n + r]);
        double hmax = 0;
        for (int r = 0; r < n; ++r) hmax = std::max(hmax, std::fabs(H[r * n + r]));
        if (lam == 0) lam = 1e-9 * std::max(hmax, 1e-300);
        bool accepted = false;
        for (int tries = 0; tries < 40 && !accepted; ++tries) {
            double A[36], mg[6], x[6];
            for (int q = 0; q < n * n; ++q) A[q] = H[q];
            for (int r = 0; r < n; ++r) A[r * n + r] += lam;
            for (int r = 0; r < n; ++r) mg[r] = -g[r];
            if (!solve(n, A, mg, x)) {
                lam *= 10;
                continue;
            }
            double step = 0;
            for (int k = 0; k < n; ++k) step += x[k] * x[k];
            step = std::sqrt(step);
            if (step > 0.5) {   // trust region on the rotation increment / translation
                for (int k = 0; k < n; ++k) x[k] *= 0.5 / step;
                step = 0.5;
            }
            Mat3 Rn;
            double tn[3] = {0, 0, 0};
            F.step(R, t, x, Rn, tn);
            const double fn = F.value(Rn, tn);
            ++*evals;
            if (std::isfinite(fn) && fn <= f) {
                const double df = f - fn;
                R = Rn;
                for (int a = 0; a < 3; ++a) t[a] = tn[a];
                f = fn;
                lam = std::max(lam * 0.3, 1e-15 * std::max(hmax, 1e-300));
                accepted = true;
                if (step < 1e-12 || df <= 1e-15 * std::fabs(f)) return 1;
            } else {
                lam *= 10;
            }
        }
        if (!accepted) return gn < 1e-8 * (1 + std::fabs(f)) ? 2 : 1;   // at a stationary point
    }
    return 0;
}

struct Timer {
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    double s() const
    {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

}  // namespace

extern "C" int dugma_minimise_surrogate(int D, const double* A, double* dR, double* dt, double* Qmin, int* exitflag)
{
    if ((D != 2 && D != 3) || !A || !dR || !dt) return DUGMA_ERR_ARG;
    SurrogatePose F{{D, D == 3 ? 637 : 45, D == 3 ? 12 : 4, A,
                     D == 3 ? &dugma::kMonoExp3D[0][0] : &dugma::kMonoExp2D[0][0]},
                    D};
    Mat3 Rm;
    double tv[3];
    int evals = 0;
    const int flag = minimise_surrogate(F, Rm, tv, &evals);
    if (exitflag) *exitflag = flag;
    if (flag < 0) return DUGMA_ERR_NUMERIC;
    for (int c = 0; c < D; ++c)
        for (int r = 0; r < D; ++r) dR[r + D * c] = Rm(r, c);
    for (int a = 0; a < D; ++a) dt[a] = tv[a];
    if (Qmin) *Qmin = F.value(Rm, tv);
    return DUGMA_OK;
}

extern "C" int dugma_register(const double* X, const double* X_C, const double* Y, const double* Y_C, int N, int M,
                              int D, const double* R0, const double* t0, int max_iter, double acc_rot,
                              double acc_trans, double acc_sig, int mode, double* R_out, double* t_out,
                              double* stats)
{
    if (!X || !X_C || !Y || !Y_C || !R0 || !t0 || !R_out || !t_out)
        return dugma::set_error(DUGMA_ERR_ARG, "register: null argument");
    if (D != 2 && D != 3) return dugma::set_error(DUGMA_ERR_ARG, "register: D must be 2 or 3");
    if (mode != DUGMA_DRIVE_REFERENCE && mode != DUGMA_DRIVE_DIRECT)
        return dugma::set_error(DUGMA_ERR_ARG, "register: unknown mode %d", mode);
    if (N < 2 || M < 2) return dugma::set_error(DUGMA_ERR_ARG, "register: each cloud needs at least 2 points");
    Timer timer;
    // normalize.m:3-26: centre each cloud, divide both by the larger RMS radius
    double xd[3] = {0, 0, 0}, yd[3] = {0, 0, 0};
    for (int i = 0; i < N; ++i)
        for (int a = 0; a < D; ++a) xd[a] += X[(size_t)i * D + a] / N;
    for (int j = 0; j < M; ++j)
        for (int a = 0; a < D; ++a) yd[a] += Y[(size_t)j * D + a] / M;
    double xs = 0, ys = 0;
    std::vector<double> Xn((size_t)N * D), Yn((size_t)M * D);
    for (int i = 0; i < N; ++i)
        for (int a = 0; a < D; ++a) {
            Xn[(size_t)i * D + a] = X[(size_t)i * D + a] - xd[a];
            xs += Xn[(size_t)i * D + a] * Xn[(size_t)i * D + a];
        }
    for (int j = 0; j < M; ++j)
        for (int a = 0; a < D; ++a) {
            Yn[(size_t)j * D + a] = Y[(size_t)j * D + a] - yd[a];
            ys += Yn[(size_t)j * D + a] * Yn[(size_t)j * D + a];
        }
    const double scale = std::max(std::sqrt(xs / N), std::sqrt(ys / M));
    if (!(scale > 0)) return dugma::set_error(DUGMA_ERR_ARG, "register: both clouds collapse to a point");
    for (double& v : Xn) v /= scale;
    for (double& v : Yn) v /= scale;
    // covariances are passed unscaled, as DUGMA.m:44 does
    float* Ptr[6];
    double ok = 0;
    int rc = dugma_init(Xn.data(), X_C, Yn.data(), Y_C, &ok, N, M, D, Ptr);
    if (rc != DUGMA_OK && rc != DUGMA_ERR_NONPD) return rc;
    double R[9] = {0}, t[3] = {0};
    for (int k = 0; k < D * D; ++k) R[k] = R0[k];
    for (int a = 0; a < D; ++a) t[a] = t0[a];
    const double Nd = N, Md = M, Dd = D;
    float sigf = 0;
    int evals = 0;
    rc = dugma_update_sig(Ptr, R, t, &Nd, &Md, &Dd, &sigf);
    double sig = sigf;
    // direct mode: one captured CUDA graph (pose prologue, fused adjoint, reduction) replayed
    // for every evaluation; without it (capture refused) the eager launches run instead
    void* graph = nullptr;
    if (rc == DUGMA_OK && mode == DUGMA_DRIVE_DIRECT && dugma_graph_create(Ptr, DUGMA_MODEL_REF, &graph) != DUGMA_OK)
        graph = nullptr;
    // reference mode: update_sig at the new pose and the next iteration's compi as one captured
    // graph per iteration (the same kernels and values as the two plugin calls); without it
    // (capture refused) the two calls run eagerly
    void* emg = nullptr;
    if (rc == DUGMA_OK && mode == DUGMA_DRIVE_REFERENCE && dugma_em_graph_create(Ptr, &emg) != DUGMA_OK)
        emg = nullptr;
    double A[640];
    bool have_A = false;   // A holds compi at the current (R, t, sig)
    auto eval = [&](const double* Rx, const double* tx, double* Ex, double* gx) {
        return graph ? dugma_graph_eval(graph, Rx, tx, sig, Ex, gx)
                     : dugma_energy_grad(Ptr, Rx, tx, sig, DUGMA_MODEL_REF, Ex, gx, nullptr);
    };
    const int NR = D == 3 ? 3 : 1;
    double angle[3] = {1e4, 1e4, 1e4}, angle0[3];
    double tprev[3] = {t[0], t[1], t[2]};
    bool con_angle = true;
    int exitflag = 1, iter = 1;
    double E = 0;
    auto tdiff2 = [&]() {
        double s = 0;
        for (int a = 0; a < D; ++a) s += (tprev[a] - t[a]) * (tprev[a] - t[a]);
        return s;
    };
    while (rc == DUGMA_OK && iter <= max_iter && (con_angle || std::fabs(tdiff2()) > acc_trans) && sig > acc_sig) {
        double dRm[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, dt[3] = {0, 0, 0};
        if (mode == DUGMA_DRIVE_REFERENCE) {
            if (!have_A) rc = dugma_compi(Ptr, R, t, &Nd, &Md, &Dd, &sig, A);
            have_A = false;
            if (rc != DUGMA_OK) break;
            SurrogatePose F{{D, D == 3 ? 637 : 45, D == 3 ? 12 : 4, A,
                             D == 3 ? &dugma::kMonoExp3D[0][0] : &dugma::kMonoExp2D[0][0]},
                            D};
            Mat3 Q;
            double tq[3];
            exitflag = minimise_surrogate(F, Q, tq, &evals);
            if (exitflag < 0) break;
            for (int c = 0; c < D; ++c)
                for (int r = 0; r < D; ++r) dRm[r + D * c] = Q(r, c);
            for (int a = 0; a < D; ++a) dt[a] = tq[a];
        } else {
            // BFGS ascent of E on the left-perturbation coordinates at fixed sig
            const int n = NR + D;
            double g[6];
            rc = eval(R, t, &E, g);
            ++evals;
            if (rc != DUGMA_OK) break;
            std::vector<double> Hi(n * n, 0.0);
            double gn = 0;
            for (int k = 0; k < n; ++k) gn += g[k] * g[k];
            gn = std::sqrt(gn);
            for (int k = 0; k < n; ++k) Hi[k * n + k] = gn > 0 ? 0.05 / gn : 0.0;
            double Rc[9], tc[3];
            memcpy(Rc, R, sizeof(Rc));
            memcpy(tc, t, sizeof(tc));
            for (int it = 0; it < 25 && rc == DUGMA_OK; ++it) {
                double s[6] = {0}, Rn[9], tn[3], En = 0, gnew[6];
                for (int r = 0; r < n; ++r)
                    for (int c = 0; c < n; ++c) s[r] += Hi[r * n + c] * g[c];   // ascent direction
                double alpha = 1.0;
                bool ok2 = false;
                for (int bt = 0; bt < 20; ++bt) {
                    double w[3] = {0, 0, 0};
                    for (int k = 0; k < NR; ++k) w[D == 3 ? k : 2] = alpha * s[k];
                    Mat3 Q{};
                    if (D == 3) {
                        Q = expso3(w);
                        Mat3 Rm{};
                        memcpy(Rm.a, Rc, sizeof(Rm.a));
                        const Mat3 P = mul(Q, Rm);
                        memcpy(Rn, P.a, sizeof(P.a));
                    } else {
                        const double c = std::cos(w[2]), sn = std::sin(w[2]);
                        Rn[0] = c * Rc[0] - sn * Rc[1];
                        Rn[1] = sn * Rc[0] + c * Rc[1];
                        Rn[2] = c * Rc[2] - sn * Rc[3];
                        Rn[3] = sn * Rc[2] + c * Rc[3];
                    }
                    for (int a = 0; a < D; ++a) tn[a] = tc[a] + alpha * s[NR + a];
                    rc = eval(Rn, tn, &En, gnew);
                    ++evals;
                    if (rc != DUGMA_OK) break;
                    double dir = 0;
                    for (int k = 0; k < n; ++k) dir += g[k] * s[k];
                    if (En >= E + 1e-4 * alpha * dir) {
                        ok2 = true;
                        break;
                    }
                    alpha *= 0.5;
                }
                if (!ok2 || rc != DUGMA_OK) break;
                // BFGS update for the inverse Hessian of -E in the new tangent coordinates
                double sv[6], yv[6], sy = 0;
                for (int k = 0; k < n; ++k) {
                    sv[k] = alpha * s[k];
                    yv[k] = -(gnew[k] - g[k]);
                    sy += sv[k] * yv[k];
                }
                if (sy > 1e-300) {
                    std::vector<double> Hy(n, 0.0);
                    double yHy = 0;
                    for (int r = 0; r < n; ++r)
                        for (int c = 0; c < n; ++c) Hy[r] += Hi[r * n + c] * yv[c];
                    for (int r = 0; r < n; ++r) yHy += yv[r] * Hy[r];
                    for (int r = 0; r < n; ++r)
                        for (int c = 0; c < n; ++c)
                            Hi[r * n + c] += (sy + yHy) * sv[r] * sv[c] / (sy * sy) - (Hy[r] * sv[c] + sv[r] * Hy[c]) / sy;
                }
                double stepn = 0;
                for (int k = 0; k < n; ++k) stepn += sv[k] * sv[k];
                const double dE = En - E;
                memcpy(Rc, Rn, sizeof(Rc));
                memcpy(tc, tn, sizeof(tc));
                E = En;
                memcpy(g, gnew, sizeof(g));
                if (std::sqrt(stepn) < 1e-10 || dE <= 1e-12 * std::fabs(E)) break;
            }
            if (rc != DUGMA_OK) break;
            // express the accepted pose as (dR, dt) relative to (R, t) for the common update below
            if (D == 3) {
                Mat3 Rn{}, Rt{};
                memcpy(Rn.a, Rc, sizeof(Rn.a));
                for (int r = 0; r < 3; ++r)
                    for (int c = 0; c < 3; ++c) Rt(r, c) = R[c + 3 * r];
                const Mat3 Q = mul(Rn, Rt);
                memcpy(dRm, Q.a, sizeof(Q.a));
            } else {
                const double c = Rc[0] * R[0] + Rc[1] * R[1], sn = Rc[1] * R[0] - Rc[0] * R[1];
                dRm[0] = c;
                dRm[1] = sn;
                dRm[2] = -sn;
                dRm[3] = c;
            }
            for (int a = 0; a < D; ++a) dt[a] = tc[a] - t[a];
        }
        // DUGMA.m:76-80: t <- dt + t, R <- dR R
        for (int a = 0; a < D; ++a) {
            tprev[a] = t[a];
            t[a] = dt[a] + t[a];
        }
        double Rn[9];
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c) {
                double s = 0;
                for (int k = 0; k < D; ++k) s += dRm[r + D * k] * R[k + D * c];
                Rn[r + D * c] = s;
            }
        memcpy(R, Rn, sizeof(double) * D * D);
        memcpy(angle0, angle, sizeof(angle));
        if (D == 3) {
            Mat3 Rm{};
            memcpy(Rm.a, R, sizeof(Rm.a));
            rotm2eul(Rm, angle);
            con_angle = std::fabs(angle0[0] - angle[0]) > acc_rot || std::fabs(angle0[1] - angle[1]) > acc_rot ||
                        std::fabs(angle0[2] - angle[2]) > acc_rot;
        } else {
            angle[0] = std::asin(std::max(-1.0, std::min(1.0, R[1]))) * 180.0 / M_PI;   // asind(R(2))
            con_angle = std::fabs(angle0[0] - angle[0]) > acc_rot;
        }
        // the host-side part of the loop test for the next iteration: when it holds, that
        // iteration's compi runs in the same graph as this update_sig
        const bool next = iter + 1 <= max_iter && (con_angle || std::fabs(tdiff2()) > acc_trans);
        if (emg && next) {
            rc = dugma_em_step(emg, R, t, &sigf, A);
            have_A = rc == DUGMA_OK;
        } else {
            rc = dugma_update_sig(Ptr, R, t, &Nd, &Md, &Dd, &sigf);
        }
        sig = sigf;
        ++iter;
    }
    if (rc == DUGMA_OK) {
        double gtmp[6];
        dugma_energy_grad(Ptr, R, t, sig, DUGMA_MODEL_REF, &E, gtmp, nullptr);
    }
    if (graph) dugma_graph_destroy(graph);
    if (emg) dugma_em_graph_destroy(emg);
    dugma_fr_m(Ptr);
    if (rc != DUGMA_OK) return rc;
    if (exitflag < 0) {   // DUGMA.m:116-118: an unsolvable surrogate returns the identity
        for (int k = 0; k < D * D; ++k) R_out[k] = (k % (D + 1) == 0) ? 1.0 : 0.0;
        for (int a = 0; a < D; ++a) t_out[a] = 0.0;
    } else {
        // DUGMA.m:122: t = xd + t * scale - R * yd
        for (int k = 0; k < D * D; ++k) R_out[k] = R[k];
        for (int a = 0; a < D; ++a) {
            double Ry = 0;
            for (int k = 0; k < D; ++k) Ry += R[a + D * k] * yd[k];
            t_out[a] = xd[a] + t[a] * scale - Ry;
        }
    }
    if (stats) {
        stats[0] = iter - 1;
        stats[1] = sig;
        stats[2] = E;
        stats[3] = exitflag;
        stats[4] = timer.s();
        stats[5] = evals;
        stats[6] = scale;
        stats[7] = 0;
    }
    return DUGMA_OK;
}

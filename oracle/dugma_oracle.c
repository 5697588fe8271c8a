/*
 * dugma_oracle.c -- FP64 CPU oracle for the DUGMA hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates the reference's formulas on the
 * CPU so that the CUDA path can be checked against it.  Only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference leg load it;
 * the product library never links or calls it.
 *
 * Parity pins: the coefficient expressions it evaluates (coef_terms.h) are
 * checked symbolically against the reference kernel source by
 * tests/test_oracle_symbolic.py, and its init / update_sig / compi outputs are
 * checked against the reference's own CUDA plugins (built from the reference
 * sources into oracle/_ref) through the fixtures in tests/golden/.
 *
 * Conventions shared with the CUDA library:
 *   points      point-major float arrays, D floats per point (MATLAB D x N column-major)
 *   covariances D x D column-major block per point (MATLAB D x D*N)
 *   R           D x D column-major (MATLAB), applied to Y:  y' = R y + t
 *   packed sym  (00,11,22,01,02,12) in 3D, (00,11,01) in 2D
 *   pose grad   g = [dE/domega (NR), dE/dt (D)], left perturbation R <- exp([w]x) R;
 *               NR = 3 in 3D, 1 in 2D.
 * All arithmetic is IEEE FP64 (built with -ffp-contract=off) except the
 * nearest-neighbour routine, which reproduces a specified FP32 sequence.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "coef_terms.h"

#define ORACLE_BLOCK 32 /* i-rows per deterministic partial */

static int nsym(int D) { return D == 3 ? 6 : 3; }
static const int S3[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
static const int S2[3][2] = {{0, 0}, {1, 1}, {0, 1}};

static void sym_pack(int D, const double* full /* col-major */, double* p)
{
    int n = nsym(D);
    for (int k = 0; k < n; ++k) {
        int a = D == 3 ? S3[k][0] : S2[k][0], b = D == 3 ? S3[k][1] : S2[k][1];
        p[k] = 0.5 * (full[a + D * b] + full[b + D * a]);
    }
}

static void sym_unpack(int D, const double* p, double* full)
{
    int n = nsym(D);
    for (int k = 0; k < n; ++k) {
        int a = D == 3 ? S3[k][0] : S2[k][0], b = D == 3 ? S3[k][1] : S2[k][1];
        full[a + D * b] = p[k];
        full[b + D * a] = p[k];
    }
}

/* ------------------------------------------------------------------------- */
/* init: per-point inverse covariance and |Sigma|^-1/2 (init.cu:72-100).     */
/* Input covariances are first rounded to FP32 (init.cu:205-234), then the    */
/* determinant and adjugate are evaluated in FP64 in the order below and the  */
/* results rounded to FP32.  det <= 0: every entry := 1e5 and weight := 0     */
/* (the point is neglected, init.cu:86-100).  Returns the count of neglected. */
/* ------------------------------------------------------------------------- */
int dugma_oracle_prepare(int D, int n, const double* cov, float* cinv, float* w)
{
    int bad = 0;
    for (int p = 0; p < n; ++p) {
        const double* c = cov + (size_t)p * D * D;
        float* o = cinv + (size_t)p * D * D;
        double a[9];
        for (int k = 0; k < D * D; ++k) a[k] = (double)(float)c[k];
        if (D == 3) {
            double a11 = a[0], a21 = a[1], a31 = a[2], a12 = a[3], a22 = a[4], a32 = a[5],
                   a13 = a[6], a23 = a[7], a33 = a[8];
            double d = a11 * a22 * a33 - a11 * a23 * a32 - a12 * a21 * a33 + a12 * a23 * a31 +
                       a13 * a21 * a32 - a13 * a22 * a31;
            if (d > 0) {
                o[0] = (float)((a22 * a33 - a23 * a32) / d);
                o[1] = (float)(-(a21 * a33 - a23 * a31) / d);
                o[2] = (float)((a21 * a32 - a22 * a31) / d);
                o[3] = (float)(-(a12 * a33 - a13 * a32) / d);
                o[4] = (float)((a11 * a33 - a13 * a31) / d);
                o[5] = (float)(-(a11 * a32 - a12 * a31) / d);
                o[6] = (float)((a12 * a23 - a13 * a22) / d);
                o[7] = (float)(-(a11 * a23 - a13 * a21) / d);
                o[8] = (float)((a11 * a22 - a12 * a21) / d);
                w[p] = (float)sqrt(1.0 / d);
            } else {
                for (int k = 0; k < 9; ++k) o[k] = 100000.0f;
                w[p] = 0.0f;
                ++bad;
            }
        } else {
            double a1 = a[0], a2 = a[1], a3 = a[2], a4 = a[3];
            double d = a1 * a4 - a2 * a3;
            if (d > 0) {
                o[0] = (float)(a4 / d);
                o[1] = (float)(-a2 / d);
                o[2] = (float)(-a3 / d);
                o[3] = (float)(a1 / d);
                w[p] = (float)sqrt(1.0 / d);
            } else {
                for (int k = 0; k < 4; ++k) o[k] = 100000.0f;
                w[p] = 0.0f;
                ++bad;
            }
        }
    }
    return bad;
}

/* y' = R y + t in FP64, evaluated as ((R[a,0] y0 + R[a,1] y1) + R[a,2] y2) + t_a (update_sig.cu:247-249). */
static inline void pose_apply(int D, const double* R, const double* t, const float* y, double* yp)
{
    for (int a = 0; a < D; ++a) {
        double v = R[a] * (double)y[0] + R[a + D] * (double)y[1];
        if (D == 3) v = v + R[a + 6] * (double)y[2];
        yp[a] = v + t[a];
    }
}

void dugma_oracle_pose(int D, int m, const float* y, const double* R, const double* t, double* yp)
{
    for (int j = 0; j < m; ++j) pose_apply(D, R, t, y + (size_t)j * D, yp + (size_t)j * D);
}

/* C' = R A R^T (packed) for a packed symmetric A. */
static void rotate_sym(int D, const double* R, const double* Ap, double* Cp)
{
    double A[9], T[9], C[9];
    sym_unpack(D, Ap, A);
    for (int r = 0; r < D; ++r)
        for (int c = 0; c < D; ++c) {
            double s = 0;
            for (int k = 0; k < D; ++k) s += A[r + D * k] * R[c + D * k];   /* (A R^T)[r][c] */
            T[r + D * c] = s;
        }
    for (int r = 0; r < D; ++r)
        for (int c = 0; c < D; ++c) {
            double s = 0;
            for (int k = 0; k < D; ++k) s += R[r + D * k] * T[k + D * c];
            C[r + D * c] = s;
        }
    sym_pack(D, C, Cp);
}

static inline void symv(int D, const double* p, const double* v, double* out)
{
    if (D == 3) {
        out[0] = p[0] * v[0] + p[3] * v[1] + p[4] * v[2];
        out[1] = p[3] * v[0] + p[1] * v[1] + p[5] * v[2];
        out[2] = p[4] * v[0] + p[5] * v[1] + p[2] * v[2];
    } else {
        out[0] = p[0] * v[0] + p[2] * v[1];
        out[1] = p[2] * v[0] + p[1] * v[1];
    }
}

static inline void cross_acc(int D, const double* a, const double* b, double s, double* g)
{
    if (D == 3) {
        g[0] += s * (a[1] * b[2] - a[2] * b[1]);
        g[1] += s * (a[2] * b[0] - a[0] * b[2]);
        g[2] += s * (a[0] * b[1] - a[1] * b[0]);
    } else {
        g[0] += s * (a[0] * b[1] - a[1] * b[0]);
    }
}

typedef struct {
    int D, N, M;
    const float *x, *xinv, *wx, *y, *yinv, *wy;
} state_t;

/* Per-pose derived quantities in FP64: y'_j, C'_j = R (s A_j) R^T, B_i = s sym(Sigma_x_i^-1),
 * weights w_i = |Sigma_x|^-1/2 s^{D/2}, v_j likewise (compi.cu:646-677, 753-765). */
typedef struct {
    double *yp, *Cp, *B, *w, *v;
} derived_t;

static void derive(const state_t* st, const double* R, const double* t, double sig, derived_t* dv)
{
    int D = st->D, ns = nsym(D);
    double s = 1.0 / sig, sD = pow(s, 0.5 * D);
    dv->yp = (double*)malloc(sizeof(double) * st->M * D);
    dv->Cp = (double*)malloc(sizeof(double) * st->M * ns);
    dv->B = (double*)malloc(sizeof(double) * st->N * ns);
    dv->w = (double*)malloc(sizeof(double) * st->N);
    dv->v = (double*)malloc(sizeof(double) * st->M);
    for (int j = 0; j < st->M; ++j) {
        double full[9], Ap[6];
        pose_apply(D, R, t, st->y + (size_t)j * D, dv->yp + (size_t)j * D);
        for (int k = 0; k < D * D; ++k) full[k] = (double)st->yinv[(size_t)j * D * D + k] * s;
        sym_pack(D, full, Ap);
        rotate_sym(D, R, Ap, dv->Cp + (size_t)j * ns);
        dv->v[j] = (double)st->wy[j] * sD;
    }
    for (int i = 0; i < st->N; ++i) {
        double full[9];
        for (int k = 0; k < D * D; ++k) full[k] = (double)st->xinv[(size_t)i * D * D + k] * s;
        sym_pack(D, full, dv->B + (size_t)i * ns);
        dv->w[i] = (double)st->wx[i] * sD;
    }
}

static void derived_free(derived_t* dv)
{
    free(dv->yp); free(dv->Cp); free(dv->B); free(dv->w); free(dv->v);
}

/* ------------------------------------------------------------------------- */
/* REF energy and its adjoint.                                                */
/*   P_ij = w_i v_j [exp(-1/2 d^T C'_j d) + exp(-1/2 d^T B_i d)], d = x_i - y'_j */
/*   (compi.cu:753-772);  E = sum_ij P_ij.                                    */
/*   dE/dt     = sum w v (e1 C'd + e2 B d)                                    */
/*   dE/domega = sum w v (e1 (x_i - t) x C'd + e2 (R y_j) x B d)              */
/*   dE/dx_i   = -sum_j w v (e1 C'd + e2 B d)                                 */
/* out7 = [E, g(NR+D)] summed over rows [i0, i1); dEdx (nullable) rows i0..i1 */
/* ------------------------------------------------------------------------- */
int dugma_oracle_energy(int D, int N, int M, const float* x, const float* xinv, const float* wx,
                        const float* y, const float* yinv, const float* wy, const double* R,
                        const double* t, double sig, int i0, int i1, double* out, double* dEdx)
{
    state_t st = {D, N, M, x, xinv, wx, y, yinv, wy};
    derived_t dv;
    derive(&st, R, t, sig, &dv);
    int ns = nsym(D), NR = D == 3 ? 3 : 1, NG = NR + D;
    int nb = (i1 - i0 + ORACLE_BLOCK - 1) / ORACLE_BLOCK;
    double* part = (double*)calloc((size_t)nb * 8, sizeof(double));
#pragma omp parallel for schedule(dynamic, 1)
    for (int b = 0; b < nb; ++b) {
        double acc[8] = {0};
        int ib = i0 + b * ORACLE_BLOCK, ie = ib + ORACLE_BLOCK < i1 ? ib + ORACLE_BLOCK : i1;
        for (int i = ib; i < ie; ++i) {
            double xi[3], xt[3], Ei = 0, gi[6] = {0}, dxi[3] = {0};
            for (int a = 0; a < D; ++a) { xi[a] = x[(size_t)i * D + a]; xt[a] = xi[a] - t[a]; }
            const double* Bi = dv.B + (size_t)i * ns;
            for (int j = 0; j < M; ++j) {
                const double* yp = dv.yp + (size_t)j * D;
                double d[3], u1[3], u2[3], r[3], m1 = 0, m2 = 0;
                for (int a = 0; a < D; ++a) d[a] = xi[a] - yp[a];
                symv(D, dv.Cp + (size_t)j * ns, d, u1);
                symv(D, Bi, d, u2);
                for (int a = 0; a < D; ++a) { m1 += d[a] * u1[a]; m2 += d[a] * u2[a]; r[a] = yp[a] - t[a]; }
                double vv = dv.v[j], e1 = exp(-0.5 * m1), e2 = exp(-0.5 * m2);
                Ei += vv * (e1 + e2);
                double a1 = vv * e1, a2 = vv * e2;
                cross_acc(D, xt, u1, a1, gi);
                cross_acc(D, r, u2, a2, gi);
                for (int a = 0; a < D; ++a) {
                    double ga = a1 * u1[a] + a2 * u2[a];
                    gi[NR + a] += ga;
                    dxi[a] -= ga;
                }
            }
            double wi = dv.w[i];
            acc[0] += wi * Ei;
            for (int k = 0; k < NG; ++k) acc[1 + k] += wi * gi[k];
            if (dEdx)
                for (int a = 0; a < D; ++a) dEdx[(size_t)(i - i0) * D + a] = wi * dxi[a];
        }
        memcpy(part + (size_t)b * 8, acc, sizeof(acc));
    }
    for (int k = 0; k < 1 + NG; ++k) out[k] = 0;
    for (int b = 0; b < nb; ++b)
        for (int k = 0; k < 1 + NG; ++k) out[k] += part[(size_t)b * 8 + k];
    free(part);
    derived_free(&dv);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* CONV energy: sum_ij N(d; 0, S_ij), S_ij = sig (R Sigma_y_j R^T + Sigma_x_i),  */
/* with the Gaussian normaliser (2 pi)^{-D/2} |S|^{-1/2}.  Covariances are the  */
/* FP32-rounded inputs (packed symmetric), not their inverses.                  */
/*   df/dt = u,  df/domega = r x u + (Sy u) x u - axial(Sy S^-1)                */
/*   with f = log N, u = S^-1 d, r = R y_j, Sy = sig R Sigma_y R^T,             */
/*   axial(A) = (A23 - A32, A31 - A13, A12 - A21)  (2D: A12 - A21).             */
/* ------------------------------------------------------------------------- */
static void sym_inv_det(int D, const double* S, double* Si, double* det)
{
    if (D == 3) {
        double a = S[0], b = S[1], c = S[2], d = S[3], e = S[4], f = S[5];
        /* [[a d e],[d b f],[e f c]] */
        double c00 = b * c - f * f, c01 = e * f - d * c, c02 = d * f - b * e;
        double c11 = a * c - e * e, c12 = d * e - a * f, c22 = a * b - d * d;
        double dt = a * c00 + d * c01 + e * c02;
        *det = dt;
        Si[0] = c00 / dt; Si[1] = c11 / dt; Si[2] = c22 / dt;
        Si[3] = c01 / dt; Si[4] = c02 / dt; Si[5] = c12 / dt;
    } else {
        double a = S[0], b = S[1], c = S[2];
        double dt = a * b - c * c;
        *det = dt;
        Si[0] = b / dt; Si[1] = a / dt; Si[2] = -c / dt;
    }
}

int dugma_oracle_energy_conv(int D, int N, int M, const float* x, const float* xcov,
                             const float* y, const float* ycov, const double* R, const double* t,
                             double sig, int i0, int i1, double* out, double* dEdx)
{
    int ns = nsym(D), NR = D == 3 ? 3 : 1, NG = NR + D;
    double* yp = (double*)malloc(sizeof(double) * M * D);
    double* Sy = (double*)malloc(sizeof(double) * M * ns);
    double* Sx = (double*)malloc(sizeof(double) * N * ns);
    const double norm = pow(2.0 * M_PI, -0.5 * D);
    for (int j = 0; j < M; ++j) {
        double full[9], p[6];
        pose_apply(D, R, t, y + (size_t)j * D, yp + (size_t)j * D);
        for (int k = 0; k < D * D; ++k) full[k] = (double)ycov[(size_t)j * D * D + k] * sig;
        sym_pack(D, full, p);
        rotate_sym(D, R, p, Sy + (size_t)j * ns);
    }
    for (int i = 0; i < N; ++i) {
        double full[9];
        for (int k = 0; k < D * D; ++k) full[k] = (double)xcov[(size_t)i * D * D + k] * sig;
        sym_pack(D, full, Sx + (size_t)i * ns);
    }
    int nb = (i1 - i0 + ORACLE_BLOCK - 1) / ORACLE_BLOCK;
    double* part = (double*)calloc((size_t)nb * 8, sizeof(double));
#pragma omp parallel for schedule(dynamic, 1)
    for (int b = 0; b < nb; ++b) {
        double acc[8] = {0};
        int ib = i0 + b * ORACLE_BLOCK, ie = ib + ORACLE_BLOCK < i1 ? ib + ORACLE_BLOCK : i1;
        for (int i = ib; i < ie; ++i) {
            double dxi[3] = {0};
            for (int j = 0; j < M; ++j) {
                double S[6], Si[6], det, d[3] = {0, 0, 0}, u[3] = {0, 0, 0}, r[3] = {0, 0, 0}, Su[3] = {0, 0, 0}, m = 0;
                for (int k = 0; k < ns; ++k) S[k] = Sy[(size_t)j * ns + k] + Sx[(size_t)i * ns + k];
                sym_inv_det(D, S, Si, &det);
                if (!(det > 0)) continue;
                for (int a = 0; a < D; ++a) {
                    d[a] = (double)x[(size_t)i * D + a] - yp[(size_t)j * D + a];
                    r[a] = yp[(size_t)j * D + a] - t[a];
                }
                symv(D, Si, d, u);
                for (int a = 0; a < D; ++a) m += d[a] * u[a];
                double Nij = norm / sqrt(det) * exp(-0.5 * m);
                acc[0] += Nij;
                /* rotation part */
                const double* sy = Sy + (size_t)j * ns;
                symv(D, sy, u, Su);
                double A[9], SyF[9], SiF[9];
                sym_unpack(D, sy, SyF);
                sym_unpack(D, Si, SiF);
                for (int rr = 0; rr < D; ++rr)
                    for (int cc = 0; cc < D; ++cc) {
                        double s = 0;
                        for (int k = 0; k < D; ++k) s += SyF[rr + D * k] * SiF[k + D * cc];
                        A[rr + D * cc] = s;
                    }
                double gw[3] = {0};
                cross_acc(D, r, u, 1.0, gw);
                cross_acc(D, Su, u, 1.0, gw);
                if (D == 3) {
                    gw[0] -= A[1 + 3 * 2] - A[2 + 3 * 1];
                    gw[1] -= A[2 + 3 * 0] - A[0 + 3 * 2];
                    gw[2] -= A[0 + 3 * 1] - A[1 + 3 * 0];
                } else {
                    gw[0] -= A[0 + 2 * 1] - A[1 + 2 * 0];
                }
                for (int k = 0; k < NR; ++k) acc[1 + k] += Nij * gw[k];
                for (int a = 0; a < D; ++a) {
                    acc[1 + NR + a] += Nij * u[a];
                    dxi[a] -= Nij * u[a];
                }
            }
            if (dEdx)
                for (int a = 0; a < D; ++a) dEdx[(size_t)(i - i0) * D + a] = dxi[a];
        }
        memcpy(part + (size_t)b * 8, acc, sizeof(acc));
    }
    for (int k = 0; k < 1 + NG; ++k) out[k] = 0;
    for (int b = 0; b < nb; ++b)
        for (int k = 0; k < 1 + NG; ++k) out[k] += part[(size_t)b * 8 + k];
    free(part); free(yp); free(Sy); free(Sx);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Nearest neighbours in the specified FP32 sequence (update_sig.cu:238-259): */
/*   y'_j = (float) FP64(R y_j + t); d = x_i - y'_j in FP32;                   */
/*   d2 = fmaf(d2, d2, fmaf(d1, d1, d0 * d0))  (2D: fmaf(d1, d1, d0 * d0));    */
/*   ordered by (d2, j): ties go to the lowest j.  k <= 16 neighbours, sorted. */
/* ------------------------------------------------------------------------- */
int dugma_oracle_nn(int D, int N, int M, const float* x, const float* y, const double* R,
                    const double* t, int k, int* idx, float* d2out)
{
    if (k < 1 || k > 16 || k > M) return 1;
    float* yp = (float*)malloc(sizeof(float) * M * D);
    for (int j = 0; j < M; ++j) {
        double v[3];
        pose_apply(D, R, t, y + (size_t)j * D, v);
        for (int a = 0; a < D; ++a) yp[(size_t)j * D + a] = (float)v[a];
    }
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < N; ++i) {
        float bd[16];
        int bi[16];
        for (int q = 0; q < k; ++q) { bd[q] = INFINITY; bi[q] = 0x7fffffff; }
        const float* xi = x + (size_t)i * D;
        for (int j = 0; j < M; ++j) {
            const float* yj = yp + (size_t)j * D;
            float d0 = xi[0] - yj[0], d1 = xi[1] - yj[1], dd;
            if (D == 3) {
                float dz = xi[2] - yj[2];
                dd = fmaf(dz, dz, fmaf(d1, d1, d0 * d0));
            } else {
                dd = fmaf(d1, d1, d0 * d0);
            }
            if (dd < bd[k - 1]) {      /* strict: an equal later j never displaces an earlier one */
                int q = k - 1;
                while (q > 0 && dd < bd[q - 1]) { bd[q] = bd[q - 1]; bi[q] = bi[q - 1]; --q; }
                bd[q] = dd;
                bi[q] = j;
            }
        }
        for (int q = 0; q < k; ++q) {
            idx[(size_t)i * k + q] = bi[q];
            d2out[(size_t)i * k + q] = bd[q];
        }
    }
    free(yp);
    return 0;
}

/* sigma from nearest squared distances:
 *   exact: sum_i d2_i / (D N) in FP64;
 *   quantised (update_sig.cu:253-258, 79-91, 384-385): q_i = rn_u32((d2_i / D) * 1e6) in FP32,
 *   sigma = (sum_i q_i) / 1e6 / N, returned as float. */
double dugma_oracle_sigma(int D, int N, const float* d2min, int quantised)
{
    if (!quantised) {
        double s = 0;
        for (int i = 0; i < N; ++i) s += (double)d2min[i];
        return s / ((double)D * N);
    }
    uint64_t q = 0;
    for (int i = 0; i < N; ++i) {
        float v = (d2min[i] / (float)D) * 1000000.0f;
        float r = nearbyintf(v);
        uint32_t u = r >= 4294967295.0f ? 0xffffffffu : (r <= 0 ? 0u : (uint32_t)r);
        q += u;
    }
    return (double)(float)((double)q / 1e6 / (double)N);
}

/* ------------------------------------------------------------------------- */
/* Surrogate coefficients (compi): A_k = sum_ij P_ij c_k(x_i, B_i, y'_j, C'_j) */
/* in FP64, 637 (3D) / 45 (2D) entries in the energy3D.m / energy2D.m order;  */
/* out has 640 slots, the unused tail is zero (compi.cpp:47-64).               */
/* ------------------------------------------------------------------------- */
int dugma_oracle_coef(int D, int N, int M, const float* x, const float* xinv, const float* wx,
                      const float* y, const float* yinv, const float* wy, const double* R,
                      const double* t, double sig, double* out640)
{
    state_t st = {D, N, M, x, xinv, wx, y, yinv, wy};
    derived_t dv;
    derive(&st, R, t, sig, &dv);
    int ns = nsym(D), K = D == 3 ? 637 : 45;
    int nb = (N + ORACLE_BLOCK - 1) / ORACLE_BLOCK;
    double* part = (double*)calloc((size_t)nb * 640, sizeof(double));
#pragma omp parallel for schedule(dynamic, 1)
    for (int b = 0; b < nb; ++b) {
        double* acc = part + (size_t)b * 640;
        double c[640];
        int ib = b * ORACLE_BLOCK, ie = ib + ORACLE_BLOCK < N ? ib + ORACLE_BLOCK : N;
        for (int i = ib; i < ie; ++i) {
            double xi[3];
            for (int a = 0; a < D; ++a) xi[a] = x[(size_t)i * D + a];
            const double* Bi = dv.B + (size_t)i * ns;
            for (int j = 0; j < M; ++j) {
                const double* yp = dv.yp + (size_t)j * D;
                const double* Cp = dv.Cp + (size_t)j * ns;
                double d[3], u1[3], u2[3], m1 = 0, m2 = 0;
                for (int a = 0; a < D; ++a) d[a] = xi[a] - yp[a];
                symv(D, Cp, d, u1);
                symv(D, Bi, d, u2);
                for (int a = 0; a < D; ++a) { m1 += d[a] * u1[a]; m2 += d[a] * u2[a]; }
                double P = dv.w[i] * dv.v[j] * (exp(-0.5 * m1) + exp(-0.5 * m2));
                if (D == 3) coef_terms_3d(xi, Bi, yp, Cp, c);
                else coef_terms_2d(xi, Bi, yp, Cp, c);
                for (int k = 0; k < K; ++k) acc[k] += P * c[k];
            }
        }
    }
    for (int k = 0; k < 640; ++k) out640[k] = 0;
    for (int b = 0; b < nb; ++b)
        for (int k = 0; k < K; ++k) out640[k] += part[(size_t)b * 640 + k];
    free(part);
    derived_free(&dv);
    return 0;
}

/* Surrogate value Q(dR, dt) = sum_k A_k b_k (energy3D.m:15-16 / energy2D.m:7-8);
 * v = [t1 t2 t3 r11 r12 r13 r21 r22 r23 r31 r32 r33] (3D) or [t1 t2 r11 r21] (2D). */
double dugma_oracle_surrogate(int D, const double* A, const double* v, const unsigned char* exps)
{
    int K = D == 3 ? 637 : 45, nv = D == 3 ? 12 : 4;
    double s = 0;
    for (int k = 0; k < K; ++k) {
        double m = 1;
        for (int q = 0; q < nv; ++q)
            for (int e = 0; e < exps[k * nv + q]; ++e) m *= v[q];
        s += A[k] * m;
    }
    return s;
}

/* Use n OpenMP threads from now on (n < 1: leave the setting alone); returns the count in use.
 * Launchers such as torchrun pin OMP_NUM_THREADS to 1; timing code sets all host cores back. */
int dugma_oracle_set_threads(int n)
{
#ifdef _OPENMP
    if (n >= 1) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

int dugma_oracle_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

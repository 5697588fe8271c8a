// knn_cov.cu -- per-point covariances from the k nearest neighbours (data preparation).
//
// For every point p_i: the k nearest other points by the brute-force kernel of nn.cu (a
// self-join, k + 1 neighbours with the point itself first), their sample covariance
// together with p_i (divided by k), and an eigenvalue clamp to [lo, hi] so that every
// covariance is positive definite with a bounded condition number.  Eigen-decomposition
// by cyclic Jacobi rotations in FP64.
#include <cmath>

#include "context.hpp"

namespace dugma {

template <int D>
__device__ void jacobi_sym(double (&A)[3][3], double (&V)[3][3])
{
    for (int r = 0; r < D; ++r)
        for (int c = 0; c < D; ++c) V[r][c] = r == c ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 12; ++sweep) {
        double off = 0;
        for (int p = 0; p < D; ++p)
            for (int q = p + 1; q < D; ++q) off += A[p][q] * A[p][q];
        if (off < 1e-40) break;
        for (int p = 0; p < D; ++p)
            for (int q = p + 1; q < D; ++q) {
                if (fabs(A[p][q]) < 1e-300) continue;
                const double th = 0.5 * (A[q][q] - A[p][p]) / A[p][q];
                const double t = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < D; ++k) {   // A <- J^T A J
                    const double akp = A[k][p], akq = A[k][q];
                    A[k][p] = c * akp - s * akq;
                    A[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < D; ++k) {
                    const double apk = A[p][k], aqk = A[q][k];
                    A[p][k] = c * apk - s * aqk;
                    A[q][k] = s * apk + c * aqk;
                }
                for (int k = 0; k < D; ++k) {
                    const double vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = c * vkp - s * vkq;
                    V[k][q] = s * vkp + c * vkq;
                }
            }
    }
}

template <int D>
__global__ void knn_cov_kernel(const double* __restrict__ pts, const int* __restrict__ idx, int n, int kk, double lo,
                               double hi, double* __restrict__ cov)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double mean[3] = {0, 0, 0};
        // the point itself plus the first k other points of its k + 1 nearest (itself is among
        // them unless more than k others coincide with it)
        int list[17];
        int m = 0;
        list[m++] = i;
        for (int q = 0; q < kk && m < kk; ++q) {
            const int j = idx[(size_t)i * kk + q];
            if (j != i) list[m++] = j;
        }
        for (int q = 0; q < m; ++q)
            for (int a = 0; a < D; ++a) mean[a] += pts[(size_t)list[q] * D + a] / m;
        double A[3][3] = {}, V[3][3];
        for (int q = 0; q < m; ++q) {
            double c[3];
            for (int a = 0; a < D; ++a) c[a] = pts[(size_t)list[q] * D + a] - mean[a];
            for (int a = 0; a < D; ++a)
                for (int b = 0; b < D; ++b) A[a][b] += c[a] * c[b] / (m - 1);
        }
        jacobi_sym<D>(A, V);
        double w[3];
        for (int a = 0; a < D; ++a) w[a] = fmin(fmax(A[a][a], lo), hi);
        for (int a = 0; a < D; ++a)
            for (int b = 0; b < D; ++b) {
                double s = 0;
                for (int k = 0; k < D; ++k) s += V[a][k] * w[k] * V[b][k];
                cov[(size_t)i * D * D + a + D * b] = s;
            }
    }
}

}  // namespace dugma

using namespace dugma;

// points (n x D, MATLAB layout) -> covariances (n blocks of D x D, column-major), k <= 15
extern "C" int dugma_knn_covariance(const double* points, int n, int D, int k, double lo, double hi, double* cov)
{
    if (!points || !cov || n < 2 || (D != 2 && D != 3) || k < 1 || k > 15 || k >= n || !(lo > 0) || !(hi >= lo))
        return set_error(DUGMA_ERR_ARG, "knn_covariance: need n >= 2, D in {2,3}, 1 <= k <= min(15, n-1), 0 < lo <= hi");
    // a self-join context: both clouds are the points, identity covariances
    std::vector<double> eye((size_t)n * D * D, 0.0);
    for (int i = 0; i < n; ++i)
        for (int a = 0; a < D; ++a) eye[(size_t)i * D * D + a * (D + 1)] = 1.0;
    float* Ptr[6];
    double ok = 0;
    int rc = dugma_init(points, eye.data(), points, eye.data(), &ok, n, n, D, Ptr);
    if (rc != DUGMA_OK) return rc;
    Context* c = find_context(Ptr);
    const int kk = k + 1;
    int* idx = nullptr;
    float* d2 = nullptr;
    double* covd = nullptr;
    double* ptsd = nullptr;   // FP64 copy: neighbour sets come from FP32 distances, moments from FP64
    const double ident[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, ident2[4] = {1, 0, 0, 1};
    cudaStream_t s = c->stream;
    do {
        // the pose block goes through the context's pinned staging (stream-ordered copy)
        double* h = c->host;
        for (int q = 0; q < 16; ++q) h[q] = 0.0;
        for (int q = 0; q < D * D; ++q) h[q] = D == 3 ? ident[q] : ident2[q];
        h[kPoseSig] = 1.0;
        if (cudaMemcpyAsync(c->pose, h, sizeof(double) * 16, cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaMallocAsync(&idx, sizeof(int) * (size_t)n * kk, s) != cudaSuccess ||
            cudaMallocAsync(&d2, sizeof(float) * (size_t)n * kk, s) != cudaSuccess ||
            cudaMallocAsync(&covd, sizeof(double) * (size_t)n * D * D, s) != cudaSuccess ||
            cudaMallocAsync(&ptsd, sizeof(double) * (size_t)n * D, s) != cudaSuccess ||
            cudaMemcpyAsync(ptsd, points, sizeof(double) * (size_t)n * D, cudaMemcpyHostToDevice, s) != cudaSuccess) {
            cudaGetLastError();
            rc = set_error(DUGMA_ERR_NOMEM, "knn_covariance: device allocation failed");
            break;
        }
        rc = launch_nn(*c, c->pose, kk, idx, d2, s);
        if (rc != DUGMA_OK) break;
        const int g = std::min((n + 127) / 128, c->num_sms * 8);
        if (D == 3)
            knn_cov_kernel<3><<<g, 128, 0, s>>>(ptsd, idx, n, kk, lo, hi, covd);
        else
            knn_cov_kernel<2><<<g, 128, 0, s>>>(ptsd, idx, n, kk, lo, hi, covd);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpyAsync(cov, covd, sizeof(double) * (size_t)n * D * D, cudaMemcpyDeviceToHost, s) != cudaSuccess)
            rc = set_error(DUGMA_ERR_CUDA, "knn_covariance: kernel failed");
    } while (false);
    if (idx) cudaFreeAsync(idx, s);
    if (d2) cudaFreeAsync(d2, s);
    if (covd) cudaFreeAsync(covd, s);
    if (ptsd) cudaFreeAsync(ptsd, s);
    if (cudaStreamSynchronize(s) != cudaSuccess && rc == DUGMA_OK)
        rc = set_error(DUGMA_ERR_CUDA, "knn_covariance: kernel failed");
    dugma_fr_m(Ptr);
    return rc;
}

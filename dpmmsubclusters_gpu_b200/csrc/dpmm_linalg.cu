// Small FP64 matrix helpers of the reference's device back-end, for callers that keep the reference's
// own NIW parameter sampler (niw::sample_distribution, priors/niw.cpp:61-107, calls both):
//   cudaKernel::inverse_matrix (cudaKernel.cu:1558-1598)                      B = A^-1
//   cudaKernel::multiplie_matrix_for_inverseWishart (cudaKernel.cu:980-1016)  C = (A B)(A B)^T
// Both run on the context's stream, from and to host arrays in the reference's (Eigen) column-major
// layout.  The reference inverts by Gauss-Jordan without pivoting (four launches per pivot) and forms
// the product with two cuBLAS DGEMMs; here one CTA inverts with partial pivoting (the same inverse to
// FP64 rounding, and a singular matrix is reported instead of dividing by zero), and one kernel per
// product forms each output element as an FP64 dot product.
#include "dpmm_internal.h"

namespace dpmm {
namespace {

constexpr int kInvThreads = 512;
constexpr int kInvWarps = kInvThreads / 32;
constexpr int kMaxLinalgDim = 2048;    // one CTA inverts: n^3 / 512 updates per thread at the limit

// In-place Gauss-Jordan inverse of the n x n matrix a by one CTA, with partial pivoting.  The array is
// read as row-major; for the caller's column-major matrix that is the transpose, and the inverse of
// the transpose is the transpose of the inverse, so the result is in the caller's layout too.
// col: n doubles of scratch (the pivot column), piv: n row exchanges, status: 1 when a pivot column
// has no nonzero entry on or below the diagonal (singular), 2 when the inverse is not finite.
__global__ void __launch_bounds__(kInvThreads) k_gauss_jordan_inverse(double* __restrict__ a, int n,
                                                                       double* __restrict__ col,
                                                                       int32_t* __restrict__ piv,
                                                                       int32_t* __restrict__ status)
{
    __shared__ double s_val[kInvWarps];
    __shared__ int s_idx[kInvWarps];
    __shared__ int s_p, s_bad;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const size_t nn = (size_t)n;
    if (tid == 0) s_bad = 0;
    for (int k = 0; k < n; ++k) {
        // pivot row: the largest |a[i][k]|, i >= k (the lowest index among equals)
        double best = -1.0;
        int bi = k;
        for (int i = k + tid; i < n; i += kInvThreads) {
            const double v = fabs(a[i * nn + k]);
            if (v > best) {
                best = v;
                bi = i;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_down_sync(0xffffffffu, best, o);
            const int oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) {
                best = ov;
                bi = oi;
            }
        }
        if (lane == 0) {
            s_val[warp] = best;
            s_idx[warp] = bi;
        }
        __syncthreads();
        if (tid == 0) {
            double b = s_val[0];
            int p = s_idx[0];
            for (int w = 1; w < kInvWarps; ++w)
                if (s_val[w] > b || (s_val[w] == b && s_idx[w] < p)) {
                    b = s_val[w];
                    p = s_idx[w];
                }
            if (!(b > 0.0)) s_bad = 1;   // zero (or NaN) on and below the diagonal
            s_p = p;
            piv[k] = p;
        }
        __syncthreads();
        if (s_bad) break;
        const int p = s_p;
        if (p != k)
            for (int j = tid; j < n; j += kInvThreads) {
                const double t = a[k * nn + j];
                a[k * nn + j] = a[p * nn + j];
                a[p * nn + j] = t;
            }
        __syncthreads();
        // the pivot column (the multipliers) before any row changes it
        for (int i = tid; i < n; i += kInvThreads) col[i] = a[i * nn + k];
        __syncthreads();
        const double inv = 1.0 / col[k];
        // row k scaled (its diagonal entry becomes 1 / pivot)
        for (int j = tid; j < n; j += kInvThreads) a[k * nn + j] = (j == k ? 1.0 : a[k * nn + j]) * inv;
        __syncthreads();
        // the other rows: a[i][j] -= col[i] a[k][j], with a[i][k] = -col[i] / pivot
        for (size_t e = tid; e < nn * nn; e += kInvThreads) {
            const size_t i = e / nn, j = e % nn;
            if (i == (size_t)k) continue;
            a[e] = (j == (size_t)k ? 0.0 : a[e]) - col[i] * a[k * nn + j];
        }
        __syncthreads();
    }
    if (s_bad) {
        if (tid == 0) *status = 1;
        return;
    }
    // undo the row exchanges on the columns, last first
    for (int k = n - 1; k >= 0; --k) {
        const int p = piv[k];
        if (p != k)
            for (int i = tid; i < n; i += kInvThreads) {
                const double t = a[i * nn + k];
                a[i * nn + k] = a[i * nn + p];
                a[i * nn + p] = t;
            }
        __syncthreads();
    }
    int finite = 1;
    for (size_t e = tid; e < nn * nn; e += kInvThreads) finite &= isfinite(a[e]) ? 1 : 0;
    if (!__syncthreads_and(finite) && tid == 0) *status = 2;
}

// t = a b: a m x n, b n x k, t m x k, all column-major
__global__ void k_matmul_cm(const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ t, int m,
                            int n, int k)
{
    const size_t total = (size_t)m * k;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const size_t i = e % m, l = e / m;
        double s = 0.0;
        for (int j = 0; j < n; ++j) s = fma(a[i + (size_t)m * j], b[j + (size_t)n * l], s);
        t[e] = s;
    }
}

// c = t t^T: t m x k, c m x m, column-major
__global__ void k_gram_cm(const double* __restrict__ t, double* __restrict__ c, int m, int k)
{
    const size_t total = (size_t)m * m;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const size_t i = e % m, i2 = e / m;
        double s = 0.0;
        for (int l = 0; l < k; ++l) s = fma(t[i + (size_t)m * l], t[i2 + (size_t)m * l], s);
        c[e] = s;
    }
}

dpmm_status linalg_scratch(dpmm_ctx* c, size_t bytes)
{
    if (c->linalg_bytes >= bytes) return DPMM_OK;
    if (c->d_linalg) cudaFree(c->d_linalg);
    c->d_linalg = nullptr;
    c->linalg_bytes = 0;
    if (cudaMalloc(&c->d_linalg, bytes) != cudaSuccess) {
        cudaGetLastError();
        return fail(DPMM_ERR_OOM, "matrix helper scratch: cudaMalloc failed");
    }
    c->linalg_bytes = bytes;
    return DPMM_OK;
}

int grid_for(size_t total)
{
    return (int)std::min<size_t>((total + 255) / 256, 148 * 8);
}

}  // namespace
}  // namespace dpmm

using namespace dpmm;

extern "C" dpmm_status dpmm_inverse_matrix(dpmm_ctx* c, int n, const double* A, double* B)
{
    if (!c || !A || !B || n < 1 || n > kMaxLinalgDim)
        return fail(DPMM_ERR_INVALID_ARG, "dpmm_inverse_matrix: null argument or n outside 1 .. 2048");
    DPMM_CUDA_TRY(cudaSetDevice(c->device));
    const size_t nn = (size_t)n * n;
    const size_t a_bytes = (nn * sizeof(double) + 255) & ~(size_t)255;
    const size_t col_bytes = ((size_t)n * sizeof(double) + 255) & ~(size_t)255;
    const size_t piv_bytes = ((size_t)n * sizeof(int32_t) + 255) & ~(size_t)255;
    DPMM_TRY(linalg_scratch(c, a_bytes + col_bytes + piv_bytes + 256));
    uint8_t* base = reinterpret_cast<uint8_t*>(c->d_linalg);
    double* d_a = reinterpret_cast<double*>(base);
    double* d_col = reinterpret_cast<double*>(base + a_bytes);
    int32_t* d_piv = reinterpret_cast<int32_t*>(base + a_bytes + col_bytes);
    int32_t* d_status = reinterpret_cast<int32_t*>(base + a_bytes + col_bytes + piv_bytes);
    DPMM_CUDA_TRY(cudaMemcpyAsync(d_a, A, nn * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    DPMM_CUDA_TRY(cudaMemsetAsync(d_status, 0, sizeof(int32_t), c->stream));
    k_gauss_jordan_inverse<<<1, kInvThreads, 0, c->stream>>>(d_a, n, d_col, d_piv, d_status);
    DPMM_LAUNCHED();
    int32_t* h_status = reinterpret_cast<int32_t*>(c->h_pinned);
    DPMM_CUDA_TRY(cudaMemcpyAsync(h_status, d_status, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaMemcpyAsync(B, d_a, nn * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    g_h2d_bytes += nn * sizeof(double);
    g_d2h_bytes += nn * sizeof(double);
    if (*h_status == 1) return fail(DPMM_ERR_NUMERIC, "dpmm_inverse_matrix: the matrix is singular");
    if (*h_status == 2) return fail(DPMM_ERR_NUMERIC, "dpmm_inverse_matrix: the inverse is not finite");
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_multiply_for_inverse_wishart(dpmm_ctx* c, int m, int n, int k, const double* A,
                                                         const double* B, double* C)
{
    if (!c || !A || !B || !C || m < 1 || n < 1 || k < 1 || m > kMaxLinalgDim || n > kMaxLinalgDim ||
        k > kMaxLinalgDim)
        return fail(DPMM_ERR_INVALID_ARG,
                    "dpmm_multiply_for_inverse_wishart: null argument or a size outside 1 .. 2048");
    DPMM_CUDA_TRY(cudaSetDevice(c->device));
    auto round = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t ab = round((size_t)m * n * sizeof(double)), bb = round((size_t)n * k * sizeof(double));
    const size_t tb = round((size_t)m * k * sizeof(double)), cb = round((size_t)m * m * sizeof(double));
    DPMM_TRY(linalg_scratch(c, ab + bb + tb + cb));
    uint8_t* base = reinterpret_cast<uint8_t*>(c->d_linalg);
    double* d_a = reinterpret_cast<double*>(base);
    double* d_b = reinterpret_cast<double*>(base + ab);
    double* d_t = reinterpret_cast<double*>(base + ab + bb);
    double* d_c = reinterpret_cast<double*>(base + ab + bb + tb);
    DPMM_CUDA_TRY(cudaMemcpyAsync(d_a, A, (size_t)m * n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    DPMM_CUDA_TRY(cudaMemcpyAsync(d_b, B, (size_t)n * k * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    k_matmul_cm<<<grid_for((size_t)m * k), 256, 0, c->stream>>>(d_a, d_b, d_t, m, n, k);
    DPMM_LAUNCHED();
    k_gram_cm<<<grid_for((size_t)m * m), 256, 0, c->stream>>>(d_t, d_c, m, k);
    DPMM_LAUNCHED();
    DPMM_CUDA_TRY(cudaMemcpyAsync(C, d_c, (size_t)m * m * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    g_h2d_bytes += ((size_t)m * n + (size_t)n * k) * sizeof(double);
    g_d2h_bytes += (size_t)m * m * sizeof(double);
    return DPMM_OK;
}

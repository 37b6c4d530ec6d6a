// dpmm_niw.cuh -- FP64 block-level helpers shared by the Hastings kernels (dpmm_hastings.cu) and the
// split/merge screen (dpmm_screen.cu): the posterior + log marginal likelihood of NIW statistics with a
// register-resident Cholesky, the Dirichlet-multinomial marginal likelihood, a triangular inverse.
//
// Reference arithmetic restated (DPMMSubClusters/):
//   posterior            priors/niw.cpp:23-49, priors/multinomial_prior.cpp:12-22
//   log marginal lik.    priors/niw.cpp:122-138 (+ logdet.h:4-26 Cholesky branch,
//                        utils.cpp:94-102), priors/multinomial_prior.cpp:56-67
// lgamma is CUDA's lgamma(double).
#pragma once

#include <math.h>

#include "dpmm_internal.h"

namespace dpmm {

// ------------------------------------------------------------------------------ block-level helpers
// One block per statistics slot or pair: kHThreads threads for the Dirichlet terms and reductions; the
// NIW kernels run RegChol<DP>::T threads (below).

constexpr int kHThreads = 128;

static __device__ __forceinline__ double warp_sum_d(double v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// sum over the block (red: 33 doubles of shared memory); every thread gets the total
static __device__ double block_sum(double v, double* red)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v = warp_sum_d(v);
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) s += red[q];
        red[32] = s;
    }
    __syncthreads();
    return red[32];
}

// In-place inverse of the lower triangular A (non-unit diagonal) by the block, column by column from
// the last (the order of LAPACK's unblocked triangular inverse): A(j,j) = 1 / A(j,j), then
// A(j+1:, j) = -A(j,j) * inv(A)(j+1:, j+1:) * A(j+1:, j).  Needs D <= blockDim.x.
static __device__ void block_tri_inverse(double* A, int D)
{
    const int i0 = threadIdx.x;
    for (int j = D - 1; j >= 0; --j) {
        double* cj = A + (size_t)j * D;
        const double inv = 1.0 / cj[j];
        double y = 0.0;
        const int i = i0;
        if (i > j && i < D)
            for (int k = j + 1; k <= i; ++k) y += A[(size_t)k * D + i] * cj[k];
        __syncthreads();
        if (i > j && i < D) cj[i] = -inv * y;
        if (i0 == 0) cj[j] = inv;
        __syncthreads();
    }
}

// Optional by-products of niw_lml_reg for the screen: sum of log diag(psi') (the Hadamard bound of log
// det psi'), trace(psi') and log det psi' itself.
struct NiwExtras {
    double hd, tr, ld;
};

// Dirichlet-multinomial log marginal likelihood of statistics (n, sum [+ sum2]) by the block
static __device__ double mult_lml_block(int D, double n, const double* sum, const double* sum2, const double* alpha0,
                                        double* red)
{
    if (n == 0) return 0.0;
    double s0 = 0, sp = 0, acc = 0;
    for (int d = threadIdx.x; d < D; d += blockDim.x) {
        const double a0 = alpha0[d], ap = a0 + (sum2 ? sum[d] + sum2[d] : sum[d]);
        s0 += a0;
        sp += ap;
        acc += lgamma(ap) - lgamma(a0);
    }
    s0 = block_sum(s0, red);
    sp = block_sum(sp, red);
    acc = block_sum(acc, red);
    return lgamma(s0) - lgamma(sp) + acc;
}

// ------------------------------------------------------------------------------ register-resident forms
// The posterior scale matrix of one statistics slot (or pair), factored by one block with the factor
// held in registers: thread t owns row i = t % DP and the columns k = c, c + C, c + 2C, ... (c = t / DP)
// of that row, so a column step updates EP independent registers per thread.  Column j travels to
// every thread through a double-buffered shared vector: one block barrier per column.
template <int DP>
struct RegChol {
    static constexpr int T = DP > 64 ? 256 : 128;                      // threads per block
    static constexpr int C = (T / DP) < DP ? (T / DP) : DP;          // column classes
    static constexpr int EP = DP / C;                                 // registers per thread
    static constexpr int SMEM = 4 * DP + 33;                          // doubles: buf[2][DP], mp[DP], red[33], piv[DP]
};

// In-place Cholesky of the symmetric D x D matrix held in registers as above (a[q] = A(i, c + q C) for
// c + q C <= i; D <= DP), by the block: for each column j, A(i,k) -= A(i,j) A(k,j) / A(j,j) for
// j < k <= i, with A(j,j) the pivot.  Returns log det A = sum of log pivots in every thread, or NaN if
// a pivot is not positive.  Lout (nullable, shared D*D column-major) receives the lower factor.
// sh: RegChol<DP>::SMEM doubles (buf[2][DP] at 0, red[33] at 3 DP, piv[DP] after it).
template <int DP>
__device__ double reg_chol_logdet(double (&a)[RegChol<DP>::EP], int D, double* sh, double* Lout)
{
    using RC = RegChol<DP>;
    double* buf = sh;
    double* red = sh + 3 * DP;
    double* piv = red + 33;
    const int t = threadIdx.x;
    const int i = t % DP, c = t / DP;
    const bool act = c < RC::C && i < D;
    if (act && c == 0) buf[i] = a[0];             // column 0, raw (k = 0 is register 0 of class 0)
    __syncthreads();
    for (int j = 0; j < D; ++j) {
        const double* col = buf + (j & 1) * DP;
        double* nxt = buf + ((j + 1) & 1) * DP;
        const double p = col[j];
        const double pv = p > 0 ? p : 1.0;
        if (t == 0) piv[j] = p;
        if (Lout && c == j % RC::C && i < D && i >= j) Lout[(size_t)j * D + i] = col[i] / sqrt(pv);
        if (act && i > j) {
            const double ci = col[i] / pv;
#pragma unroll
            for (int q = 0; q < RC::EP; ++q) {
                const int k = c + q * RC::C;
                if (k > j && k <= i) {
                    a[q] -= ci * col[k];
                    if (k == j + 1) nxt[i] = a[q];
                }
            }
        }
        __syncthreads();
    }
    double lp = 0, bad = 0;
    for (int j = t; j < D; j += blockDim.x) {
        const double p = piv[j];
        bad += !(p > 0);
        lp += log(p > 0 ? p : 1.0);
    }
    const double ldp = block_sum(lp, red);
    return block_sum(bad, red) > 0 ? NAN : ldp;
}

// NIW posterior and log marginal likelihood (niw.cpp:23-49, 122-138; statistics (n, sum, S) plus the
// optional (sum2, S2) aggregated into them, niw.cpp:140-148) by one block of RegChol<DP>::T threads,
// D <= DP.  sh: RegChol<DP>::SMEM doubles of shared memory (mp[DP] at 2 DP).  The posterior scale psi'
// (upper triangle mirrored, as selfadjointView<Upper>) is built in registers and factored by
// reg_chol_logdet.  Lout (nullable) receives its lower Cholesky factor.  Valid in every thread.
// With allow_empty, an empty slot (n = 0) is factored too (its posterior is the prior; the
// parameter draw needs the factor) and its statistics are read as zero; otherwise it returns 0.
template <int DP>
__device__ double niw_lml_reg(int D, double n, const double* sum, const double* S, const double* sum2, const double* S2,
                              double k0, double v0, const double* m0, const double* psi0, double ld0, double* sh,
                              NiwExtras* ex = nullptr, double* Lout = nullptr, bool allow_empty = false)
{
    using RC = RegChol<DP>;
    if (n == 0 && !allow_empty) return 0.0;   // posterior == prior (niw.cpp:27-30): every term cancels
    const bool has = n > 0;
    double* mp = sh + 2 * DP;
    double* red = sh + 3 * DP;
    const int t = threadIdx.x;
    const int i = t % DP, c = t / DP;
    const bool act = c < RC::C && i < D;
    const double kp = k0 + n, vp = v0 + n;
    for (int d = t; d < D; d += blockDim.x)
        mp[d] = (m0[d] * k0 + (has ? (sum2 ? sum[d] + sum2[d] : sum[d]) : 0.0)) / kp;
    __syncthreads();
    double a[RC::EP];
    double h = 0, tr = 0;
#pragma unroll
    for (int q = 0; q < RC::EP; ++q) {
        const int k = c + q * RC::C;
        a[q] = 0.0;
        if (act && k <= i) {
            const size_t ki = (size_t)i * D + k;   // upper-triangle source: row k <= column i
            const double tm = v0 * psi0[ki] + k0 * m0[k] * m0[i];
            const double sv = has ? (S2 ? S[ki] + S2[ki] : S[ki]) : 0.0;
            a[q] = (tm - kp * mp[k] * mp[i] + sv) / vp;
            if (k == i) {
                h += log(a[q]);
                tr += a[q];
            }
        }
    }
    if (ex) {
        ex->hd = block_sum(h, red);
        ex->tr = block_sum(tr, red);
    }
    const double ld = reg_chol_logdet<DP>(a, D, sh, Lout);
    if (ex) ex->ld = ld;
    double g = 0.0;
    for (int d = 1 + t; d <= D; d += blockDim.x) g += lgamma(vp / 2.0 + (1 - d) / 2.0) - lgamma(v0 / 2.0 + (1 - d) / 2.0);
    g = block_sum(g, red);
    return -n * D * 0.5 * log(M_PI) + g + (v0 / 2.0) * (D * log(v0) + ld0) - (vp / 2.0) * (D * log(vp) + ld) +
           (D / 2.0) * (log(k0 / kp));
}

// merge log Hastings ratio of clusters i < j (shared_actions.cpp:88-99) with the register Cholesky
template <int DP>
__device__ double merge_log_hr_reg(const double* __restrict__ stats, int stat_len, int D, int gauss, double k0,
                                   double v0, double ld0, const double* __restrict__ prior,
                                   const double* __restrict__ lml, int i, int j, double alpha, double* sh)
{
    const double* si = stats + (size_t)(3 * i) * stat_len;
    const double* sj = stats + (size_t)(3 * j) * stat_len;
    const double ni = si[0], nj = sj[0];
    if (ni == 0 || nj == 0) return NAN;
    double lij;
    if (gauss)
        lij = niw_lml_reg<DP>(D, ni + nj, si + 1, si + 1 + D, sj + 1, sj + 1 + D, k0, v0, prior, prior + D, ld0, sh);
    else
        lij = mult_lml_block(D, ni + nj, si + 1, sj + 1, prior, sh + 3 * DP);
    const double n = ni + nj;
    return -log(alpha) + lgamma(alpha) - 2 * lgamma(0.5 * alpha) + lgamma(n) - lgamma(n + alpha) +
           lgamma(ni + 0.5 * alpha) - lgamma(ni) - lgamma(nj) + lgamma(nj + 0.5 * alpha) + lij - lml[3 * i] -
           lml[3 * j];
}

// Kernels templated on DP are launched through this: DPV is the padded dimension (4 ... 128), and
// `body` a statement using the constexpr DP.
#define DPMM_WITH_DP(DPV, body)                                   \
    switch (DPV) {                                                \
    case 4: { constexpr int DP = 4; body; } break;                \
    case 8: { constexpr int DP = 8; body; } break;                \
    case 16: { constexpr int DP = 16; body; } break;              \
    case 32: { constexpr int DP = 32; body; } break;              \
    case 64: { constexpr int DP = 64; body; } break;              \
    default: { constexpr int DP = 128; body; } break;             \
    }

// opt a kernel in to more than 48 KB of dynamic shared memory when it needs it
template <typename Kern>
static inline dpmm_status allow_smem(Kern k, size_t bytes)
{
    if (bytes > 48 * 1024) DPMM_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    return DPMM_OK;
}

// split log Hastings ratio of cluster k (local_clusters_actions.cpp:222-233) from the slot counts
// and the log marginal likelihoods of slots 3k, 3k+1, 3k+2; NaN when a sub-cluster is empty
static __device__ double split_log_hr_slot(const double* __restrict__ stats, int stat_len,
                                           const double* __restrict__ lml, int k, double alpha)
{
    const double n = stats[(size_t)(3 * k) * stat_len], nl = stats[(size_t)(3 * k + 1) * stat_len],
                 nr = stats[(size_t)(3 * k + 2) * stat_len];
    if (nl == 0 || nr == 0) return NAN;
    return log(alpha) + lgamma(nl) + lml[3 * k + 1] + lgamma(nr) + lml[3 * k + 2] - (lgamma(n) + lml[3 * k]);
}

}  // namespace dpmm

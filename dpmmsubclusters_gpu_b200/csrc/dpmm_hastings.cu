// dpmm_hastings.cu -- split / merge Metropolis-Hastings ratios of every cluster and every
// cluster pair, each in one launch, in FP64 on the device.
//
// Reference arithmetic restated (DPMMSubClusters/):
//   posterior            priors/niw.cpp:23-49, priors/multinomial_prior.cpp:12-22
//   log marginal lik.    priors/niw.cpp:122-138 (+ logdet.h:4-26 Cholesky branch,
//                        utils.cpp:94-102), priors/multinomial_prior.cpp:56-67
//   split ratio          local_clusters_actions.cpp:222-233
//   merge ratio          shared_actions.cpp:88-99
// lgamma is CUDA's lgamma(double).
#include <math.h>

#include "dpmm_internal.h"

namespace dpmm {

constexpr int kHThreads = 128;

__device__ double block_sum(double v, double* red)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double s = 0;
    if (threadIdx.x == 0) {
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) s += red[q];
        red[32] = s;
    }
    __syncthreads();
    return red[32];
}

// In-place Cholesky of the lower triangle of A (D x D, column-major, shared memory);
// returns log det A, or NaN when A is not positive definite.
__device__ double chol_logdet(double* A, int D, double* red)
{
    __shared__ int bad;
    if (threadIdx.x == 0) bad = 0;
    __syncthreads();
    for (int j = 0; j < D; ++j) {
        if (threadIdx.x == 0) {
            double a = A[(size_t)j * D + j];
            if (!(a > 0)) bad = 1;
            A[(size_t)j * D + j] = a > 0 ? sqrt(a) : 1.0;
        }
        __syncthreads();
        const double djj = A[(size_t)j * D + j];
        for (int i = j + 1 + threadIdx.x; i < D; i += blockDim.x) A[(size_t)j * D + i] /= djj;
        __syncthreads();
        // trailing update of the lower triangle: A(i,k) -= L(i,j) L(k,j), j < k <= i; one column
        // k per thread, walking its rows (no index division)
        const double* cj = A + (size_t)j * D;
        for (int kk = j + 1 + threadIdx.x; kk < D; kk += blockDim.x) {
            const double lkj = cj[kk];
            double* ck = A + (size_t)kk * D;
            for (int ii = kk; ii < D; ++ii) ck[ii] -= cj[ii] * lkj;
        }
        __syncthreads();
    }
    double v = 0;
    for (int j = threadIdx.x; j < D; j += blockDim.x) v += log(A[(size_t)j * D + j]);
    double s = block_sum(v, red);
    return bad ? NAN : 2 * s;
}

// NIW posterior (upper triangle mirrored into the lower, as selfadjointView<Upper>) of the
// statistics (n, sum, S) into shared memory: psi'[D*D], m'[D]; returns log marginal likelihood.
// (sum2, S2: optional second statistics aggregated into the first, niw.cpp:140-148)
__device__ double niw_lml_from_stats(int D, double n, const double* sum, const double* S, const double* sum2,
                                     const double* S2, double k0, double v0, const double* m0, const double* psi0,
                                     double ld0, double* psi, double* mp, double* red)
{
    if (n == 0) return 0.0;      // posterior == prior (niw.cpp:27-30): every term cancels
    const double kp = k0 + n, vp = v0 + n;
    for (int i = threadIdx.x; i < D; i += blockDim.x) mp[i] = (m0[i] * k0 + (sum2 ? sum[i] + sum2[i] : sum[i])) / kp;
    __syncthreads();
    for (int e = threadIdx.x; e < D * D; e += blockDim.x) {
        int j = e / D, i = e % D;            // column j, row i
        int a = i <= j ? i : j, b = i <= j ? j : i;   // upper-triangle source (a <= b)
        size_t ab = (size_t)b * D + a;
        double tm = v0 * psi0[ab] + k0 * m0[a] * m0[b];
        const double sab = S2 ? S[ab] + S2[ab] : S[ab];
        psi[(size_t)j * D + i] = (tm - kp * mp[a] * mp[b] + sab) / vp;
    }
    __syncthreads();
    const double ldp = chol_logdet(psi, D, red);
    const double logpi = log(M_PI);
    // log Gamma_D(vp / 2) - log Gamma_D(v0 / 2): the D(D-1)/4 log(pi) terms cancel; one lgamma
    // pair per thread, then a block sum
    double g = 0.0;
    for (int d = 1 + threadIdx.x; d <= D; d += blockDim.x) g += lgamma(vp / 2.0 + (1 - d) / 2.0) - lgamma(v0 / 2.0 + (1 - d) / 2.0);
    g = block_sum(g, red);
    return -n * D * 0.5 * logpi + g + (v0 / 2.0) * (D * log(v0) + ld0) - (vp / 2.0) * (D * log(vp) + ldp) +
           (D / 2.0) * (log(k0 / kp));
}

// Dirichlet-multinomial log marginal likelihood of statistics (n, sum)
__device__ double mult_lml_from_stats(int D, double n, const double* sum, const double* sum2, const double* alpha0,
                                      double* red)
{
    if (n == 0) return 0.0;
    double s0 = 0, sp = 0, acc = 0;
    for (int d = threadIdx.x; d < D; d += blockDim.x) {
        double a0 = alpha0[d], ap = a0 + (sum2 ? sum[d] + sum2[d] : sum[d]);
        s0 += a0;
        sp += ap;
        acc += lgamma(ap) - lgamma(a0);
    }
    s0 = block_sum(s0, red);
    sp = block_sum(sp, red);
    acc = block_sum(acc, red);
    return lgamma(s0) - lgamma(sp) + acc;
}

// one block per slot (3K): log marginal likelihood of each cluster / sub-cluster
__global__ void __launch_bounds__(kHThreads) k_slot_lml(const double* __restrict__ stats, int stat_len, int D, int gauss,
                                                        double k0, double v0, double ld0, const double* __restrict__ prior,
                                                        double* __restrict__ lml)
{
    extern __shared__ double sh[];
    // NIW: psi'[D*D], m'[D], reduction[33]; multinomial: reduction[33] only
    double* psi = sh;
    double* mp = gauss ? psi + (size_t)D * D : sh;
    double* red = gauss ? mp + D : sh;
    const double* st = stats + (size_t)blockIdx.x * stat_len;
    double v;
    if (gauss)
        v = niw_lml_from_stats(D, st[0], st + 1, st + 1 + D, nullptr, nullptr, k0, v0, prior, prior + D, ld0, psi, mp,
                               red);
    else
        v = mult_lml_from_stats(D, st[0], st + 1, nullptr, prior, red);
    if (threadIdx.x == 0) lml[blockIdx.x] = v;
}

__global__ void k_split_hr(const double* __restrict__ stats, int stat_len, const double* __restrict__ lml, int K,
                           double alpha, double* __restrict__ hr)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K) return;
    double n = stats[(size_t)(3 * k) * stat_len], nl = stats[(size_t)(3 * k + 1) * stat_len],
           nr = stats[(size_t)(3 * k + 2) * stat_len];
    if (nl == 0 || nr == 0) { hr[k] = NAN; return; }
    hr[k] = log(alpha) + lgamma(nl) + lml[3 * k + 1] + lgamma(nr) + lml[3 * k + 2] - (lgamma(n) + lml[3 * k]);
}

// one block per pair i < j: statistics aggregated (niw.cpp:140-148), posterior, lml, ratio
__global__ void __launch_bounds__(kHThreads) k_merge_hr(const double* __restrict__ stats, int stat_len, int D, int gauss,
                                                        double k0, double v0, double ld0, const double* __restrict__ prior,
                                                        const double* __restrict__ lml, int K, double alpha,
                                                        double* __restrict__ hr)
{
    extern __shared__ double sh[];
    double* psi = sh;
    double* mp = gauss ? psi + (size_t)D * D : sh;
    double* red = gauss ? mp + D : sh;
    // unrank pair b -> (i, j), i < j, row-major over the strict upper triangle
    long long b = blockIdx.x;
    int i = 0;
    long long rowlen = K - 1;
    while (b >= rowlen) { b -= rowlen; ++i; --rowlen; }
    const int j = i + 1 + (int)b;
    const double* si = stats + (size_t)(3 * i) * stat_len;
    const double* sj = stats + (size_t)(3 * j) * stat_len;
    const double ni = si[0], nj = sj[0];
    if (ni == 0 || nj == 0) {
        if (threadIdx.x == 0) hr[(size_t)i * K + j] = NAN;
        return;
    }
    double lij;
    if (gauss)
        lij = niw_lml_from_stats(D, ni + nj, si + 1, si + 1 + D, sj + 1, sj + 1 + D, k0, v0, prior, prior + D, ld0, psi,
                                 mp, red);
    else
        lij = mult_lml_from_stats(D, ni + nj, si + 1, sj + 1, prior, red);
    if (threadIdx.x != 0) return;
    const double n = ni + nj;
    hr[(size_t)i * K + j] = -log(alpha) + lgamma(alpha) - 2 * lgamma(0.5 * alpha) + lgamma(n) - lgamma(n + alpha) +
                            lgamma(ni + 0.5 * alpha) - lgamma(ni) - lgamma(nj) + lgamma(nj + 0.5 * alpha) + lij -
                            lml[3 * i] - lml[3 * j];
}

static size_t hastings_smem(const dpmm_ctx* c, bool merge)
{
    (void)merge;
    const size_t D = c->D;
    size_t s = c->prior == DPMM_PRIOR_GAUSSIAN ? D * D + D + 33 : 33;
    return s * sizeof(double);
}

dpmm_status launch_split_hastings(dpmm_ctx* c, int K, double alpha)
{
    if (!c->prior_set) return fail(DPMM_ERR_STATE, "prior hyper-parameters not set");
    DPMM_TRY(ensure_stats(c, K));
    const int gauss = c->prior == DPMM_PRIOR_GAUSSIAN;
    const double ld0 = c->prior_logdet;
    size_t sm = hastings_smem(c, false);
    if (sm > 48 * 1024) DPMM_CUDA_TRY(cudaFuncSetAttribute(k_slot_lml, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_slot_lml<<<3 * K, kHThreads, sm, c->stream>>>(c->d_stats, c->stat_len, c->D, gauss, c->prior_k, c->prior_v, ld0,
                                                    c->d_prior, c->d_lml);
    DPMM_LAUNCHED();
    k_split_hr<<<(K + 127) / 128, 128, 0, c->stream>>>(c->d_stats, c->stat_len, c->d_lml, K, alpha, c->d_split_hr);
    DPMM_LAUNCHED();
    return DPMM_OK;
}

dpmm_status launch_merge_hastings(dpmm_ctx* c, int K, double alpha)
{
    if (!c->prior_set) return fail(DPMM_ERR_STATE, "prior hyper-parameters not set");
    DPMM_TRY(ensure_stats(c, K));
    const int gauss = c->prior == DPMM_PRIOR_GAUSSIAN;
    const double ld0 = c->prior_logdet;
    // cluster-level lml of every cluster (slots 3k only are needed; all 3K are cheap)
    size_t sm = hastings_smem(c, false);
    if (sm > 48 * 1024) DPMM_CUDA_TRY(cudaFuncSetAttribute(k_slot_lml, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_slot_lml<<<3 * K, kHThreads, sm, c->stream>>>(c->d_stats, c->stat_len, c->D, gauss, c->prior_k, c->prior_v, ld0,
                                                    c->d_prior, c->d_lml);
    DPMM_LAUNCHED();
    DPMM_CUDA_TRY(cudaMemsetAsync(c->d_merge_hr, 0xff, sizeof(double) * (size_t)K * K, c->stream));   // NaN
    const long long pairs = (long long)K * (K - 1) / 2;
    if (pairs == 0) return DPMM_OK;
    size_t sm2 = hastings_smem(c, true);
    if (sm2 > 48 * 1024) DPMM_CUDA_TRY(cudaFuncSetAttribute(k_merge_hr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2));
    k_merge_hr<<<(unsigned)pairs, kHThreads, sm2, c->stream>>>(c->d_stats, c->stat_len, c->D, gauss, c->prior_k, c->prior_v,
                                                                ld0, c->d_prior, c->d_lml, K, alpha, c->d_merge_hr);
    DPMM_LAUNCHED();
    return DPMM_OK;
}

}  // namespace dpmm

// ============================================================================= allocation-free variant
// The all-pairs merge ratio for callers that cannot allocate device memory.  Its only scratch --
// the prior's log-determinant and each cluster's log marginal likelihood, written by the first
// two kernels and read by the pair kernel -- lives in the file-scope array below, sized for
// kStaticMaxClusters clusters.  Every device that loads this library holds the array until exit.
// All calls on a device share it: calls whose work overlaps on the GPU (different streams, or
// different host threads) race on it and must be serialised by the caller.
namespace dpmm {

constexpr int kStaticMaxClusters = 1024;
static __device__ __align__(256) double g_merge_scratch[1 + kStaticMaxClusters];

// scratch[0] = log det psi0 (NIW prior)
__global__ void __launch_bounds__(kHThreads) k_static_prior_logdet(const double* __restrict__ prior, int D,
                                                                    double* __restrict__ scratch)
{
    extern __shared__ double sh[];
    double* A = sh;                       // D*D
    double* red = A + (size_t)D * D;      // 33
    for (int e = threadIdx.x; e < D * D; e += blockDim.x) A[e] = prior[D + e];
    __syncthreads();
    const double ld = chol_logdet(A, D, red);
    if (threadIdx.x == 0) scratch[0] = ld;
}

// scratch[1 + k] = log marginal likelihood of cluster k (statistics slot 3k)
__global__ void __launch_bounds__(kHThreads) k_static_cluster_lml(const double* __restrict__ stats, int stat_len, int D,
                                                                   int gauss, double k0, double v0,
                                                                   const double* __restrict__ prior,
                                                                   double* __restrict__ scratch)
{
    extern __shared__ double sh[];
    double* psi = sh;
    double* mp = gauss ? psi + (size_t)D * D : sh;
    double* red = gauss ? mp + D : sh;
    const double* st = stats + (size_t)(3 * blockIdx.x) * stat_len;
    double v;
    if (gauss)
        v = niw_lml_from_stats(D, st[0], st + 1, st + 1 + D, nullptr, nullptr, k0, v0, prior, prior + D, scratch[0],
                               psi, mp, red);
    else
        v = mult_lml_from_stats(D, st[0], st + 1, nullptr, prior, red);
    if (threadIdx.x == 0) scratch[1 + blockIdx.x] = v;
}

// one block per pair i < j, as k_merge_hr, with the per-cluster terms read from the scratch
__global__ void __launch_bounds__(kHThreads) k_static_merge_hr(const double* __restrict__ stats, int stat_len, int D,
                                                                int gauss, double k0, double v0,
                                                                const double* __restrict__ prior,
                                                                const double* __restrict__ scratch, int K,
                                                                double alpha, double* __restrict__ hr)
{
    extern __shared__ double sh[];
    double* psi = sh;
    double* mp = gauss ? psi + (size_t)D * D : sh;
    double* red = gauss ? mp + D : sh;
    long long b = blockIdx.x;
    int i = 0;
    long long rowlen = K - 1;
    while (b >= rowlen) { b -= rowlen; ++i; --rowlen; }
    const int j = i + 1 + (int)b;
    const double* si = stats + (size_t)(3 * i) * stat_len;
    const double* sj = stats + (size_t)(3 * j) * stat_len;
    const double ni = si[0], nj = sj[0];
    if (ni == 0 || nj == 0) return;       // stays NaN
    double lij;
    if (gauss)
        lij = niw_lml_from_stats(D, ni + nj, si + 1, si + 1 + D, sj + 1, sj + 1 + D, k0, v0, prior, prior + D,
                                 scratch[0], psi, mp, red);
    else
        lij = mult_lml_from_stats(D, ni + nj, si + 1, sj + 1, prior, red);
    if (threadIdx.x != 0) return;
    const double n = ni + nj;
    hr[(size_t)i * K + j] = -log(alpha) + lgamma(alpha) - 2 * lgamma(0.5 * alpha) + lgamma(n) - lgamma(n + alpha) +
                            lgamma(ni + 0.5 * alpha) - lgamma(ni) - lgamma(nj) + lgamma(nj + 0.5 * alpha) + lij -
                            scratch[1 + i] - scratch[1 + j];
}

}  // namespace dpmm

#include <mutex>

// Device address of g_merge_scratch, looked up once per device (with that device current) on the
// first call made on it.
static double* static_scratch_for_current_device(dpmm_status* st)
{
    static std::mutex mu;
    static double* ptr[128] = {nullptr};
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 128) {
        *st = e != cudaSuccess ? dpmm::cuda_status(e, "cudaGetDevice") : dpmm::fail(DPMM_ERR_NO_DEVICE, "device ordinal");
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (!ptr[dev]) {
        double* p = nullptr;
        e = cudaGetSymbolAddress((void**)&p, dpmm::g_merge_scratch);
        if (e != cudaSuccess || !p) {
            *st = dpmm::cuda_status(e != cudaSuccess ? e : cudaErrorInvalidSymbol, "cudaGetSymbolAddress(g_merge_scratch)");
            return nullptr;
        }
        ptr[dev] = p;
    }
    *st = DPMM_OK;
    return ptr[dev];
}

extern "C" dpmm_status dpmm_merge_hastings_static(int32_t prior_type, int32_t D, int32_t K, double alpha, double k0,
                                                  double v0, const double* prior, const double* stats,
                                                  double* merge_log_hr, void* stream)
{
    using namespace dpmm;
    const bool gauss = prior_type == DPMM_PRIOR_GAUSSIAN;
    if (prior_type != DPMM_PRIOR_GAUSSIAN && prior_type != DPMM_PRIOR_MULTINOMIAL)
        return fail(DPMM_ERR_INVALID_ARG, "unknown prior_type");
    if (!prior || !stats || !merge_log_hr) return fail(DPMM_ERR_INVALID_ARG, "null device pointer");
    if (K < 1 || K > kStaticMaxClusters)
        return fail(DPMM_ERR_INVALID_ARG, "dpmm_merge_hastings_static: K must be in [1, " +
                                              std::to_string(kStaticMaxClusters) + "], got " + std::to_string(K));
    if (D < 1 || (gauss && D > kMaxGaussDim) || (!gauss && D > kMaxMultDim))
        return fail(DPMM_ERR_INVALID_ARG, "dpmm_merge_hastings_static: dimension out of range");
    if (!(alpha > 0)) return fail(DPMM_ERR_INVALID_ARG, "alpha must be positive");
    dpmm_status st;
    double* scratch = static_scratch_for_current_device(&st);
    if (!scratch) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int stat_len = gauss ? 1 + D + D * D : 1 + D;
    const size_t sm = sizeof(double) * (gauss ? (size_t)D * D + D + 33 : 33);
    if (sm > 48 * 1024) {
        DPMM_CUDA_TRY(cudaFuncSetAttribute(k_static_prior_logdet, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        DPMM_CUDA_TRY(cudaFuncSetAttribute(k_static_cluster_lml, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        DPMM_CUDA_TRY(cudaFuncSetAttribute(k_static_merge_hr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    }
    DPMM_CUDA_TRY(cudaMemsetAsync(merge_log_hr, 0xff, sizeof(double) * (size_t)K * K, s));   // NaN
    if (gauss) {
        k_static_prior_logdet<<<1, kHThreads, sm, s>>>(prior, D, scratch);
        DPMM_LAUNCHED();
    }
    k_static_cluster_lml<<<K, kHThreads, sm, s>>>(stats, stat_len, D, gauss ? 1 : 0, k0, v0, prior, scratch);
    DPMM_LAUNCHED();
    const long long pairs = (long long)K * (K - 1) / 2;
    if (pairs > 0) {
        k_static_merge_hr<<<(unsigned)pairs, kHThreads, sm, s>>>(stats, stat_len, D, gauss ? 1 : 0, k0, v0, prior,
                                                                 scratch, K, alpha, merge_log_hr);
        DPMM_LAUNCHED();
    }
    return DPMM_OK;
}

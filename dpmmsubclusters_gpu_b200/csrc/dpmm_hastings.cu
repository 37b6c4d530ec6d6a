// dpmm_hastings.cu -- split / merge Metropolis-Hastings ratios of every cluster and every
// cluster pair, each in one launch, in FP64 on the device.
//
// Reference arithmetic restated (DPMMSubClusters/):
//   posterior            priors/niw.cpp:23-49, priors/multinomial_prior.cpp:12-22
//   log marginal lik.    priors/niw.cpp:122-138 (+ logdet.h:4-26 Cholesky branch,
//                        utils.cpp:94-102), priors/multinomial_prior.cpp:56-67
//   split ratio          local_clusters_actions.cpp:222-233
//   merge ratio          shared_actions.cpp:88-99
// (the posterior / marginal-likelihood helpers are in dpmm_niw.cuh)
// lgamma is CUDA's lgamma(double).
#include <math.h>

#include "dpmm_internal.h"
#include "dpmm_niw.cuh"

namespace dpmm {

// one block per slot (3K): log marginal likelihood of each cluster / sub-cluster
// sel (nullable): clusters whose slots use the second prior (k1, v1, ld1, prior1), the outlier layout
template <int DP>
__global__ void __launch_bounds__(RegChol<DP>::T) k_slot_lml(const double* __restrict__ stats, int stat_len, int D,
                                                             int gauss, double k0, double v0, double ld0,
                                                             const double* __restrict__ prior, double k1, double v1,
                                                             double ld1, const double* __restrict__ prior1,
                                                             const uint8_t* __restrict__ sel, double* __restrict__ lml)
{
    __shared__ double sh[RegChol<DP>::SMEM];
    if (sel && sel[blockIdx.x / 3]) {
        k0 = k1;
        v0 = v1;
        ld0 = ld1;
        prior = prior1;
    }
    const double* st = stats + (size_t)blockIdx.x * stat_len;
    double v;
    if (gauss)
        v = niw_lml_reg<DP>(D, st[0], st + 1, st + 1 + D, nullptr, nullptr, k0, v0, prior, prior + D, ld0, sh);
    else
        v = mult_lml_block(D, st[0], st + 1, nullptr, prior, sh + 3 * DP);
    if (threadIdx.x == 0) lml[blockIdx.x] = v;
}

__global__ void k_split_hr(const double* __restrict__ stats, int stat_len, const double* __restrict__ lml, int K,
                           double alpha, double* __restrict__ hr)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K) return;
    hr[k] = split_log_hr_slot(stats, stat_len, lml, k, alpha);
}

// one block per pair i < j: statistics aggregated (niw.cpp:140-148), posterior, lml, ratio
// the merged cluster takes cluster i's prior (shared_actions.cpp:88-95): the second one where sel[i]
template <int DP>
__global__ void __launch_bounds__(RegChol<DP>::T) k_merge_hr(const double* __restrict__ stats, int stat_len, int D,
                                                             int gauss, double k0, double v0, double ld0,
                                                             const double* __restrict__ prior, double k1, double v1,
                                                             double ld1, const double* __restrict__ prior1,
                                                             const uint8_t* __restrict__ sel,
                                                             const double* __restrict__ lml, int K, double alpha,
                                                             double* __restrict__ hr)
{
    __shared__ double sh[RegChol<DP>::SMEM];
    // unrank pair b -> (i, j), i < j, row-major over the strict upper triangle
    long long b = blockIdx.x;
    int i = 0;
    long long rowlen = K - 1;
    while (b >= rowlen) { b -= rowlen; ++i; --rowlen; }
    const int j = i + 1 + (int)b;
    if (sel && sel[i]) {
        k0 = k1;
        v0 = v1;
        ld0 = ld1;
        prior = prior1;
    }
    const double v = merge_log_hr_reg<DP>(stats, stat_len, D, gauss, k0, v0, ld0, prior, lml, i, j, alpha, sh);
    if (threadIdx.x == 0) hr[(size_t)i * K + j] = v;
}

// padded dimension of the register Cholesky (the Dirichlet prior needs none: 4)
static int chol_dp(const dpmm_ctx* c) { return c->prior == DPMM_PRIOR_GAUSSIAN ? c->Dp : 4; }

static dpmm_status launch_slot_lml(dpmm_ctx* c, int K)
{
    const int gauss = c->prior == DPMM_PRIOR_GAUSSIAN;
    const bool out = c->outlier_layout != 0;
    DPMM_WITH_DP(chol_dp(c), (k_slot_lml<DP><<<3 * K, RegChol<DP>::T, 0, c->stream>>>(
                                 c->d_stats, c->stat_len, c->D, gauss, c->prior_k, c->prior_v, c->prior_logdet,
                                 c->d_prior, c->prior2_k, c->prior2_v, c->prior2_logdet,
                                 out ? c->d_prior2 : c->d_prior, out ? c->d_prior_sel : nullptr, c->d_lml)));
    DPMM_LAUNCHED();
    return DPMM_OK;
}

dpmm_status slot_lml_as_is(dpmm_ctx* c, int K, double* lml)
{
    if (!c->prior_set) return fail(DPMM_ERR_STATE, "prior hyper-parameters not set");
    DPMM_TRY(launch_slot_lml(c, K));
    DPMM_CUDA_TRY(cudaMemcpyAsync(lml, c->d_lml, sizeof(double) * 3 * K, cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    g_d2h_bytes.fetch_add(sizeof(double) * 3 * K, std::memory_order_relaxed);
    return DPMM_OK;
}

dpmm_status launch_split_hastings(dpmm_ctx* c, int K, double alpha)
{
    if (!c->prior_set) return fail(DPMM_ERR_STATE, "prior hyper-parameters not set");
    DPMM_TRY(ensure_stats(c, K));
    DPMM_TRY(launch_slot_lml(c, K));
    k_split_hr<<<(K + 127) / 128, 128, 0, c->stream>>>(c->d_stats, c->stat_len, c->d_lml, K, alpha, c->d_split_hr);
    DPMM_LAUNCHED();
    return DPMM_OK;
}

dpmm_status launch_merge_hastings(dpmm_ctx* c, int K, double alpha)
{
    if (!c->prior_set) return fail(DPMM_ERR_STATE, "prior hyper-parameters not set");
    DPMM_TRY(ensure_stats(c, K));
    // cluster-level lml of every cluster (slots 3k only are needed; all 3K are cheap)
    DPMM_TRY(launch_slot_lml(c, K));
    DPMM_CUDA_TRY(cudaMemsetAsync(c->d_merge_hr, 0xff, sizeof(double) * (size_t)K * K, c->stream));   // NaN
    const long long pairs = (long long)K * (K - 1) / 2;
    if (pairs == 0) return DPMM_OK;
    const int gauss = c->prior == DPMM_PRIOR_GAUSSIAN;
    const bool out = c->outlier_layout != 0;
    DPMM_WITH_DP(chol_dp(c), (k_merge_hr<DP><<<(unsigned)pairs, RegChol<DP>::T, 0, c->stream>>>(
                                 c->d_stats, c->stat_len, c->D, gauss, c->prior_k, c->prior_v, c->prior_logdet,
                                 c->d_prior, c->prior2_k, c->prior2_v, c->prior2_logdet, out ? c->d_prior2 : c->d_prior,
                                 out ? c->d_prior_sel : nullptr, c->d_lml, K, alpha, c->d_merge_hr)));
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
template <int DP>
__global__ void __launch_bounds__(RegChol<DP>::T) k_static_prior_logdet(const double* __restrict__ prior, int D,
                                                                         double* __restrict__ scratch)
{
    using RC = RegChol<DP>;
    __shared__ double sh[RC::SMEM];
    const int i = threadIdx.x % DP, c = threadIdx.x / DP;
    double a[RC::EP];
#pragma unroll
    for (int q = 0; q < RC::EP; ++q) {
        const int k = c + q * RC::C;
        a[q] = (c < RC::C && i < D && k <= i) ? prior[D + (size_t)i * D + k] : 0.0;   // psi0(k, i), k <= i
    }
    const double ld = reg_chol_logdet<DP>(a, D, sh, nullptr);
    if (threadIdx.x == 0) scratch[0] = ld;
}

// scratch[1 + k] = log marginal likelihood of cluster k (statistics slot 3k)
template <int DP>
__global__ void __launch_bounds__(RegChol<DP>::T) k_static_cluster_lml(const double* __restrict__ stats, int stat_len,
                                                                        int D, int gauss, double k0, double v0,
                                                                        const double* __restrict__ prior,
                                                                        double* __restrict__ scratch)
{
    __shared__ double sh[RegChol<DP>::SMEM];
    const double* st = stats + (size_t)(3 * blockIdx.x) * stat_len;
    double v;
    if (gauss)
        v = niw_lml_reg<DP>(D, st[0], st + 1, st + 1 + D, nullptr, nullptr, k0, v0, prior, prior + D, scratch[0], sh);
    else
        v = mult_lml_block(D, st[0], st + 1, nullptr, prior, sh + 3 * DP);
    if (threadIdx.x == 0) scratch[1 + blockIdx.x] = v;
}

// one block per pair i < j, as k_merge_hr, with the per-cluster terms read from the scratch
template <int DP>
__global__ void __launch_bounds__(RegChol<DP>::T) k_static_merge_hr(const double* __restrict__ stats, int stat_len,
                                                                     int D, int gauss, double k0, double v0,
                                                                     const double* __restrict__ prior,
                                                                     const double* __restrict__ scratch, int K,
                                                                     double alpha, double* __restrict__ hr)
{
    __shared__ double sh[RegChol<DP>::SMEM];
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
        lij = niw_lml_reg<DP>(D, ni + nj, si + 1, si + 1 + D, sj + 1, sj + 1 + D, k0, v0, prior, prior + D, scratch[0],
                              sh);
    else
        lij = mult_lml_block(D, ni + nj, si + 1, sj + 1, prior, sh + 3 * DP);
    if (threadIdx.x != 0) return;
    const double n = ni + nj;
    hr[(size_t)i * K + j] = -log(alpha) + lgamma(alpha) - 2 * lgamma(0.5 * alpha) + lgamma(n) - lgamma(n + alpha) +
                            lgamma(ni + 0.5 * alpha) - lgamma(ni) - lgamma(nj) + lgamma(nj + 0.5 * alpha) + lij -
                            scratch[1 + i] - scratch[1 + j];
}

}  // namespace dpmm

#include <cuda.h>   // CUcontext / CUresult types only: the two driver calls are fetched through the runtime

#include <mutex>

// Identity of the calling thread's current CUDA context: cuCtxGetId's process-unique id (0 when no
// context is current yet).  The driver functions come from cudaGetDriverEntryPoint, so the library
// does not link libcuda itself.
static dpmm_status current_context_id(unsigned long long* id)
{
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, nullptr) == cudaSuccess)
            get_current = (GetCurrent)f;
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, nullptr) == cudaSuccess) get_id = (GetId)f;
    });
    if (!get_current || !get_id) return dpmm::fail(DPMM_ERR_CUDA, "cuCtxGetCurrent / cuCtxGetId unavailable");
    CUcontext ctx = nullptr;
    *id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS) return dpmm::fail(DPMM_ERR_CUDA, "cuCtxGetCurrent failed");
    if (ctx && get_id(ctx, id) != CUDA_SUCCESS) return dpmm::fail(DPMM_ERR_CUDA, "cuCtxGetId failed");
    return DPMM_OK;
}

// Device address of g_merge_scratch in the calling thread's current context.  It is looked up (with
// that context current) on the first call made in a context and cached per device together with the
// context's id: when the context changes -- cudaDeviceReset, or a context the caller made current --
// the module is loaded anew there and the address is looked up again, so a stale address is never used.
static double* static_scratch_for_current_device(dpmm_status* st)
{
    static std::mutex mu;
    static double* ptr[128] = {nullptr};
    static unsigned long long ctx_of[128] = {0};
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 128) {
        *st = e != cudaSuccess ? dpmm::cuda_status(e, "cudaGetDevice") : dpmm::fail(DPMM_ERR_NO_DEVICE, "device ordinal");
        return nullptr;
    }
    unsigned long long id = 0;
    if ((*st = current_context_id(&id)) != DPMM_OK) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!ptr[dev] || id == 0 || id != ctx_of[dev]) {
        double* p = nullptr;
        e = cudaGetSymbolAddress((void**)&p, dpmm::g_merge_scratch);   // makes the device's context current
        if (e != cudaSuccess || !p) {
            *st = dpmm::cuda_status(e != cudaSuccess ? e : cudaErrorInvalidSymbol, "cudaGetSymbolAddress(g_merge_scratch)");
            return nullptr;
        }
        if (id == 0 && (*st = current_context_id(&id)) != DPMM_OK) return nullptr;
        ptr[dev] = p;
        ctx_of[dev] = id;
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
    const int dp = gauss ? padded_dim(D) : 4;
    DPMM_CUDA_TRY(cudaMemsetAsync(merge_log_hr, 0xff, sizeof(double) * (size_t)K * K, s));   // NaN
    if (gauss) {
        DPMM_WITH_DP(dp, (k_static_prior_logdet<DP><<<1, RegChol<DP>::T, 0, s>>>(prior, D, scratch)));
        DPMM_LAUNCHED();
    }
    DPMM_WITH_DP(dp, (k_static_cluster_lml<DP><<<K, RegChol<DP>::T, 0, s>>>(stats, stat_len, D, gauss ? 1 : 0, k0, v0,
                                                                            prior, scratch)));
    DPMM_LAUNCHED();
    const long long pairs = (long long)K * (K - 1) / 2;
    if (pairs > 0) {
        DPMM_WITH_DP(dp, (k_static_merge_hr<DP><<<(unsigned)pairs, RegChol<DP>::T, 0, s>>>(
                             stats, stat_len, D, gauss ? 1 : 0, k0, v0, prior, scratch, K, alpha, merge_log_hr)));
        DPMM_LAUNCHED();
    }
    return DPMM_OK;
}

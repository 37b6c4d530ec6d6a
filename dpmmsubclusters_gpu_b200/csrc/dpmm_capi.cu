// dpmm_capi.cu -- the device back-end half of the C ABI (include/dpmm_capi.h): context
// lifetime, point upload, parameter packing, and one entry point per method of the
// reference's cudaKernel class.  Kernels live in dpmm_kernels.cu / dpmm_hastings.cu /
// dpmm_tc.cu.
#include <cuda_runtime.h>
#include <curand_kernel.h>

#include <algorithm>
#include <unordered_map>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "dpmm_internal.h"
#include "linalg.h"

namespace dpmm {

static thread_local std::string g_last_error;
std::atomic<uint64_t> g_launches{0}, g_h2d_bytes{0}, g_d2h_bytes{0};

void set_error(const std::string& msg) { g_last_error = msg; }

dpmm_status fail(dpmm_status s, const std::string& msg)
{
    g_last_error = msg;
    return s;
}

dpmm_status cuda_status(cudaError_t e, const char* what)
{
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return DPMM_ERR_OOM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return DPMM_ERR_NO_DEVICE;
    return DPMM_ERR_CUDA;
}

int padded_dim(int d)
{
    int p = 4;
    while (p < d) p <<= 1;
    return p;
}

static int mult_padded_dim(int d) { return (d + 31) / 32 * 32; }

template <typename T>
static dpmm_status dev_alloc(T** p, size_t count)
{
    *p = nullptr;
    if (count == 0) return DPMM_OK;
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * count);
    if (e != cudaSuccess) {
        *p = nullptr;
        return cuda_status(e, "cudaMalloc");
    }
    return DPMM_OK;
}

// ----------------------------------------------------------------- point conversion kernels
// column sums of the sampled rows i0 + q * stride, q < ns: block b sums samples [b*R, (b+1)*R) for
// every column, then atomically adds (FP64)
template <typename T>
__global__ void k_col_sums(const T* __restrict__ x, int64_t i0, int64_t stride, int64_t ns, int D,
                           double* __restrict__ out)
{
    const int64_t R = 4096;
    const int64_t q0 = (int64_t)blockIdx.x * R;
    for (int d = threadIdx.x; d < D; d += blockDim.x) {
        double s = 0;
        for (int64_t q = q0; q < min(ns, q0 + R); ++q) s += (double)x[(i0 + q * stride) * D + d];
        atomicAdd(&out[d], s);
    }
}

template <typename T>
__global__ void k_convert_points(const T* __restrict__ x, int64_t N, int D, int Dp, const double* __restrict__ shift,
                                 float* __restrict__ out)
{
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= N * Dp) return;
    int64_t n = e / Dp;
    int d = (int)(e % Dp);
    float v = 0.f;
    if (d < D) v = (float)((double)x[n * D + d] - (shift ? shift[d] : 0.0));
    out[e] = v;
}

__global__ void k_count_nonfinite(const float* __restrict__ x, int64_t n, int32_t* __restrict__ bad)
{
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n && !isfinite(x[i])) atomicAdd(bad, 1);
}

// Contingency table of the labels 1..K against the dense ground-truth ids 0..G-1: table[k][g] =
// points with label k + 1 and ground truth g (labels outside 1..K are not counted).  Counts per block
// in shared memory when the table fits, else global atomics.
constexpr int kCtabSmem = 12288;
__global__ void __launch_bounds__(256) k_contingency(const int32_t* __restrict__ labels, const int32_t* __restrict__ gt,
                                                     int64_t N, int K, int G, unsigned long long* __restrict__ table)
{
    extern __shared__ unsigned int sct[];
    const int T = K * G;
    const bool local = T <= kCtabSmem;
    if (local)
        for (int e = threadIdx.x; e < T; e += blockDim.x) sct[e] = 0u;
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const int l = labels[i] - 1, g = gt[i];
        if (l < 0 || l >= K || g < 0 || g >= G) continue;
        if (local) atomicAdd(&sct[l * G + g], 1u);
        else atomicAdd(&table[(size_t)l * G + g], 1ull);
    }
    __syncthreads();
    if (local)
        for (int e = threadIdx.x; e < T; e += blockDim.x)
            if (sct[e]) atomicAdd(&table[e], (unsigned long long)sct[e]);
}

}  // namespace dpmm

using namespace dpmm;

// ----------------------------------------------------------------- status / version
extern "C" const char* dpmm_status_string(dpmm_status s)
{
    switch (s) {
        case DPMM_OK: return "ok";
        case DPMM_ERR_INVALID_ARG: return "invalid argument";
        case DPMM_ERR_OOM: return "out of memory";
        case DPMM_ERR_CUDA: return "CUDA error";
        case DPMM_ERR_NOT_PD: return "matrix not positive definite";
        case DPMM_ERR_TIMEOUT: return "device wait timed out";
        case DPMM_ERR_NUMERIC: return "non-finite value";
        case DPMM_ERR_STATE: return "call out of order";
        case DPMM_ERR_IO: return "I/O or parse error";
        case DPMM_ERR_NO_DEVICE: return "no CUDA device";
        case DPMM_ERR_EXCHANGE: return "shard exchange failed";
    }
    return "unknown status";
}

extern "C" const char* dpmm_last_error(void) { return g_last_error.c_str(); }

extern "C" int dpmm_capi_version(void) { return DPMM_CAPI_VERSION; }

extern "C" uint64_t dpmm_kernel_launch_count(void) { return g_launches.load(); }

extern "C" void dpmm_transfer_bytes(uint64_t* h2d, uint64_t* d2h)
{
    if (h2d) *h2d = g_h2d_bytes.load();
    if (d2h) *d2h = g_d2h_bytes.load();
}

extern "C" dpmm_status dpmm_phase_times(dpmm_ctx* c, int enable, double* ms, int64_t* calls)
{
    if (!c) return fail(DPMM_ERR_INVALID_ARG, "null context");
    for (int i = 0; i < PH_COUNT; ++i) {
        if (ms) ms[i] = c->phase_ms[i];
        if (calls) calls[i] = c->phase_calls[i];
    }
    if (enable >= 0) {
        c->timing = enable != 0;
        for (int i = 0; i < PH_COUNT; ++i) { c->phase_ms[i] = 0; c->phase_calls[i] = 0; }
    }
    return DPMM_OK;
}

// ----------------------------------------------------------------- lifetime
static void free_ctx(dpmm_ctx* c)
{
    if (!c) return;
    if (c->device >= 0) cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    void* bufs[] = {c->d_x, c->d_gshift, c->d_labels, c->d_sub, c->d_curand, c->d_Wt, c->d_b, c->d_c, c->d_lrw,
                    c->d_mu, c->d_perm, c->d_blk_hist, c->d_seg, c->d_chunk, c->d_nchunks, c->d_part, c->d_stats,
                    c->d_u, c->d_bits, c->d_remap, c->d_aux, c->d_r64, c->d_dbl_scratch, c->d_prior, c->d_lml,
                    c->d_split_hr, c->d_merge_hr, c->d_post_logdet, c->d_mask, c->d_Btc, c->d_Atc, c->d_rbuf,
                    c->d_rpart, c->d_Bsub, c->d_scr_rec, c->d_scr_vec, c->d_scr_linv, c->d_scr_feat,
                    c->d_scr_prox, c->d_scr_score, c->d_scr_w, c->d_scr_wdep, c->d_scr_elig, c->d_scr_sel,
                    c->d_scr_list, c->d_scr_slots, c->d_scr_hr, c->d_stats_tmp, c->d_logw, c->d_prune_rh,
                    c->d_prune_cand, c->d_prune_lam, c->d_prune_M, c->d_prune_cnt, c->d_prune_V,
                    c->d_prune_beta, c->d_prune_list, c->d_gt, c->d_ctab, c->d_xchg, c->d_Amult, c->d_Bmult,
                    c->d_prior2, c->d_prior_sel, c->d_cbase, c->d_linalg};
    for (void* p : bufs)
        if (p) cudaFree(p);
    if (c->h_pinned) cudaFreeHost(c->h_pinned);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->kev0) cudaEventDestroy(c->kev0);
    if (c->kev1) cudaEventDestroy(c->kev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

extern "C" dpmm_status dpmm_create(const dpmm_desc* desc, dpmm_ctx** out)
{
    if (!desc || !out) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    if (desc->n_points <= 0 || desc->n_points > (int64_t)INT32_MAX - 1) return fail(DPMM_ERR_INVALID_ARG, "n_points out of range");
    if (desc->dim <= 0) return fail(DPMM_ERR_INVALID_ARG, "dim must be positive");
    if (desc->prior_type != DPMM_PRIOR_GAUSSIAN && desc->prior_type != DPMM_PRIOR_MULTINOMIAL)
        return fail(DPMM_ERR_INVALID_ARG, "unknown prior_type");
    if (desc->prior_type == DPMM_PRIOR_GAUSSIAN && desc->dim > kMaxGaussDim)
        return fail(DPMM_ERR_INVALID_ARG, "Gaussian dimension above 128 is not supported");
    if (desc->prior_type == DPMM_PRIOR_MULTINOMIAL && desc->dim > kMaxMultDim)
        return fail(DPMM_ERR_INVALID_ARG, "multinomial dimension above 4096 is not supported");
    if (desc->rng_kind != DPMM_RNG_PHILOX && desc->rng_kind != DPMM_RNG_CURAND_XORWOW)
        return fail(DPMM_ERR_INVALID_ARG, "unknown rng_kind");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return fail(DPMM_ERR_NO_DEVICE, "no CUDA device available");
    if (desc->device < 0 || desc->device >= ndev) return fail(DPMM_ERR_INVALID_ARG, "device ordinal out of range");

    dpmm_ctx* c = new dpmm_ctx();
    c->device = desc->device;
    c->N = desc->n_points;
    c->n_total = desc->n_points;
    c->D = desc->dim;
    c->prior = desc->prior_type;
    c->Dp = c->prior == DPMM_PRIOR_GAUSSIAN ? padded_dim(c->D) : mult_padded_dim(c->D);
    c->k_max = desc->k_max > 0 ? desc->k_max : 256;
    c->rng_kind = desc->rng_kind;
    c->seed = desc->seed;
    c->ll_mode = desc->loglik_mode;
    c->verbose = desc->verbose;
    c->shift.assign(c->D, 0.0);
    dpmm_status st = DPMM_OK;
    auto chk = [&](dpmm_status s) {
        if (st == DPMM_OK) st = s;
    };
    if (cudaSetDevice(c->device) != cudaSuccess) {
        free_ctx(c);
        return fail(DPMM_ERR_NO_DEVICE, "cudaSetDevice failed");
    }
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        free_ctx(c);
        return fail(DPMM_ERR_CUDA, "cudaStreamCreate failed");
    }
    if (cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess ||
        c->num_sms <= 0)
        c->num_sms = 1;
    cudaEventCreate(&c->ev0);
    cudaEventCreate(&c->ev1);
    cudaEventCreate(&c->kev0);
    cudaEventCreate(&c->kev1);
    const int64_t N = c->N;
    const int Dp = c->Dp, KM = c->k_max;
    const bool gauss = c->prior == DPMM_PRIOR_GAUSSIAN;
    c->nblk_hist = (int)((N + 2047) / 2048);
    {
        // about four waves of two blocks per SM over N points, in whole units, at most kChunkMax
        const int64_t want = N / ((int64_t)c->num_sms * 2 * 4);
        const int64_t units = std::max<int64_t>(1, std::min<int64_t>(kChunkMax / kChunkUnit, (want + kChunkUnit - 1) / kChunkUnit));
        c->chunk_len = (int)(units * kChunkUnit);
    }
    c->max_chunks = (int)(N / c->chunk_len) + KM + 1;
    const int T = Dp * (Dp + 1) / 2;
    const int SL = gauss ? 1 + Dp + T : 1 + Dp;
    c->stat_len = gauss ? 1 + c->D + c->D * c->D : 1 + c->D;
    chk(dev_alloc(&c->d_x, (size_t)N * Dp));
    chk(dev_alloc(&c->d_gshift, (size_t)c->D));
    chk(dev_alloc(&c->d_labels, (size_t)N));
    chk(dev_alloc(&c->d_sub, (size_t)N));
    chk(dev_alloc(&c->d_perm, (size_t)N));
    chk(dev_alloc(&c->d_u, (size_t)2 * N));
    chk(dev_alloc(&c->d_bits, (size_t)N));
    chk(dev_alloc(&c->d_r64, (size_t)N));
    if (gauss) {
        chk(dev_alloc(&c->d_Wt, (size_t)3 * KM * Dp * Dp));
        chk(dev_alloc(&c->d_b, (size_t)3 * KM * Dp));
        if ((Dp == 32 || Dp == 64) && c->ll_mode != DPMM_LL_FP32) {
            chk(dev_alloc(&c->d_Btc, tc_param_bytes(KM)));
            chk(dev_alloc(&c->d_Atc, (size_t)((N + 127) / 128) * 32768));
            chk(dev_alloc(&c->d_rbuf, (size_t)N * KM));
            chk(dev_alloc(&c->d_rpart, (size_t)4 * N));
            chk(dev_alloc(&c->d_Bsub, (size_t)KM * 32768));
        }
    }
    if (!gauss && c->ll_mode != DPMM_LL_FP32 && c->D <= kMaxMultDim) {
        chk(dev_alloc(&c->d_Amult, mult_tc_a_bytes(N, c->D)));
        chk(dev_alloc(&c->d_Bmult, mult_tc_b_bytes(KM, c->D)));
        chk(dev_alloc(&c->d_rbuf, (size_t)N * KM));
        chk(dev_alloc(&c->d_rpart, (size_t)4 * N));
    }
    chk(dev_alloc(&c->d_c, (size_t)3 * KM));
    chk(dev_alloc(&c->d_lrw, (size_t)2 * KM));
    chk(dev_alloc(&c->d_mu, (size_t)3 * KM * Dp));
    chk(dev_alloc(&c->d_blk_hist, (size_t)c->nblk_hist * (KM + 1)));
    chk(dev_alloc(&c->d_seg, (size_t)KM + 2));
    chk(dev_alloc(&c->d_chunk, (size_t)3 * c->max_chunks));
    chk(dev_alloc(&c->d_nchunks, (size_t)1));
    chk(dev_alloc(&c->d_part, (size_t)c->max_chunks * 2 * SL));
    chk(dev_alloc(&c->d_stats, (size_t)3 * KM * c->stat_len));
    chk(dev_alloc(&c->d_stats_tmp, (size_t)3 * KM * c->stat_len));
    chk(dev_alloc(&c->d_logw, (size_t)KM));
    chk(dev_alloc(&c->d_remap, (size_t)KM + 2));
    chk(dev_alloc(&c->d_mask, (size_t)KM));
    c->stats_ok.assign(KM, 0);
    chk(dev_alloc(&c->d_aux, (size_t)KM + 16));
    chk(dev_alloc(&c->d_dbl_scratch, (size_t)std::max(2 + c->D + c->D * c->D, 4 * KM) + 64));
    chk(dev_alloc(&c->d_prior, (size_t)(gauss ? c->D + c->D * c->D : c->D)));
    chk(dev_alloc(&c->d_lml, (size_t)3 * KM));
    chk(dev_alloc(&c->d_split_hr, (size_t)KM));
    chk(dev_alloc(&c->d_merge_hr, (size_t)KM * KM));
    chk(dev_alloc(&c->d_post_logdet, (size_t)3 * KM));
    {
        const size_t rows = std::max<size_t>((size_t)KM, (size_t)KM * (KM - 1) / 2);
        chk(dev_alloc(&c->d_scr_rec, (size_t)3 * KM * kScrRec));
        chk(dev_alloc(&c->d_scr_vec, (size_t)3 * KM * 2 * c->D));
        if (gauss) chk(dev_alloc(&c->d_scr_linv, (size_t)KM * c->D * c->D));
        chk(dev_alloc(&c->d_scr_feat, rows * kScrF));
        chk(dev_alloc(&c->d_scr_prox, rows));
        chk(dev_alloc(&c->d_scr_score, rows));
        chk(dev_alloc(&c->d_scr_w, (size_t)kScrParams));
        chk(dev_alloc(&c->d_scr_wdep, (size_t)kScrParams));
        chk(dev_alloc(&c->d_scr_elig, (size_t)KM));
        chk(dev_alloc(&c->d_scr_sel, (size_t)kScrMaxTop + 1));
        chk(dev_alloc(&c->d_scr_list, (size_t)2 * kScrMaxTop));
        chk(dev_alloc(&c->d_scr_slots, (size_t)3 * kScrMaxTop));
        chk(dev_alloc(&c->d_scr_hr, (size_t)kScrMaxTop));
    }
    if (gauss && Dp <= 64) {
        chk(dev_alloc(&c->d_prune_rh, (size_t)N));
        chk(dev_alloc(&c->d_prune_cand, (size_t)c->max_chunks * 17));
        chk(dev_alloc(&c->d_prune_list, (size_t)c->max_chunks));
        const size_t KP = (size_t)std::min(KM, 256);   // the pruned phase takes K <= 256
        chk(dev_alloc(&c->d_prune_lam, KP));
        chk(dev_alloc(&c->d_prune_M, KP * KP));
        chk(dev_alloc(&c->d_prune_V, KP * KP * Dp));
        chk(dev_alloc(&c->d_prune_beta, KP * KP));
        chk(dev_alloc(&c->d_prune_cnt, (size_t)2));
    } else {
        c->prune_margin = 0.f;
    }
    if (c->rng_kind == DPMM_RNG_CURAND_XORWOW) chk(dev_alloc(&c->d_curand, (size_t)N));
    if (st == DPMM_OK) {
        c->h_pinned_bytes = std::max({sizeof(double) * 3 * KM * (size_t)c->stat_len, sizeof(double) * (size_t)KM * KM,
                                      sizeof(float) * 3 * KM * ((size_t)Dp * Dp + 2 * Dp + 2)});
        if (cudaMallocHost((void**)&c->h_pinned, c->h_pinned_bytes) != cudaSuccess) {
            c->h_pinned = nullptr;
            st = fail(DPMM_ERR_OOM, "cudaMallocHost failed");
        }
    }
    if (st == DPMM_OK) {
        cudaMemsetAsync(c->d_x, 0, sizeof(float) * (size_t)N * Dp, c->stream);
        cudaMemsetAsync(c->d_labels, 0, sizeof(int32_t) * N, c->stream);
        cudaMemsetAsync(c->d_sub, 0, sizeof(int32_t) * N, c->stream);
        cudaMemsetAsync(c->d_gshift, 0, sizeof(double) * c->D, c->stream);
        cudaMemsetAsync(c->d_mu, 0, sizeof(float) * 3 * KM * Dp, c->stream);
        if (gauss) {
            cudaMemsetAsync(c->d_Wt, 0, sizeof(float) * 3 * KM * (size_t)Dp * Dp, c->stream);
            cudaMemsetAsync(c->d_b, 0, sizeof(float) * 3 * KM * Dp, c->stream);
        }
        if (c->d_curand) st = launch_init_curand(c);
    }
    if (st == DPMM_OK) {
        cudaError_t e2 = cudaStreamSynchronize(c->stream);
        if (e2 != cudaSuccess) st = cuda_status(e2, "dpmm_create");
    }
    if (st != DPMM_OK) {
        std::string msg = g_last_error;
        free_ctx(c);
        g_last_error = msg;
        return st;
    }
    *out = c;
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_destroy(dpmm_ctx* ctx)
{
    free_ctx(ctx);
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_synchronize(dpmm_ctx* c)
{
    if (!c) return fail(DPMM_ERR_INVALID_ARG, "null context");
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return DPMM_OK;
}

// ----------------------------------------------------------------- points

// the shift keeps 20 significant bits of the mean: any value near the mean serves, and the rounding
// makes it the same whatever order the sums were added in (one context or shards)
static double round_shift(double m)
{
    int ex = 0;
    std::frexp(m, &ex);
    return m == 0.0 ? 0.0 : std::ldexp(std::nearbyint(std::ldexp(m, 20 - ex)), ex - 20);
}

// Points in pageable host memory.  The shift (Gaussian prior) is the mean of a strided sample: the
// points whose global index is a multiple of n_total / 65536, so the shards of one data set sample
// the same points as one context would.  Host threads then write the FP32 rows relative to it, padded
// to Dp, straight into two pinned staging buffers that the copy engine drains into d_x in turn: half
// the bytes of FP64 points cross PCIe, the host writes half as much, and no FP64 copy is made on the
// device.
constexpr int64_t kShiftSample = 65536;

template <typename T>
static dpmm_status upload_host_points_t(dpmm_ctx* c, const T* points)
{
    const int64_t N = c->N;
    const int D = c->D, Dp = c->Dp;
    const bool gauss = c->prior == DPMM_PRIOR_GAUSSIAN;
    if (gauss) {
        const int64_t stride = std::max<int64_t>(1, c->n_total / kShiftSample);
        const int64_t i0 = (stride - c->pt_offset % stride) % stride;
        std::vector<double> sums(D + 1, 0.0);
        const int64_t ns = i0 < N ? (N - 1 - i0) / stride + 1 : 0;
#pragma omp parallel
        {
            std::vector<double> part(D, 0.0);
#pragma omp for schedule(static) nowait
            for (int64_t q = 0; q < ns; ++q) {
                const T* row = points + (size_t)(i0 + q * stride) * D;
                for (int d = 0; d < D; ++d) part[d] += (double)row[d];
            }
#pragma omp critical
            for (int d = 0; d < D; ++d) sums[d] += part[d];
        }
        sums[D] = (double)ns;
        if (c->shard_world > 1) {   // the sample of the whole data set
            DPMM_CUDA_TRY(cudaMemcpy(c->d_xchg, sums.data(), sizeof(double) * (D + 1), cudaMemcpyHostToDevice));
            DPMM_TRY(shard_allreduce(c, c->d_xchg, D + 1));
            DPMM_CUDA_TRY(cudaMemcpy(sums.data(), c->d_xchg, sizeof(double) * (D + 1), cudaMemcpyDeviceToHost));
        }
        for (int d = 0; d < D; ++d) c->shift[d] = sums[D] > 0 ? round_shift(sums[d] / sums[D]) : 0.0;
        DPMM_CUDA_TRY(cudaMemcpy(c->d_gshift, c->shift.data(), sizeof(double) * D, cudaMemcpyHostToDevice));
    }
    const std::vector<double> shift = gauss ? c->shift : std::vector<double>(D, 0.0);
    constexpr size_t kChunkBytes = (size_t)64 << 20;
    // staging rows: 64 MB worth, or the whole data set when smaller (small data sets pin little)
    const int64_t rows = std::min<int64_t>(N, std::max<int64_t>(1, (int64_t)(kChunkBytes / (sizeof(float) * (size_t)Dp))));
    float* hb[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    cudaError_t e = cudaSuccess;
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
        e = cudaMallocHost(&hb[b], sizeof(float) * (size_t)rows * Dp);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming);
    }
    int64_t bad = 0;
    for (int64_t r0 = 0, i = 0; e == cudaSuccess && r0 < N; r0 += rows, ++i) {
        const int b = (int)(i & 1);
        const int64_t n = std::min(rows, N - r0);
        if (i >= 2) e = cudaEventSynchronize(ev[b]);   // its previous copy has left the buffer
        if (e != cudaSuccess) break;
        float* dst = hb[b];
        int64_t nb = 0;
#pragma omp parallel for schedule(static) reduction(+ : nb)
        for (int64_t r = 0; r < n; ++r) {
            const T* src = points + (size_t)(r0 + r) * D;
            float* out = dst + (size_t)r * Dp;
            for (int d = 0; d < D; ++d) {
                const float v = (float)((double)src[d] - shift[d]);
                nb += std::isfinite(v) ? 0 : 1;
                out[d] = v;
            }
            for (int d = D; d < Dp; ++d) out[d] = 0.f;
        }
        bad += nb;
        e = cudaMemcpyAsync(c->d_x + (size_t)r0 * Dp, dst, sizeof(float) * (size_t)n * Dp, cudaMemcpyHostToDevice,
                            c->stream);
        if (e == cudaSuccess) e = cudaEventRecord(ev[b], c->stream);
    }
    const cudaError_t es = cudaStreamSynchronize(c->stream);   // nothing reads the buffers after this
    if (e == cudaSuccess) e = es;
    for (int b = 0; b < 2; ++b) {
        if (ev[b]) cudaEventDestroy(ev[b]);
        if (hb[b]) cudaFreeHost(hb[b]);
    }
    if (e != cudaSuccess) return cuda_status(e, "dpmm_upload_points (host staging)");
    g_h2d_bytes += sizeof(float) * (size_t)N * Dp;
    if (bad) return fail(DPMM_ERR_NUMERIC, "points contain NaN or Inf");
    DPMM_TRY(pack_tc_points(c));
    DPMM_TRY(pack_mult_tc_points(c));
    c->points_ready = true;
    c->perm_K = -1;
    invalidate_stats(c);
    return DPMM_OK;
}

template <typename T>
static dpmm_status upload_points_t(dpmm_ctx* c, const T* points)
{
    if (!c || !points) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    DPMM_CUDA_TRY(cudaSetDevice(c->device));
    const int64_t N = c->N;
    const int D = c->D;
    // the points may live in pageable or pinned host memory or in device memory
    cudaPointerAttributes pa{};
    const bool attr_ok = cudaPointerGetAttributes(&pa, points) == cudaSuccess;
    cudaGetLastError();
    if (attr_ok && pa.type == cudaMemoryTypeUnregistered) return upload_host_points_t(c, points);
    T* tmp = nullptr;
    DPMM_TRY(dev_alloc(&tmp, (size_t)N * D));
    const size_t bytes = sizeof(T) * (size_t)N * D;
    cudaError_t e = cudaMemcpyAsync(tmp, points, bytes, cudaMemcpyDefault, c->stream);
    if (attr_ok && pa.type != cudaMemoryTypeDevice) g_h2d_bytes += bytes;
    const bool gauss = c->prior == DPMM_PRIOR_GAUSSIAN;
    if (e == cudaSuccess && gauss) {
        // FP64 column means (the shift)
        // the same strided sample as host points (upload_host_points_t)
        const int64_t stride = std::max<int64_t>(1, c->n_total / kShiftSample);
        const int64_t i0 = (stride - c->pt_offset % stride) % stride;
        const int64_t ns = i0 < N ? (N - 1 - i0) / stride + 1 : 0;
        cudaMemsetAsync(c->d_gshift, 0, sizeof(double) * D, c->stream);
        if (ns > 0)
            k_col_sums<T><<<(unsigned)((ns + 4095) / 4096), 128, 0, c->stream>>>(tmp, i0, stride, ns, D, c->d_gshift);
        e = cudaStreamSynchronize(c->stream);
        if (e == cudaSuccess) {
            std::vector<double> sums(D);
            e = cudaMemcpy(sums.data(), c->d_gshift, sizeof(double) * D, cudaMemcpyDeviceToHost);
            double n = (double)ns;
            if (e == cudaSuccess && c->shard_world > 1) {   // the sample of the whole data set
                sums.push_back(n);
                e = cudaMemcpy(c->d_xchg, sums.data(), sizeof(double) * (D + 1), cudaMemcpyHostToDevice);
                if (e == cudaSuccess) {
                    const dpmm_status xs = shard_allreduce(c, c->d_xchg, D + 1);
                    if (xs != DPMM_OK) {
                        cudaFree(tmp);
                        return xs;
                    }
                    e = cudaMemcpy(sums.data(), c->d_xchg, sizeof(double) * (D + 1), cudaMemcpyDeviceToHost);
                    n = sums[D];
                }
            }
            for (int d = 0; d < D; ++d) c->shift[d] = n > 0 ? round_shift(sums[d] / n) : 0.0;
            if (e == cudaSuccess)
                e = cudaMemcpy(c->d_gshift, c->shift.data(), sizeof(double) * D, cudaMemcpyHostToDevice);
        }
    }
    if (e == cudaSuccess) {
        const int64_t total = N * c->Dp;
        k_convert_points<T><<<(unsigned)((total + 255) / 256), 256, 0, c->stream>>>(
            tmp, N, D, c->Dp, gauss ? c->d_gshift : nullptr, c->d_x);
        cudaMemsetAsync(c->d_aux, 0, sizeof(int32_t), c->stream);
        k_count_nonfinite<<<(unsigned)((total + 255) / 256), 256, 0, c->stream>>>(c->d_x, total, c->d_aux);
        e = cudaStreamSynchronize(c->stream);
    }
    cudaFree(tmp);
    if (e != cudaSuccess) return cuda_status(e, "dpmm_upload_points");
    DPMM_TRY(pack_tc_points(c));
    DPMM_TRY(pack_mult_tc_points(c));
    int32_t bad = 0;
    DPMM_CUDA_TRY(cudaMemcpy(&bad, c->d_aux, sizeof(int32_t), cudaMemcpyDeviceToHost));
    if (bad) return fail(DPMM_ERR_NUMERIC, "points contain NaN or Inf");
    c->points_ready = true;
    c->perm_K = -1;
    invalidate_stats(c);
    return DPMM_OK;
}

namespace dpmm {
dpmm_status shard_allreduce(dpmm_ctx* c, double* d_buf, int64_t count)
{
    if (c->shard_world <= 1 || count <= 0) return DPMM_OK;
    const int rc = c->allreduce(c->allreduce_user, d_buf, count, (void*)c->stream);
    if (rc != 0) return fail(DPMM_ERR_EXCHANGE, "shard allreduce of " + std::to_string(count) +
                                                    " values failed (code " + std::to_string(rc) + ")");
    return DPMM_OK;
}
}  // namespace dpmm

extern "C" dpmm_status dpmm_set_wait_test(dpmm_ctx* c, int32_t stall)
{
    if (!c) return fail(DPMM_ERR_INVALID_ARG, "null context");
    c->stall_tc_mma = stall != 0;
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_set_fused_sub_stats(dpmm_ctx* c, int32_t on)
{
    if (!c) return fail(DPMM_ERR_INVALID_ARG, "null context");
    c->fuse_sub_stats = on != 0;
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_set_shard(dpmm_ctx* c, const dpmm_shard* sh)
{
    if (!c || !sh) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    if (c->points_ready) return fail(DPMM_ERR_STATE, "dpmm_set_shard must come before the points are uploaded");
    if (sh->world < 1 || sh->rank < 0 || sh->rank >= sh->world)
        return fail(DPMM_ERR_INVALID_ARG, "shard rank / world out of range");
    if (sh->world > 1 && !sh->allreduce) return fail(DPMM_ERR_INVALID_ARG, "a sharded context needs an allreduce");
    if (sh->point_offset < 0 || sh->n_total < c->N || sh->point_offset + c->N > sh->n_total)
        return fail(DPMM_ERR_INVALID_ARG, "shard point range outside [0, n_total)");
    DPMM_CUDA_TRY(cudaSetDevice(c->device));
    c->shard_world = sh->world;
    c->shard_rank = sh->rank;
    c->pt_offset = sh->point_offset;
    c->n_total = sh->n_total;
    c->allreduce = sh->allreduce;
    c->allreduce_user = sh->user;
    if (sh->world > 1 && !c->d_xchg) {
        c->xchg_len = std::max<size_t>((size_t)3 * c->k_max * c->stat_len, (size_t)c->D + 1);
        DPMM_TRY(dev_alloc(&c->d_xchg, c->xchg_len));
    }
    // the per-point XORWOW states are keyed by the global point index
    if (c->rng_kind == DPMM_RNG_CURAND_XORWOW && c->d_curand) {
        DPMM_TRY(launch_init_curand(c));
        DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    }
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_upload_points(dpmm_ctx* c, const double* points) { return upload_points_t(c, points); }
extern "C" dpmm_status dpmm_upload_points_f32(dpmm_ctx* c, const float* points) { return upload_points_t(c, points); }

// ----------------------------------------------------------------- labels
static dpmm_status stage_uniforms(dpmm_ctx* c, const float* u, int64_t n, const float** d_u)
{
    *d_u = nullptr;
    if (!u) return DPMM_OK;
    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_u, u, sizeof(float) * n, cudaMemcpyHostToDevice, c->stream));
    g_h2d_bytes += sizeof(float) * n;
    *d_u = c->d_u;
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_sample_labels(dpmm_ctx* c, int initial_clusters, double outlier_mod, const float* u)
{
    if (!c || initial_clusters < 1) return fail(DPMM_ERR_INVALID_ARG, "invalid argument");
    const float* du;
    DPMM_TRY(stage_uniforms(c, u, c->N, &du));
    DPMM_TRY(launch_labels_init(c, initial_clusters, outlier_mod, du));
    invalidate_stats(c);
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_draw_uniforms(dpmm_ctx* c, float* u)
{
    if (!c || !u) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    DPMM_TRY(launch_draw_uniforms(c, c->d_u));
    DPMM_CUDA_TRY(cudaMemcpyAsync(u, c->d_u, sizeof(float) * 2 * c->N, cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    g_d2h_bytes += sizeof(float) * 2 * c->N;
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_sample_sub_labels(dpmm_ctx* c, const float* u)
{
    if (!c) return fail(DPMM_ERR_INVALID_ARG, "null context");
    const float* du;
    DPMM_TRY(stage_uniforms(c, u, c->N, &du));
    DPMM_TRY(launch_sub_labels_init(c, du));
    invalidate_stats(c);
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_set_labels(dpmm_ctx* c, const int32_t* labels)
{
    if (!c || !labels) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_labels, labels, sizeof(int32_t) * c->N, cudaMemcpyHostToDevice, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->perm_K = -1;
    invalidate_stats(c);
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_set_sub_labels(dpmm_ctx* c, const int32_t* sub)
{
    if (!c || !sub) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_sub, sub, sizeof(int32_t) * c->N, cudaMemcpyHostToDevice, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    invalidate_stats(c);
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_get_labels(dpmm_ctx* c, int32_t* labels)
{
    if (!c || !labels) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    DPMM_CUDA_TRY(cudaMemcpyAsync(labels, c->d_labels, sizeof(int32_t) * c->N, cudaMemcpyDeviceToHost, c->stream));
    g_d2h_bytes += sizeof(int32_t) * c->N;
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_get_sub_labels(dpmm_ctx* c, int32_t* sub)
{
    if (!c || !sub) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    DPMM_CUDA_TRY(cudaMemcpyAsync(sub, c->d_sub, sizeof(int32_t) * c->N, cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_get_sub_labels_count(dpmm_ctx* c, int32_t* l, int32_t* r)
{
    if (!c || !l || !r) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    return launch_sub_count(c, l, r);
}

// ----------------------------------------------------------------- cluster parameters
// Pack one Gaussian slot: Wt[j][i] = W(i, j), b = W^T (mu - shift), c = -logdet/2 (+ log w), mu - shift.
static void pack_gauss_slot(dpmm_ctx* c, int slot, const double* mu, const std::vector<double>& W, double cval,
                            float* hWt, float* hb, float* hc, float* hmu)
{
    const int D = c->D, Dp = c->Dp;
    float* wt = hWt + (size_t)slot * Dp * Dp;
    std::fill(wt, wt + (size_t)Dp * Dp, 0.f);
    for (int j = 0; j < D; ++j)
        for (int i = 0; i < D; ++i) wt[(size_t)j * Dp + i] = (float)W[(size_t)j * D + i];
    for (int j = 0; j < Dp; ++j) {
        double s = 0;
        if (j < D)
            for (int i = 0; i < D; ++i) s += W[(size_t)j * D + i] * (mu[i] - c->shift[i]);
        hb[(size_t)slot * Dp + j] = (float)s;
        hmu[(size_t)slot * Dp + j] = j < D ? (float)(mu[j] - c->shift[j]) : 0.f;
    }
    hc[slot] = (float)cval;
}

static dpmm_status upload_gauss_params(dpmm_ctx* c, int K, const double* mu, const double* mat, bool is_factor,
                                       const double* logdet, const double* weights, const double* mu_lr,
                                       const double* mat_lr, const double* logdet_lr, const double* lr_weights)
{
    if (!c) return fail(DPMM_ERR_INVALID_ARG, "null context");
    if (c->prior != DPMM_PRIOR_GAUSSIAN) return fail(DPMM_ERR_STATE, "context is not Gaussian");
    if (K < 1 || K > c->k_max) return fail(DPMM_ERR_INVALID_ARG, "K out of range [1, k_max]");
    if (!mu || !mat || !logdet || !weights) return fail(DPMM_ERR_INVALID_ARG, "null cluster parameter");
    const int D = c->D, Dp = c->Dp;
    float* hWt = reinterpret_cast<float*>(c->h_pinned);
    float* hb = hWt + (size_t)3 * K * Dp * Dp;
    float* hc = hb + (size_t)3 * K * Dp;
    float* hmu = hc + 3 * K;
    std::vector<float> hlrw(2 * K, 0.f);
    std::vector<double> hcb(3 * (size_t)K, 0.0);   // -log det Sigma / 2 per slot (kept for the outlier layout)
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));   // the pinned stage may still be in flight
    // every slot is independent: pack them in parallel, keep the first error
    int err_slot = -1;
    dpmm_status err_status = DPMM_OK;
#pragma omp parallel
    {
        std::vector<double> W;
#pragma omp for schedule(dynamic, 4)
        for (int q = 0; q < 3 * K; ++q) {
            const int k = q / 3, s = q % 3;
            const bool sub = s > 0;
            if (sub && !mu_lr) {
                // no sub-cluster parameters: zero slots (sub-label phase then needs them set later)
                std::fill(hWt + (size_t)q * Dp * Dp, hWt + (size_t)(q + 1) * Dp * Dp, 0.f);
                std::fill(hb + (size_t)q * Dp, hb + (size_t)(q + 1) * Dp, 0.f);
                std::fill(hmu + (size_t)q * Dp, hmu + (size_t)(q + 1) * Dp, 0.f);
                hc[q] = 0.f;
                continue;
            }
            const int idx = sub ? 2 * k + (s - 1) : k;
            const double* m = sub ? mu_lr + (size_t)idx * D : mu + (size_t)k * D;
            const double* A = sub ? mat_lr + (size_t)idx * D * D : mat + (size_t)k * D * D;
            const double ld = sub ? logdet_lr[idx] : logdet[k];
            dpmm_status st = DPMM_OK;
            if (is_factor) {
                W.assign(A, A + (size_t)D * D);
            } else if (!la::cholesky(A, D, W)) {
                st = DPMM_ERR_NOT_PD;
            }
            double cval = -ld / 2;
            hcb[q] = cval;
            if (!sub) cval += std::log(weights[k]);
            if (st == DPMM_OK && !std::isfinite(cval) && !(cval < 0)) st = DPMM_ERR_NUMERIC;
            if (st != DPMM_OK) {
#pragma omp critical(dpmm_pack_err)
                if (err_slot < 0 || q < err_slot) { err_slot = q; err_status = st; }
                continue;
            }
            pack_gauss_slot(c, q, m, W, cval, hWt, hb, hc, hmu);
            if (sub) hlrw[idx] = lr_weights ? (float)std::log(lr_weights[idx]) : 0.f;
        }
    }
    if (err_slot >= 0) {
        const int k = err_slot / 3;
        const bool sub = err_slot % 3 != 0;
        if (err_status == DPMM_ERR_NOT_PD)
            return fail(DPMM_ERR_NOT_PD, "inv_sigma of cluster " + std::to_string(k) + (sub ? " (sub)" : "") +
                                             " is not positive definite");
        return fail(DPMM_ERR_NUMERIC, "non-finite log-likelihood constant");
    }
    // relocate packed arrays to their device buffers
    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_Wt, hWt, sizeof(float) * 3 * K * (size_t)Dp * Dp, cudaMemcpyHostToDevice, c->stream));
    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_b, hb, sizeof(float) * 3 * K * (size_t)Dp, cudaMemcpyHostToDevice, c->stream));
    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_c, hc, sizeof(float) * 3 * K, cudaMemcpyHostToDevice, c->stream));
    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_mu, hmu, sizeof(float) * 3 * K * (size_t)Dp, cudaMemcpyHostToDevice, c->stream));
    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_lrw, hlrw.data(), sizeof(float) * 2 * K, cudaMemcpyHostToDevice, c->stream));
    if (c->d_cbase)
        DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_cbase, hcb.data(), sizeof(double) * 3 * K, cudaMemcpyHostToDevice, c->stream));
    g_h2d_bytes += sizeof(float) * 3 * (size_t)K * ((size_t)Dp * Dp + 2 * Dp + 1) + sizeof(float) * 2 * K;
    {
        PhaseTimer pt(c, PH_PARAMS);
        DPMM_TRY(pack_tc_params(c, K));
    }
    c->K_params = K;
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_set_gaussian_params(dpmm_ctx* c, int K, const double* mu, const double* inv_sigma,
                                                const double* logdet_sigma, const double* weights, const double* mu_lr,
                                                const double* inv_sigma_lr, const double* logdet_sigma_lr,
                                                const double* lr_weights)
{
    return upload_gauss_params(c, K, mu, inv_sigma, false, logdet_sigma, weights, mu_lr, inv_sigma_lr, logdet_sigma_lr,
                               lr_weights);
}

extern "C" dpmm_status dpmm_set_gaussian_factors(dpmm_ctx* c, int K, const double* mu, const double* w,
                                                 const double* logdet_sigma, const double* weights, const double* mu_lr,
                                                 const double* w_lr, const double* logdet_sigma_lr,
                                                 const double* lr_weights)
{
    return upload_gauss_params(c, K, mu, w, true, logdet_sigma, weights, mu_lr, w_lr, logdet_sigma_lr, lr_weights);
}

extern "C" dpmm_status dpmm_set_multinomial_params(dpmm_ctx* c, int K, const double* log_theta, const double* weights,
                                                   const double* log_theta_lr, const double* lr_weights)
{
    (void)weights;
    if (!c) return fail(DPMM_ERR_INVALID_ARG, "null context");
    if (c->prior != DPMM_PRIOR_MULTINOMIAL) return fail(DPMM_ERR_STATE, "context is not multinomial");
    if (K < 1 || K > c->k_max) return fail(DPMM_ERR_INVALID_ARG, "K out of range [1, k_max]");
    if (!log_theta) return fail(DPMM_ERR_INVALID_ARG, "null log_theta");
    const int D = c->D, Dp = c->Dp;
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    float* hmu = reinterpret_cast<float*>(c->h_pinned);
    float* hc = hmu + (size_t)3 * K * Dp;
    std::vector<float> hlrw(2 * K, 0.f);
    for (int k = 0; k < K; ++k)
        for (int s = 0; s < 3; ++s) {
            const double* src = s == 0 ? log_theta + (size_t)k * D
                                       : (log_theta_lr ? log_theta_lr + (size_t)(2 * k + s - 1) * D : nullptr);
            float* dst = hmu + (size_t)(3 * k + s) * Dp;
            for (int d = 0; d < Dp; ++d) dst[d] = (src && d < D) ? (float)src[d] : 0.f;
            hc[3 * k + s] = 0.f;
            if (s > 0) hlrw[2 * k + s - 1] = lr_weights ? (float)std::log(lr_weights[2 * k + s - 1]) : 0.f;
        }
    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_mu, hmu, sizeof(float) * 3 * K * (size_t)Dp, cudaMemcpyHostToDevice, c->stream));
    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_c, hc, sizeof(float) * 3 * K, cudaMemcpyHostToDevice, c->stream));
    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_lrw, hlrw.data(), sizeof(float) * 2 * K, cudaMemcpyHostToDevice, c->stream));
    c->K_params = K;
    c->mult_tc_K = -1;
    return DPMM_OK;
}

// ----------------------------------------------------------------- phases
static dpmm_status check_ready(dpmm_ctx* c, int K)
{
    if (!c) return fail(DPMM_ERR_INVALID_ARG, "null context");
    if (!c->points_ready) return fail(DPMM_ERR_STATE, "points not uploaded");
    if (K < 1 || K > c->k_max) return fail(DPMM_ERR_INVALID_ARG, "K out of range [1, k_max]");
    if (K > c->K_params) return fail(DPMM_ERR_STATE, "cluster parameters not set for K clusters");
    return DPMM_OK;
}

namespace dpmm {
// The label phase of one context as a job of a batched launch (launch_labels_batched): the same
// checks and random stream as dpmm_create_clusters_labels with device uniforms, SIMT FP32 form.
dpmm_status make_label_job(dpmm_ctx* c, int K, int final_, LabelJob* job)
{
    DPMM_TRY(check_ready(c, K));
    if (c->prior != DPMM_PRIOR_GAUSSIAN) return fail(DPMM_ERR_INVALID_ARG, "batched label phase: NIW prior only");
    job->x = c->d_x;
    job->N = c->N;
    job->Wt = c->d_Wt;
    job->b = c->d_b;
    job->c = c->d_c;
    job->K = K;
    job->final_ = final_;
    job->rng = rng_args(c, nullptr);
    job->labels = c->d_labels;
    c->perm_K = -1;
    invalidate_stats(c);
    return DPMM_OK;
}
}  // namespace dpmm

extern "C" dpmm_status dpmm_create_clusters_labels(dpmm_ctx* c, int K, int final_, const float* u, float* loglik_out)
{
    DPMM_TRY(check_ready(c, K));
    const float* du = nullptr;
    if (!final_) DPMM_TRY(stage_uniforms(c, u, 2 * c->N, &du));
    float* d_rout = nullptr;
    if (loglik_out) DPMM_TRY(dev_alloc(&d_rout, (size_t)c->N * K));
    dpmm_status s;
    const bool mult_tc = c->prior == DPMM_PRIOR_MULTINOMIAL && tc_mult_supported(c, K);
    const bool use_tc = c->ll_mode != DPMM_LL_FP32 && (tc_supported(c, K) || mult_tc);
    PhaseTimer pt(c, PH_LABELS);
    bool pruned = false;
    s = DPMM_OK;
    if (!d_rout) s = launch_cluster_labels_pruned(c, K, final_, du, &pruned);
    if (s != DPMM_OK || pruned) {
    } else if (c->ll_mode == DPMM_LL_TC_BF16X3 && !use_tc) {
        s = fail(DPMM_ERR_INVALID_ARG, "tensor-core log-likelihood not available for this shape");
    } else {
        s = mult_tc  ? launch_mult_labels_tc(c, K, final_, du, d_rout)
            : use_tc ? launch_cluster_labels_tc(c, K, final_, du, d_rout)
                     : launch_cluster_labels(c, K, final_, du, d_rout);
    }
    if (s == DPMM_OK && d_rout) {
        cudaError_t e = cudaMemcpyAsync(loglik_out, d_rout, sizeof(float) * (size_t)c->N * K, cudaMemcpyDeviceToHost,
                                        c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) s = cuda_status(e, "loglik_out copy");
    }
    if (d_rout) cudaFree(d_rout);
    if (s == DPMM_OK && u) {
        cudaError_t e = cudaStreamSynchronize(c->stream);   // caller's uniforms staged: keep order simple
        if (e != cudaSuccess) s = cuda_status(e, "dpmm_create_clusters_labels");
    }
    c->perm_K = -1;
    invalidate_stats(c);
    return s;
}

extern "C" dpmm_status dpmm_create_subclusters_labels(dpmm_ctx* c, int K, const float* u, float* loglik_out)
{
    DPMM_TRY(check_ready(c, K));
    const float* du = nullptr;
    DPMM_TRY(stage_uniforms(c, u, 2 * c->N, &du));
    float* d_rout = nullptr;
    if (loglik_out) DPMM_TRY(dev_alloc(&d_rout, (size_t)c->N * 2));
    dpmm_status s;
    {
        PhaseTimer pt(c, PH_SUB_STATS);
        s = launch_sub_labels_and_stats(c, K, du, d_rout, true);
    }
    if (s == DPMM_OK && d_rout) {
        cudaError_t e = cudaMemcpyAsync(loglik_out, d_rout, sizeof(float) * (size_t)c->N * 2, cudaMemcpyDeviceToHost,
                                        c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) s = cuda_status(e, "loglik_out copy");
    }
    if (d_rout) cudaFree(d_rout);
    return s;
}

extern "C" dpmm_status dpmm_create_sufficient_statistics(dpmm_ctx* c, int n, const int32_t* indices, int64_t* count,
                                                         double* sum, double* S)
{
    if (!c) return fail(DPMM_ERR_INVALID_ARG, "null context");
    if (!c->points_ready) return fail(DPMM_ERR_STATE, "points not uploaded");
    if (n < 0 || (n > 0 && !indices)) return fail(DPMM_ERR_INVALID_ARG, "bad index list");
    int K = 0;
    for (int i = 0; i < n; ++i) {
        if (indices[i] < 0 || indices[i] >= c->k_max) return fail(DPMM_ERR_INVALID_ARG, "cluster index out of range");
        K = std::max(K, indices[i] + 1);
    }
    if (n == 0) return DPMM_OK;
    // statistics are (re)computed for every current cluster, so that the Hastings launches
    // that follow see all of them; each cluster's accumulation is shifted by its mean parameter
    const int Keff = std::min(c->k_max, std::max(K, c->K_params));
    DPMM_TRY(ensure_stats(c, Keff));
    g_d2h_bytes += sizeof(double) * 3 * (size_t)K * c->stat_len;
    const int L = c->stat_len, D = c->D;
    double* h = c->h_pinned;
    DPMM_CUDA_TRY(cudaMemcpyAsync(h, c->d_stats, sizeof(double) * 3 * (size_t)K * L, cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    for (int q = 0; q < n; ++q) {
        const int k = indices[q];
        for (int s = 0; s < 3; ++s) {
            const double* src = h + (size_t)(3 * k + s) * L;
            if (count) count[3 * q + s] = (int64_t)llround(src[0]);
            if (sum) std::memcpy(sum + (size_t)(3 * q + s) * D, src + 1, sizeof(double) * D);
            if (S && c->prior == DPMM_PRIOR_GAUSSIAN)
                std::memcpy(S + (size_t)(3 * q + s) * D * D, src + 1 + D, sizeof(double) * D * D);
        }
    }
    return DPMM_OK;
}

// ----------------------------------------------------------------- label maintenance
static bool has_repeats(int n, const int32_t* a, const int32_t* b)
{
    std::vector<int32_t> v;
    for (int i = 0; i < n; ++i) {
        v.push_back(a[i]);
        if (b) v.push_back(b[i]);
    }
    std::sort(v.begin(), v.end());
    return std::adjacent_find(v.begin(), v.end()) != v.end();
}

static dpmm_status stage_bits(dpmm_ctx* c, const uint32_t* bits, const uint32_t** d_bits)
{
    *d_bits = nullptr;
    if (!bits) return DPMM_OK;
    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_bits, bits, sizeof(uint32_t) * c->N, cudaMemcpyHostToDevice, c->stream));
    *d_bits = c->d_bits;
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_split_clusters(dpmm_ctx* c, int n, const int32_t* index, const int32_t* new_index,
                                           const uint32_t* bits)
{
    if (!c || n < 0 || (n > 0 && (!index || !new_index))) return fail(DPMM_ERR_INVALID_ARG, "bad split list");
    const int tlen = c->k_max + 2;
    for (int i = 0; i < n; ++i)
        if (index[i] < 0 || new_index[i] < 0 || index[i] + 1 >= tlen || new_index[i] + 1 >= tlen)
            return fail(DPMM_ERR_INVALID_ARG, "split index out of range");
    const uint32_t* db;
    DPMM_TRY(stage_bits(c, bits, &db));
    const bool seq = has_repeats(n, index, new_index);
    std::vector<int32_t> table(tlen, 0);
    for (int i = 0; i < n; ++i) {
        if (seq) std::fill(table.begin(), table.end(), 0);
        table[index[i] + 1] = new_index[i] + 1;
        if (seq || i == n - 1) DPMM_TRY(launch_relabel(c, 0, 0, table.data(), tlen, db));
    }
    for (int i = 0; i < n; ++i) {
        invalidate_stats(c, index[i]);
        invalidate_stats(c, new_index[i]);
    }
    if (c->outlier_layout) {
        // create_splittable_from_params (local_clusters_actions.cpp:264-285): the new cluster starts
        // from the parent's r sub-cluster parameters.  Drawn at the next iteration like every cluster,
        // except when it is renumbered to index 1 before that, which is never redrawn (:348-351).
        for (int i = 0; i < n; ++i) {
            if (index[i] >= c->K_params) continue;
            const size_t src = 3 * (size_t)index[i] + 2;
            for (int s = 0; s < 3; ++s) {
                const size_t dst = 3 * (size_t)new_index[i] + s;
                if (c->prior == DPMM_PRIOR_GAUSSIAN) {
                    const size_t m = (size_t)c->Dp * c->Dp;
                    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_Wt + dst * m, c->d_Wt + src * m, sizeof(float) * m,
                                                  cudaMemcpyDeviceToDevice, c->stream));
                    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_b + dst * c->Dp, c->d_b + src * c->Dp, sizeof(float) * c->Dp,
                                                  cudaMemcpyDeviceToDevice, c->stream));
                    if (c->d_cbase)
                        DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_cbase + dst, c->d_cbase + src, sizeof(double),
                                                      cudaMemcpyDeviceToDevice, c->stream));
                }
                DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_mu + dst * c->Dp, c->d_mu + src * c->Dp, sizeof(float) * c->Dp,
                                              cudaMemcpyDeviceToDevice, c->stream));
                DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_c + dst, c->d_c + src, sizeof(float), cudaMemcpyDeviceToDevice,
                                              c->stream));
            }
        }
    }
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_merge_clusters(dpmm_ctx* c, int n, const int32_t* index, const int32_t* new_index)
{
    if (!c || n < 0 || (n > 0 && (!index || !new_index))) return fail(DPMM_ERR_INVALID_ARG, "bad merge list");
    const int tlen = c->k_max + 2;
    for (int i = 0; i < n; ++i)
        if (index[i] < 0 || new_index[i] < 0 || index[i] + 1 >= tlen || new_index[i] + 1 >= tlen)
            return fail(DPMM_ERR_INVALID_ARG, "merge index out of range");
    const bool seq = has_repeats(n, index, new_index);
    std::vector<int32_t> table(tlen, 0);
    for (int i = 0; i < n; ++i) {
        if (seq) std::fill(table.begin(), table.end(), 0);
        table[index[i] + 1] = 1;
        table[new_index[i] + 1] = -(index[i] + 1);
        if (seq || i == n - 1) DPMM_TRY(launch_relabel(c, 1, 0, table.data(), tlen, nullptr));
    }
    for (int i = 0; i < n; ++i) {
        invalidate_stats(c, index[i]);
        invalidate_stats(c, new_index[i]);
    }
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_reset_bad_clusters(dpmm_ctx* c, int n, const int32_t* index, const uint32_t* bits)
{
    if (!c || n < 0 || (n > 0 && !index)) return fail(DPMM_ERR_INVALID_ARG, "bad reset list");
    if (n == 0) return DPMM_OK;
    const int tlen = c->k_max + 2;
    std::vector<int32_t> table(tlen, 0);
    for (int i = 0; i < n; ++i) {
        if (index[i] < 0 || index[i] + 1 >= tlen) return fail(DPMM_ERR_INVALID_ARG, "reset index out of range");
        table[index[i] + 1] = 1;
    }
    const uint32_t* db;
    DPMM_TRY(stage_bits(c, bits, &db));
    if (has_repeats(n, index, nullptr)) {
        // a repeated index re-randomises the same points again (one draw per listing)
        for (int i = 0; i < n; ++i) {
            std::fill(table.begin(), table.end(), 0);
            table[index[i] + 1] = 1;
            DPMM_TRY(launch_relabel(c, 2, 0, table.data(), tlen, db));
        }
    } else {
        DPMM_TRY(launch_relabel(c, 2, 0, table.data(), tlen, db));
    }
    for (int i = 0; i < n; ++i) invalidate_stats(c, index[i]);
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_remove_empty_clusters(dpmm_ctx* c, int n, const int32_t* limits)
{
    if (!c || n < 0 || (n > 0 && !limits)) return fail(DPMM_ERR_INVALID_ARG, "bad limit list");
    if (n == 0) return DPMM_OK;
    const int tlen = c->k_max + 2;
    std::vector<int32_t> table(tlen);
    for (int v = 0; v < tlen; ++v) {
        int x = v;
        for (int i = 0; i < n; ++i)
            if (x > limits[i]) x -= 1;
        table[v] = x;
    }
    DPMM_TRY(launch_relabel(c, 3, 0, table.data(), tlen, nullptr));
    invalidate_stats(c);
    return DPMM_OK;
}

// ----------------------------------------------------------------- test seams
extern "C" dpmm_status dpmm_log_likelihood_labels_gaussian(dpmm_ctx* c, const double* mu, const double* inv_sigma,
                                                           double logdet_sigma, double weight, double* r_out)
{
    if (!c || !mu || !inv_sigma || !r_out) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    if (c->prior != DPMM_PRIOR_GAUSSIAN) return fail(DPMM_ERR_STATE, "context is not Gaussian");
    if (!c->points_ready) return fail(DPMM_ERR_STATE, "points not uploaded");
    const int D = c->D;
    std::vector<double> prm((size_t)D + D * D + 2);
    std::memcpy(prm.data(), mu, sizeof(double) * D);
    std::memcpy(prm.data() + D, inv_sigma, sizeof(double) * D * D);
    prm[D + D * D] = -(((double)D * D * std::log(2 * M_PI) + logdet_sigma) / 2);   // sigma.size() == D*D
    prm[D + D * D + 1] = std::log(weight);
    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_dbl_scratch, prm.data(), sizeof(double) * prm.size(), cudaMemcpyHostToDevice,
                                  c->stream));
    DPMM_TRY(launch_loglik_gauss_one(c, c->d_r64));
    DPMM_CUDA_TRY(cudaMemcpyAsync(r_out, c->d_r64, sizeof(double) * c->N, cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_log_likelihood_labels_multinomial(dpmm_ctx* c, const double* log_theta, double* r_out)
{
    if (!c || !log_theta || !r_out) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    if (!c->points_ready) return fail(DPMM_ERR_STATE, "points not uploaded");
    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_dbl_scratch, log_theta, sizeof(double) * c->D, cudaMemcpyHostToDevice, c->stream));
    DPMM_TRY(launch_loglik_mult_one(c, c->d_r64));
    DPMM_CUDA_TRY(cudaMemcpyAsync(r_out, c->d_r64, sizeof(double) * c->N, cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_sample_log_cat_array(dpmm_ctx* c, int K, const double* loglik, const float* u)
{
    if (!c || !loglik || K < 1) return fail(DPMM_ERR_INVALID_ARG, "invalid argument");
    double* d_r = nullptr;
    DPMM_TRY(dev_alloc(&d_r, (size_t)c->N * K));
    const float* du;
    dpmm_status s = stage_uniforms(c, u, 2 * c->N, &du);
    cudaError_t e = cudaMemcpyAsync(d_r, loglik, sizeof(double) * c->N * K, cudaMemcpyHostToDevice, c->stream);
    if (s == DPMM_OK && e != cudaSuccess) s = cuda_status(e, "copy");
    if (s == DPMM_OK) s = launch_sample_log_cat(c, K, d_r, du);
    if (s == DPMM_OK) {
        e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) s = cuda_status(e, "dpmm_sample_log_cat_array");
    }
    cudaFree(d_r);
    c->perm_K = -1;
    invalidate_stats(c);
    return s;
}

extern "C" dpmm_status dpmm_sample_log_cat_array_sub_cluster(dpmm_ctx* c, int m, const double* loglik,
                                                             const int32_t* indices, const double* lr_weights,
                                                             const float* u)
{
    if (!c || m < 0 || (m > 0 && (!loglik || !indices || !lr_weights))) return fail(DPMM_ERR_INVALID_ARG, "invalid argument");
    if (m == 0) return DPMM_OK;
    double* d_r = nullptr;
    int32_t* d_idx = nullptr;
    DPMM_TRY(dev_alloc(&d_r, (size_t)2 * m + 2));
    dpmm_status s = dev_alloc(&d_idx, (size_t)m);
    const float* du = nullptr;
    if (s == DPMM_OK) s = stage_uniforms(c, u, 2 * c->N, &du);
    if (s == DPMM_OK) {
        cudaError_t e = cudaMemcpyAsync(d_r, loglik, sizeof(double) * 2 * m, cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_r + 2 * m, lr_weights, sizeof(double) * 2, cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_idx, indices, sizeof(int32_t) * m, cudaMemcpyHostToDevice, c->stream);
        if (e != cudaSuccess) s = cuda_status(e, "copy");
    }
    if (s == DPMM_OK) s = launch_sample_log_cat_sub(c, m, d_r, d_idx, d_r + 2 * m, du);
    if (s == DPMM_OK) {
        cudaError_t e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) s = cuda_status(e, "dpmm_sample_log_cat_array_sub_cluster");
    }
    cudaFree(d_r);
    if (d_idx) cudaFree(d_idx);
    invalidate_stats(c);
    return s;
}

// ----------------------------------------------------------------- priors + Hastings
extern "C" dpmm_status dpmm_set_prior_niw(dpmm_ctx* c, double k, const double* m, double v, const double* psi)
{
    if (!c || !m || !psi) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    if (c->prior != DPMM_PRIOR_GAUSSIAN) return fail(DPMM_ERR_STATE, "context is not Gaussian");
    const int D = c->D;
    std::vector<double> L;
    if (!la::cholesky(psi, D, L)) return fail(DPMM_ERR_NOT_PD, "prior psi is not positive definite");
    c->prior_logdet = la::logdet_from_chol(L, D);
    c->prior_identity = true;
    for (int j = 0; j < D && c->prior_identity; ++j) {
        if (m[j] != 0.0) c->prior_identity = false;
        for (int i = 0; i < D; ++i)
            if (psi[(size_t)j * D + i] != (i == j ? 1.0 : 0.0)) c->prior_identity = false;
    }
    c->prior_k = k;
    c->prior_v = v;
    std::vector<double> h((size_t)D + D * D);
    std::memcpy(h.data(), m, sizeof(double) * D);
    std::memcpy(h.data() + D, psi, sizeof(double) * D * D);
    DPMM_CUDA_TRY(cudaMemcpy(c->d_prior, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice));
    c->prior_set = true;
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_set_outlier_prior_niw(dpmm_ctx* c, double k, const double* m, double v, const double* psi)
{
    if (!c || !m || !psi) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    if (c->prior != DPMM_PRIOR_GAUSSIAN) return fail(DPMM_ERR_STATE, "context is not Gaussian");
    const int D = c->D;
    std::vector<double> L;
    if (!la::cholesky(psi, D, L)) return fail(DPMM_ERR_NOT_PD, "outlier prior psi is not positive definite");
    if (!c->d_prior2) DPMM_TRY(dev_alloc(&c->d_prior2, (size_t)D + (size_t)D * D));
    if (!c->d_prior_sel) {
        DPMM_TRY(dev_alloc(&c->d_prior_sel, (size_t)c->k_max));
        DPMM_CUDA_TRY(cudaMemset(c->d_prior_sel, 0, (size_t)c->k_max));
    }
    std::vector<double> h((size_t)D + D * D);
    std::memcpy(h.data(), m, sizeof(double) * D);
    std::memcpy(h.data() + D, psi, sizeof(double) * D * D);
    DPMM_CUDA_TRY(cudaMemcpy(c->d_prior2, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice));
    c->prior2_logdet = la::logdet_from_chol(L, D);
    c->prior2_k = k;
    c->prior2_v = v;
    if (!c->d_cbase) {
        DPMM_TRY(dev_alloc(&c->d_cbase, 3 * (size_t)c->k_max));
        DPMM_CUDA_TRY(cudaMemset(c->d_cbase, 0, sizeof(double) * 3 * (size_t)c->k_max));
    }
    c->outlier_layout = 1;
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_set_cluster_priors(dpmm_ctx* c, int K, const uint8_t* second)
{
    if (!c || (K > 0 && !second)) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    if (K < 0 || K > c->k_max) return fail(DPMM_ERR_INVALID_ARG, "K out of range [0, k_max]");
    if (!c->outlier_layout) return fail(DPMM_ERR_STATE, "no outlier prior set");
    if (K == 0) return DPMM_OK;
    uint8_t* h = reinterpret_cast<uint8_t*>(c->h_pinned) + sizeof(double) * 3 * (size_t)c->k_max;
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));   // the pinned stage may still be in flight
    std::memcpy(h, second, (size_t)K);
    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_prior_sel, h, (size_t)K, cudaMemcpyHostToDevice, c->stream));
    g_h2d_bytes.fetch_add((size_t)K, std::memory_order_relaxed);
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_set_outlier_prior_multinomial(dpmm_ctx* c, const double* alpha)
{
    if (!c || !alpha) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    if (c->prior != DPMM_PRIOR_MULTINOMIAL) return fail(DPMM_ERR_STATE, "context is not multinomial");
    if (!c->d_prior2) DPMM_TRY(dev_alloc(&c->d_prior2, (size_t)c->D));
    if (!c->d_prior_sel) {
        DPMM_TRY(dev_alloc(&c->d_prior_sel, (size_t)c->k_max));
        DPMM_CUDA_TRY(cudaMemset(c->d_prior_sel, 0, (size_t)c->k_max));
    }
    DPMM_CUDA_TRY(cudaMemcpy(c->d_prior2, alpha, sizeof(double) * c->D, cudaMemcpyHostToDevice));
    c->outlier_layout = 1;
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_set_prior_multinomial(dpmm_ctx* c, const double* alpha)
{
    if (!c || !alpha) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    if (c->prior != DPMM_PRIOR_MULTINOMIAL) return fail(DPMM_ERR_STATE, "context is not multinomial");
    DPMM_CUDA_TRY(cudaMemcpy(c->d_prior, alpha, sizeof(double) * c->D, cudaMemcpyHostToDevice));
    c->prior_set = true;
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_split_hastings(dpmm_ctx* c, int K, double alpha, double* lml, double* split_log_hr)
{
    if (!c || K < 1 || K > c->k_max) return fail(DPMM_ERR_INVALID_ARG, "invalid argument");
    {
        PhaseTimer pt(c, PH_SPLIT_HR);
        DPMM_TRY(launch_split_hastings(c, K, alpha));
    }
    if (lml) DPMM_CUDA_TRY(cudaMemcpyAsync(lml, c->d_lml, sizeof(double) * 3 * K, cudaMemcpyDeviceToHost, c->stream));
    if (split_log_hr)
        DPMM_CUDA_TRY(cudaMemcpyAsync(split_log_hr, c->d_split_hr, sizeof(double) * K, cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_merge_hastings(dpmm_ctx* c, int K, double alpha, double* merge_log_hr)
{
    if (!c || K < 1 || K > c->k_max) return fail(DPMM_ERR_INVALID_ARG, "invalid argument");
    {
        PhaseTimer pt(c, PH_MERGE_HR);
        DPMM_TRY(launch_merge_hastings(c, K, alpha));
    }
    if (merge_log_hr)
        DPMM_CUDA_TRY(cudaMemcpyAsync(merge_log_hr, c->d_merge_hr, sizeof(double) * (size_t)K * K,
                                      cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return DPMM_OK;
}

// ----------------------------------------------------------------- all-points statistics
namespace dpmm {

__global__ void k_fill_i32(int32_t* __restrict__ a, int64_t n, int32_t v)
{
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) a[i] = v;
}

dpmm_status launch_fill_labels(dpmm_ctx* c, int32_t value)
{
    k_fill_i32<<<(unsigned)((c->N + 255) / 256), 256, 0, c->stream>>>(c->d_labels, c->N, value);
    DPMM_CUDA_TRY(cudaGetLastError());
    c->perm_K = -1;
    invalidate_stats(c);
    return DPMM_OK;
}

// Statistics of every point (slot 0 of a one-cluster reduction over the label-ordered
// machinery); the labels are saved and restored around it.  Points need sub-labels in {1, 2}.
dpmm_status all_points_stats(dpmm_ctx* c, int64_t* count, double* sum, double* S)
{
    int32_t* saved = reinterpret_cast<int32_t*>(c->d_bits);
    DPMM_CUDA_TRY(cudaMemcpyAsync(saved, c->d_labels, sizeof(int32_t) * c->N, cudaMemcpyDeviceToDevice, c->stream));
    const int kp = c->K_params;
    DPMM_TRY(launch_fill_labels(c, 1));
    // shift of the accumulation: the mean parameter slot 0 is replaced by zeros for the call
    std::vector<float> zero(c->Dp, 0.f), keep(c->Dp);
    DPMM_CUDA_TRY(cudaMemcpyAsync(keep.data(), c->d_mu, sizeof(float) * c->Dp, cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_mu, zero.data(), sizeof(float) * c->Dp, cudaMemcpyHostToDevice, c->stream));
    c->K_params = std::max(kp, 1);
    int32_t idx = 0;
    int64_t cnt[3];
    const int D = c->D;
    std::vector<double> sm(3 * (size_t)D), SS(c->prior == DPMM_PRIOR_GAUSSIAN ? 3 * (size_t)D * D : 0);
    invalidate_stats(c);
    dpmm_status st = dpmm_create_sufficient_statistics(c, 1, &idx, cnt, sm.data(), SS.empty() ? nullptr : SS.data());
    c->K_params = kp;
    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_mu, keep.data(), sizeof(float) * c->Dp, cudaMemcpyHostToDevice, c->stream));
    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_labels, saved, sizeof(int32_t) * c->N, cudaMemcpyDeviceToDevice, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->perm_K = -1;
    invalidate_stats(c);
    DPMM_TRY(st);
    if (count) *count = cnt[0];
    if (sum) std::memcpy(sum, sm.data(), sizeof(double) * D);
    if (S && !SS.empty()) std::memcpy(S, SS.data(), sizeof(double) * D * D);
    return DPMM_OK;
}

}  // namespace dpmm

namespace dpmm {

void invalidate_stats(dpmm_ctx* c)
{
    c->stats_K = -1;
    std::fill(c->stats_ok.begin(), c->stats_ok.end(), 0);
}

void invalidate_stats(dpmm_ctx* c, int k)
{
    if (k >= 0 && k < (int)c->stats_ok.size()) c->stats_ok[k] = 0;
}

dpmm_status ensure_stats(dpmm_ctx* c, int K)
{
    if (K > c->k_max) return fail(DPMM_ERR_INVALID_ARG, "K above capacity");
    int missing = 0;
    for (int k = 0; k < K; ++k) missing += !c->stats_ok[k];
    if (!missing) return DPMM_OK;
    PhaseTimer pt(c, PH_STATS);
    if (c->stats_K < 0 || missing == K) {
        DPMM_TRY(launch_sub_labels_and_stats(c, K, nullptr, nullptr, false));
        return DPMM_OK;
    }
    std::vector<uint8_t> m(K);
    for (int k = 0; k < K; ++k) m[k] = !c->stats_ok[k];
    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_mask, m.data(), K, cudaMemcpyHostToDevice, c->stream));
    DPMM_TRY(launch_sub_labels_and_stats(c, K, nullptr, nullptr, false, c->d_mask));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));   // the host mask must outlive the copy
    for (int k = 0; k < K; ++k) c->stats_ok[k] = 1;
    c->stats_K = std::max(c->stats_K, K);
    return DPMM_OK;
}

}  // namespace dpmm

extern "C" dpmm_status dpmm_set_label_pruning(dpmm_ctx* c, double margin)
{
    if (!c) return fail(DPMM_ERR_INVALID_ARG, "null context");
    if (!c->d_prune_rh) {
        if (margin > 0) return fail(DPMM_ERR_INVALID_ARG, "the pruned label phase needs the NIW prior and D <= 64");
        return DPMM_OK;
    }
    c->prune_margin = margin > 0 ? (float)margin : 0.f;
    c->prune_wait = 0;
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_label_pruning_stats(const dpmm_ctx* c, double* out)
{
    if (!c || !out) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    out[0] = (double)c->prune_tries;
    out[1] = (double)c->prune_used;
    out[2] = c->prune_used ? c->prune_extra / (double)c->prune_used : 0.0;
    out[3] = c->prune_margin;
    out[4] = c->prune_last_extra;
    out[5] = (double)c->prune_last_over;
    return DPMM_OK;
}

// ----------------------------------------------------------------- label agreement (verbose mode)
// NMI = 2 I(X;Y) / (H(X) + H(Y)) as dp_parallel_sampling.cpp:171-179 computes it (through MIToolbox's
// calcMutualInformation / calcEntropy; the ratio does not depend on the logarithm's base), and the
// variation of information H(X) + H(Y) - 2 I(X;Y) in nats, from a contingency table.
extern "C" dpmm_status dpmm_nmi_from_table(const int64_t* table, int K, int G, double* nmi, double* vi)
{
    if (!table || K < 1 || G < 1) return fail(DPMM_ERR_INVALID_ARG, "bad contingency table");
    std::vector<double> a(K, 0.0), b(G, 0.0);
    double n = 0.0;
    for (int k = 0; k < K; ++k)
        for (int g = 0; g < G; ++g) {
            const double v = (double)table[(size_t)k * G + g];
            a[k] += v;
            b[g] += v;
            n += v;
        }
    if (n <= 0) return fail(DPMM_ERR_INVALID_ARG, "empty contingency table");
    double ha = 0, hb = 0, mi = 0;
    for (double v : a) if (v > 0) ha -= v / n * std::log(v / n);
    for (double v : b) if (v > 0) hb -= v / n * std::log(v / n);
    for (int k = 0; k < K; ++k)
        for (int g = 0; g < G; ++g) {
            const double v = (double)table[(size_t)k * G + g];
            if (v > 0) mi += v / n * std::log(v * n / (a[k] * b[g]));
        }
    if (nmi) *nmi = (ha + hb) > 0 ? 2 * mi / (ha + hb) : 1.0;
    if (vi) *vi = std::max(0.0, ha + hb - 2 * mi);
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_set_ground_truth(dpmm_ctx* c, const int32_t* gt)
{
    if (!c) return fail(DPMM_ERR_INVALID_ARG, "null context");
    DPMM_CUDA_TRY(cudaSetDevice(c->device));
    if (c->d_gt) cudaFree(c->d_gt);
    if (c->d_ctab) cudaFree(c->d_ctab);
    c->d_gt = nullptr;
    c->d_ctab = nullptr;
    c->gt_G = 0;
    if (!gt) return DPMM_OK;
    std::vector<int32_t> ids(c->N);
    int G = 0;
    if (c->shard_world > 1) {
        // the same dense ids on every shard: values in [0, 65536), ids in ascending order of the
        // values present anywhere in the data set (presence summed over the shards)
        constexpr int kV = 1 << 16;
        std::vector<double> present(kV, 0.0);
        for (int64_t i = 0; i < c->N; ++i) {
            if (gt[i] < 0 || gt[i] >= kV)
                return fail(DPMM_ERR_INVALID_ARG, "a sharded context takes ground-truth values in [0, 65536)");
            present[gt[i]] = 1.0;
        }
        double* d_pres = nullptr;
        DPMM_TRY(dev_alloc(&d_pres, (size_t)kV));
        DPMM_CUDA_TRY(cudaMemcpy(d_pres, present.data(), sizeof(double) * kV, cudaMemcpyHostToDevice));
        const dpmm_status xs = shard_allreduce(c, d_pres, kV);
        cudaError_t e = xs == DPMM_OK ? cudaMemcpy(present.data(), d_pres, sizeof(double) * kV, cudaMemcpyDeviceToHost)
                                      : cudaSuccess;
        cudaFree(d_pres);
        DPMM_TRY(xs);
        DPMM_CUDA_TRY(e);
        std::vector<int32_t> id_of(kV, -1);
        for (int v = 0; v < kV; ++v)
            if (present[v] > 0) id_of[v] = G++;
        for (int64_t i = 0; i < c->N; ++i) ids[i] = id_of[gt[i]];
    } else {
        // dense ids in order of first appearance
        std::unordered_map<int32_t, int32_t> map;
        for (int64_t i = 0; i < c->N; ++i) {
            auto it = map.emplace(gt[i], (int32_t)map.size()).first;
            ids[i] = it->second;
        }
        G = (int)map.size();
    }
    if ((size_t)G * (size_t)c->k_max > ((size_t)1 << 26))
        return fail(DPMM_ERR_INVALID_ARG, "too many ground-truth classes for k_max (k_max x classes > 2^26)");
    DPMM_TRY(dev_alloc(&c->d_gt, (size_t)c->N));
    DPMM_TRY(dev_alloc(&c->d_ctab, (size_t)G * c->k_max));
    DPMM_CUDA_TRY(cudaMemcpy(c->d_gt, ids.data(), sizeof(int32_t) * (size_t)c->N, cudaMemcpyHostToDevice));
    g_h2d_bytes += sizeof(int32_t) * (size_t)c->N;
    c->gt_G = G;
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_label_agreement(dpmm_ctx* c, int K, double* nmi, double* vi)
{
    if (!c) return fail(DPMM_ERR_INVALID_ARG, "null context");
    if (!c->d_gt) return fail(DPMM_ERR_STATE, "no ground truth set (dpmm_set_ground_truth)");
    if (K < 1 || K > c->k_max) return fail(DPMM_ERR_INVALID_ARG, "K out of range [1, k_max]");
    DPMM_CUDA_TRY(cudaSetDevice(c->device));
    const int G = c->gt_G;
    const size_t T = (size_t)K * G;
    DPMM_CUDA_TRY(cudaMemsetAsync(c->d_ctab, 0, sizeof(unsigned long long) * T, c->stream));
    const size_t sm = T <= (size_t)kCtabSmem ? sizeof(unsigned int) * T : 0;
    const int64_t blocks = std::min<int64_t>((c->N + 255) / 256, (int64_t)c->num_sms * 4);
    k_contingency<<<(unsigned)std::max<int64_t>(blocks, 1), 256, sm, c->stream>>>(c->d_labels, c->d_gt, c->N, K, G,
                                                                              c->d_ctab);
    DPMM_LAUNCHED();
    std::vector<int64_t> table(T);
    DPMM_CUDA_TRY(cudaMemcpyAsync(table.data(), c->d_ctab, sizeof(int64_t) * T, cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    g_d2h_bytes += sizeof(int64_t) * T;
    if (c->shard_world > 1) {   // the whole data set's table (counts below 2^53 are exact as doubles)
        if (T > c->xchg_len) return fail(DPMM_ERR_INVALID_ARG, "contingency table larger than the exchange buffer");
        std::vector<double> tv(table.begin(), table.end());
        DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_xchg, tv.data(), sizeof(double) * T, cudaMemcpyHostToDevice, c->stream));
        DPMM_TRY(shard_allreduce(c, c->d_xchg, (int64_t)T));
        DPMM_CUDA_TRY(cudaMemcpyAsync(tv.data(), c->d_xchg, sizeof(double) * T, cudaMemcpyDeviceToHost, c->stream));
        DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
        for (size_t i = 0; i < T; ++i) table[i] = (int64_t)tv[i];
    }
    return dpmm_nmi_from_table(table.data(), K, G, nmi, vi);
}

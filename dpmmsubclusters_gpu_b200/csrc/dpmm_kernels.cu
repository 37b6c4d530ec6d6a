// dpmm_kernels.cu -- SIMT kernels of the per-iteration path (the "plain FP32 form") and the
// integer passes shared by every form: label-ordered permutation, fused sub-label draw +
// segmented sufficient statistics, relabel passes, test seams.
//
// Reference correspondence (DPMMSubClusters/):
//   k_gauss_labels_simt   cudaKernel_gaussian.cu:82-113 + cudaKernel.cu:374-403, 805-829, 27-124
//                         (one kernel: K log-likelihood columns, softmax, alias draw / argmax)
//   k_mult_labels_simt    cudaKernel_multinomial.cu:22-35, 60-76 + the same softmax/draw
//   k_hist/k_scan/k_scatter  replace find_indices (cudaKernel.cu:189-200): a stable counting
//                         sort of the points by label instead of K atomic compactions
//   k_gauss_sub_stats     cudaKernel.cu:1299-1398 + cudaKernel_gaussian.cu:43-79 (sub-labels)
//                         fused with cudaKernel.cu:844-941 + cudaKernel_gaussian.cu:126-168
//   k_relabel             cudaKernel.cu:172-263 (split / merge / reset / remove)
#include <algorithm>
#include <vector>

#include "dpmm_device.cuh"

namespace dpmm {

RngArgs rng_args(dpmm_ctx* c, const float* d_ucaller)
{
    RngArgs r;
    r.kind = c->rng_kind;
    r.seed = c->seed;
    r.ctr = c->philox_ctr++;
    r.states = c->d_curand;
    r.ucaller = d_ucaller;
    r.offset = c->pt_offset;
    return r;
}

static inline int blocks_for(int64_t n, int t) { return (int)((n + t - 1) / t); }

// ----------------------------------------------------------------------------- init draws
// per-point XORWOW state, subsequence = the global point index (offset: the shard's first point)
__global__ void k_init_curand(curandStateXORWOW* st, uint64_t seed, int64_t n, int64_t offset)
{
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) curand_init(seed, (unsigned long long)(i + offset), 0, &st[i]);   // cudaKernel.cu:19-25
}

dpmm_status launch_init_curand(dpmm_ctx* c)
{
    k_init_curand<<<blocks_for(c->N, 256), 256, 0, c->stream>>>(c->d_curand, c->seed, c->N, c->pt_offset);
    DPMM_LAUNCHED();
    return DPMM_OK;
}

__global__ void k_labels_init(RngArgs r, int64_t n, int ic, int outlier, int32_t* labels)
{
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float u = draw_uniform1(r, i);
    // cudaKernel.cu:158-161
    labels[i] = (int)((double)u * ((double)(ic - 1) + 0.999999) + 1.0 + (outlier ? 1.0 : 0.0));
}

__global__ void k_sub_labels_init(RngArgs r, int64_t n, int32_t* sub)
{
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float u = draw_uniform1(r, i);
    sub[i] = (int)((double)u * (2.0 - 1.0 + 0.999999) + 1.0);   // cudaKernel.cu:144-147
}

dpmm_status launch_labels_init(dpmm_ctx* c, int ic, double outlier_mod, const float* d_u)
{
    RngArgs r = rng_args(c, d_u);
    k_labels_init<<<blocks_for(c->N, 256), 256, 0, c->stream>>>(r, c->N, ic, outlier_mod > 0 ? 1 : 0, c->d_labels);
    DPMM_LAUNCHED();
    c->perm_K = -1;
    return DPMM_OK;
}

dpmm_status launch_sub_labels_init(dpmm_ctx* c, const float* d_u)
{
    RngArgs r = rng_args(c, d_u);
    k_sub_labels_init<<<blocks_for(c->N, 256), 256, 0, c->stream>>>(r, c->N, c->d_sub);
    DPMM_LAUNCHED();
    return DPMM_OK;
}

// the two uniforms per point of the next draw, written out (d_u: 2N), advancing the generator
__global__ void k_draw_uniform2(RngArgs r, int64_t n, float* d_u)
{
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float u1, u2;
    draw_uniform2(r, i, u1, u2);
    d_u[2 * i] = u1;
    d_u[2 * i + 1] = u2;
}

dpmm_status launch_draw_uniforms(dpmm_ctx* c, float* d_u)
{
    RngArgs r = rng_args(c, nullptr);
    k_draw_uniform2<<<blocks_for(c->N, 256), 256, 0, c->stream>>>(r, c->N, d_u);
    DPMM_LAUNCHED();
    return DPMM_OK;
}

// ----------------------------------------------------------------------------- label phase
// Shared epilogue: r values of one point (stride P in shared memory) -> label.
template <int P>
__device__ __forceinline__ int draw_from_r(float* sr, int p, int K, int final_, const RngArgs& rng, int64_t pt)
{
    if (final_) {
        // update_labels_by_max_index_kernel (cudaKernel.cu:405-424): first maximum wins
        float best = sr[p];
        int arg = 0;
        for (int k = 1; k < K; ++k) {
            float v = sr[k * P + p];
            if (best < v) { best = v; arg = k; }
        }
        return arg + 1;
    }
    // build_log_likelihood_array_kernel (cudaKernel.cu:374-403): max, exp, normalise
    float mx = sr[p];
    for (int k = 1; k < K; ++k) mx = fmaxf(mx, sr[k * P + p]);
    float sum = 0.f;
    for (int k = 0; k < K; ++k) {
        float e = __expf(sr[k * P + p] - mx);
        sr[k * P + p] = e;
        sum += e;
    }
    const float inv = 1.0f / sum;
    const float fk = (float)K;
    for (int k = 0; k < K; ++k) sr[k * P + p] = (sr[k * P + p] * inv) * fk;   // y_k = p_k * K
    float u1, u2;
    draw_uniform2(rng, pt, u1, u2);
    return alias_draw_stream(sr + p, P, K, u1, u2);
}

// Gaussian label phase, FP32 SIMT: one thread per point, x in registers, each cluster's
// precision factor (transposed) broadcast from shared memory.
//   z_j = sum_i W(i,j) x_i - b_j,   r_k = c_k - 0.5 * sum_j z_j^2
// r = c - 0.5 |W^T x - b|^2 for one point (x in registers) and one cluster whose transposed factor
// (Wt[j][i] = W(i, j)) and b are staged in shared memory
template <int DP>
__device__ __forceinline__ float gauss_r_point(const float* __restrict__ sW, const float* __restrict__ sbv,
                                               const float (&xr)[DP], float c)
{
    float q = 0.f;
#pragma unroll 2
    for (int j = 0; j < DP; j += 2) {
        const float4* w0 = reinterpret_cast<const float4*>(sW + j * DP);
        const float4* w1 = reinterpret_cast<const float4*>(sW + (j + 1) * DP);
        float z0 = -sbv[j], z1 = -sbv[j + 1];
        float z0b = 0.f, z1b = 0.f;
#pragma unroll
        for (int i4 = 0; i4 < DP / 4; ++i4) {
            float4 a = w0[i4], b = w1[i4];
            z0 = fmaf(a.x, xr[4 * i4 + 0], z0);
            z1 = fmaf(b.x, xr[4 * i4 + 0], z1);
            z0b = fmaf(a.y, xr[4 * i4 + 1], z0b);
            z1b = fmaf(b.y, xr[4 * i4 + 1], z1b);
            z0 = fmaf(a.z, xr[4 * i4 + 2], z0);
            z1 = fmaf(b.z, xr[4 * i4 + 2], z1);
            z0b = fmaf(a.w, xr[4 * i4 + 3], z0b);
            z1b = fmaf(b.w, xr[4 * i4 + 3], z1b);
        }
        z0 += z0b;
        z1 += z1b;
        q = fmaf(z0, z0, q);
        q = fmaf(z1, z1, q);
    }
    return c - 0.5f * q;
}

// one block of P points starting at pt0 (the body of k_gauss_labels_simt and of its batched form)
template <int DP, int P>
__device__ __forceinline__ void gauss_labels_tile(const float* __restrict__ x, int64_t N,
                                                  const float* __restrict__ Wt, const float* __restrict__ bvec,
                                                  const float* __restrict__ cvec, int K, int final_,
                                                  const RngArgs& rng, int32_t* __restrict__ labels,
                                                  float* __restrict__ r_out, int64_t pt0, unsigned char* smem)
{
    float* sW = reinterpret_cast<float*>(smem);          // DP*DP
    float* sbv = sW + DP * DP;                            // DP
    float* sx = sbv + DP;                                 // P*(DP+1)
    float* sr = sx + P * (DP + 1);                        // K*P

    const int p = threadIdx.x;
    const int64_t pt = pt0 + p;
    const bool valid = pt < N;

    // stage the tile's points (contiguous rows) with coalesced loads
    const int64_t rows = min((int64_t)P, N - pt0);
    for (int e = p; e < P * DP; e += P) {
        int pp = e / DP, i = e % DP;
        sx[pp * (DP + 1) + i] = pp < rows ? x[(pt0 + pp) * DP + i] : 0.f;
    }
    __syncthreads();
    float xr[DP];
#pragma unroll
    for (int i = 0; i < DP; ++i) xr[i] = sx[p * (DP + 1) + i];

    for (int k = 0; k < K; ++k) {
        __syncthreads();
        const float4* src = reinterpret_cast<const float4*>(Wt + (size_t)3 * k * DP * DP);
        float4* dst = reinterpret_cast<float4*>(sW);
        for (int e = p; e < DP * DP / 4; e += P) dst[e] = src[e];
        for (int e = p; e < DP; e += P) sbv[e] = bvec[(size_t)3 * k * DP + e];
        __syncthreads();
        const float r = gauss_r_point<DP>(sW, sbv, xr, cvec[3 * k]);
        sr[k * P + p] = r;
        if (r_out && valid) r_out[pt * K + k] = r;
    }
    if (!valid) return;
    labels[pt] = draw_from_r<P>(sr, p, K, final_, rng, pt);
}

template <int DP, int P>
__global__ void __launch_bounds__(P) k_gauss_labels_simt(
    const float* __restrict__ x, int64_t N, const float* __restrict__ Wt, const float* __restrict__ bvec,
    const float* __restrict__ cvec, int K, int final_, RngArgs rng, int32_t* __restrict__ labels,
    float* __restrict__ r_out)
{
    extern __shared__ __align__(16) unsigned char smem[];
    gauss_labels_tile<DP, P>(x, N, Wt, bvec, cvec, K, final_, rng, labels, r_out, (int64_t)blockIdx.x * P, smem);
}

// Batched form: one launch for many data sets of the same padded dimension.  Block b works on
// item items[b] = (data set, block of P points of it); the data set's buffers, K, mode and random
// stream come from its descriptor.  Shared memory is sized for the largest K of the batch.
template <int DP, int P>
__global__ void __launch_bounds__(P) k_gauss_labels_batched(const LabelJob* __restrict__ jobs,
                                                            const int2* __restrict__ items)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int2 it = items[blockIdx.x];
    const LabelJob& j = jobs[it.x];
    gauss_labels_tile<DP, P>(j.x, j.N, j.Wt, j.b, j.c, j.K, j.final_, j.rng, j.labels, nullptr, (int64_t)it.y * P,
                             smem);
}

size_t gauss_label_smem_bytes(int DP, int P, int K)
{
    return sizeof(float) * (DP * DP + DP + P * (DP + 1) + (size_t)K * P);
}

template <int DP, int P>
static dpmm_status launch_labels_batched_t(const LabelJob* d_jobs, const int2* d_items, int nitems, int kmax,
                                           cudaStream_t st)
{
    const size_t sm = gauss_label_smem_bytes(DP, P, kmax);
    if (sm > 220 * 1024) return fail(DPMM_ERR_INVALID_ARG, "too many clusters for the batched label kernel");
    auto kern = k_gauss_labels_batched<DP, P>;
    DPMM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    kern<<<nitems, P, sm, st>>>(d_jobs, d_items);
    DPMM_LAUNCHED();
    return DPMM_OK;
}

template <int DP>
static dpmm_status launch_labels_batched_dp(int P, const LabelJob* d_jobs, const int2* d_items, int nitems, int kmax,
                                            cudaStream_t st)
{
    switch (P) {
        case 32: return launch_labels_batched_t<DP, 32>(d_jobs, d_items, nitems, kmax, st);
        case 64: return launch_labels_batched_t<DP, 64>(d_jobs, d_items, nitems, kmax, st);
        default: return launch_labels_batched_t<DP, 128>(d_jobs, d_items, nitems, kmax, st);
    }
}

dpmm_status launch_labels_batched(int Dp, int P, const LabelJob* d_jobs, const int2* d_items, int nitems, int kmax,
                                  cudaStream_t st)
{
    switch (Dp) {
        case 4: return launch_labels_batched_dp<4>(P, d_jobs, d_items, nitems, kmax, st);
        case 8: return launch_labels_batched_dp<8>(P, d_jobs, d_items, nitems, kmax, st);
        case 16: return launch_labels_batched_dp<16>(P, d_jobs, d_items, nitems, kmax, st);
        case 32: return launch_labels_batched_dp<32>(P, d_jobs, d_items, nitems, kmax, st);
        case 64: return launch_labels_batched_dp<64>(P, d_jobs, d_items, nitems, kmax, st);
        case 128: return launch_labels_batched_dp<128>(P, d_jobs, d_items, nitems, kmax, st);
        default: return fail(DPMM_ERR_INVALID_ARG, "unsupported padded dimension");
    }
}

// Multinomial label phase, FP32 SIMT: tiled dot products r[p][k] = sum_d x[p][d] * logtheta[k][d]
// (64 points x 64 clusters per pass, 256 threads, 4x4 register tile), then the same draw.
template <int P>
__global__ void __launch_bounds__(256) k_mult_labels_simt(
    const float* __restrict__ x, int64_t N, int Dp, const float* __restrict__ logtheta,
    int K, int final_, RngArgs rng, int32_t* __restrict__ labels, float* __restrict__ r_out)
{
    constexpr int KG = 64, DC = 32;
    extern __shared__ __align__(16) unsigned char smem[];
    float* sX = reinterpret_cast<float*>(smem);          // P x (DC+1)
    float* sT = sX + P * (DC + 1);                        // KG x (DC+1)
    float* sr = sT + KG * (DC + 1);                       // K*P

    const int tid = threadIdx.x;
    const int64_t pt0 = (int64_t)blockIdx.x * P;
    const int64_t rows = min((int64_t)P, N - pt0);
    const int tp = tid / 16, tk = tid % 16;              // 16 x 16 thread grid, 4 x 4 outputs each

    for (int g = 0; g < K; g += KG) {
        float acc[4][4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] = 0.f;
        for (int d0 = 0; d0 < Dp; d0 += DC) {
            __syncthreads();
            for (int e = tid; e < P * DC; e += 256) {
                int pp = e / DC, dd = e % DC;
                sX[pp * (DC + 1) + dd] = pp < rows ? x[(pt0 + pp) * Dp + d0 + dd] : 0.f;
            }
            for (int e = tid; e < KG * DC; e += 256) {
                int kk = e / DC, dd = e % DC;
                sT[kk * (DC + 1) + dd] = (g + kk) < K ? logtheta[(size_t)3 * (g + kk) * Dp + d0 + dd] : 0.f;
            }
            __syncthreads();
#pragma unroll 8
            for (int dd = 0; dd < DC; ++dd) {
                float xv[4], tv[4];
#pragma unroll
                for (int a = 0; a < 4; ++a) xv[a] = sX[(tp + 16 * a) * (DC + 1) + dd];
#pragma unroll
                for (int b = 0; b < 4; ++b) tv[b] = sT[(tk + 16 * b) * (DC + 1) + dd];
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < 4; ++b) acc[a][b] = fmaf(xv[a], tv[b], acc[a][b]);
            }
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                int pp = tp + 16 * a, kk = g + tk + 16 * b;
                if (kk < K) {
                    sr[kk * P + pp] = acc[a][b];
                    if (r_out && pp < rows) r_out[(pt0 + pp) * K + kk] = acc[a][b];
                }
            }
    }
    __syncthreads();
    if (tid >= P || tid >= rows) return;
    const int64_t pt = pt0 + tid;
    labels[pt] = draw_from_r<P>(sr, tid, K, final_, rng, pt);
}

static size_t gauss_label_smem(int DP, int P, int K)
{
    return sizeof(float) * (DP * DP + DP + P * (DP + 1) + (size_t)K * P);
}

template <int DP, int P>
static dpmm_status launch_gauss_labels_t(dpmm_ctx* c, int K, int final_, RngArgs r, float* d_rout)
{
    const size_t sm = gauss_label_smem(DP, P, K);
    auto kern = k_gauss_labels_simt<DP, P>;
    DPMM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    kern<<<blocks_for(c->N, P), P, sm, c->stream>>>(c->d_x, c->N, c->d_Wt, c->d_b, c->d_c, K, final_, r,
                                                     c->d_labels, d_rout);
    DPMM_LAUNCHED();
    return DPMM_OK;
}

template <int DP>
static dpmm_status launch_gauss_labels_dp(dpmm_ctx* c, int K, int final_, RngArgs r, float* d_rout)
{
    const size_t cap = 220 * 1024;
    if (gauss_label_smem(DP, 128, K) <= cap) return launch_gauss_labels_t<DP, 128>(c, K, final_, r, d_rout);
    if (gauss_label_smem(DP, 64, K) <= cap) return launch_gauss_labels_t<DP, 64>(c, K, final_, r, d_rout);
    if (gauss_label_smem(DP, 32, K) <= cap) return launch_gauss_labels_t<DP, 32>(c, K, final_, r, d_rout);
    return fail(DPMM_ERR_INVALID_ARG, "too many clusters for the label kernel's shared-memory table");
}

dpmm_status launch_cluster_labels(dpmm_ctx* c, int K, int final_, const float* d_u, float* d_rout)
{
    RngArgs r = rng_args(c, d_u);
    if (c->prior == DPMM_PRIOR_GAUSSIAN) {
        switch (c->Dp) {
            case 4: return launch_gauss_labels_dp<4>(c, K, final_, r, d_rout);
            case 8: return launch_gauss_labels_dp<8>(c, K, final_, r, d_rout);
            case 16: return launch_gauss_labels_dp<16>(c, K, final_, r, d_rout);
            case 32: return launch_gauss_labels_dp<32>(c, K, final_, r, d_rout);
            case 64: return launch_gauss_labels_dp<64>(c, K, final_, r, d_rout);
            case 128: return launch_gauss_labels_dp<128>(c, K, final_, r, d_rout);
            default: return fail(DPMM_ERR_INVALID_ARG, "unsupported padded dimension");
        }
    }
    constexpr int P = 64;
    size_t sm = sizeof(float) * (P * 33 + 64 * 33 + (size_t)K * P);
    if (sm > 220 * 1024) return fail(DPMM_ERR_INVALID_ARG, "too many clusters for the multinomial label kernel");
    DPMM_CUDA_TRY(cudaFuncSetAttribute(k_mult_labels_simt<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_mult_labels_simt<P><<<blocks_for(c->N, P), 256, sm, c->stream>>>(c->d_x, c->N, c->Dp, c->d_mu, K, final_, r,
                                                                       c->d_labels, d_rout);
    DPMM_LAUNCHED();
    return DPMM_OK;
}

// ----------------------------------------------------------------------------- pruned label phase
// The points are taken in chunks of one current cluster h (the label-ordered permutation).  For a
// chunk, r_h is computed exactly for every point; another cluster k is kept only if some point of the
// chunk could have r_k within `margin` nats of its r_h, by two bounds (r_k = c_k - 0.5 |W_k^T (x - mu_k)|^2):
//   chunk bound: |W_k^T (x - mu_k)| >= M_hk - sigma_max(W_k) |x - mu_h|, with M_hk = |W_k^T (mu_h - mu_k)|,
//                sigma_max(W_k)^2 <= max_i sum_j |Lambda_k(i,j)| (Gershgorin), |x - mu_h| <= R;
//   point bound: |W_k^T (x - mu_k)| >= |u^T W_k^T (x - mu_k)| = |v_hk^T x - beta_hk| for the unit vector
//                u = W_k^T (mu_h - mu_k) / M_hk, v_hk = W_k u, beta_hk = v_hk^T mu_k.
// A left-out cluster has r_k(x) < r_h(x) - margin <= max_k' r_k'(x) - margin at every point of the chunk,
// so it carries less than K e^-margin of the point's probability; the draw runs over all K columns with
// it at probability 0, which gives the dense draw's label unless a uniform falls inside that mass.  A
// chunk left with its own cluster only takes it as every point's label.
constexpr int kPrTh = 128;       // threads per block

// one block per cluster k: lam[k] = sqrt of the Gershgorin bound of lambda_max(W_k W_k^T) (inflated);
// for every h: M[h][k] (deflated), v[h][k][DP] and beta[h][k]
template <int DP>
__global__ void __launch_bounds__(kPrTh) k_prune_prep(const float* __restrict__ Wt, const float* __restrict__ mu,
                                                      int K, float* __restrict__ lam, float* __restrict__ M,
                                                      float* __restrict__ V, float* __restrict__ beta)
{
    constexpr int NW = kPrTh / 32;
    constexpr int SW = DP + 1;   // padded row stride: the z loop's lanes read one column each
    constexpr int TPR = kPrTh / DP < DP ? kPrTh / DP : DP;   // threads per Gershgorin row (each >= 1 column)
    static_assert(kPrTh % DP == 0 && DP % TPR == 0, "row split");
    __shared__ float sW[DP * SW];
    __shared__ double red[NW];
    __shared__ double srow_part[kPrTh];
    __shared__ double zs[NW][DP];
    __shared__ double dm[NW][DP];
    const int k = blockIdx.x, t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for (int e = t; e < DP * DP; e += blockDim.x) sW[(e / DP) * SW + e % DP] = Wt[(size_t)3 * k * DP * DP + e];
    __syncthreads();
    if (t < DP * TPR) {   // Gershgorin row sums of W W^T: row t % DP, column share t / DP, four chains
        const int i = t % DP, j0 = (t / DP) * (DP / TPR);
        double srow = 0;
        for (int j = j0; j < j0 + DP / TPR; ++j) {
            double l0 = 0, l1 = 0, l2 = 0, l3 = 0;
#pragma unroll
            for (int cc = 0; cc < DP; cc += 4) {
                l0 = fma((double)sW[cc * SW + i], (double)sW[cc * SW + j], l0);
                l1 = fma((double)sW[(cc + 1) * SW + i], (double)sW[(cc + 1) * SW + j], l1);
                l2 = fma((double)sW[(cc + 2) * SW + i], (double)sW[(cc + 2) * SW + j], l2);
                l3 = fma((double)sW[(cc + 3) * SW + i], (double)sW[(cc + 3) * SW + j], l3);
            }
            srow += fabs((l0 + l1) + (l2 + l3));
        }
        srow_part[t] = srow;
    }
    __syncthreads();
    double rmax = 0;
    if (t < DP) {
        double tot = 0;
        for (int p = 0; p < TPR; ++p) tot += srow_part[t + p * DP];
        rmax = tot;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) rmax = fmax(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
    if (lane == 0) red[warp] = rmax;
    __syncthreads();
    if (t == 0) {
        double m = 0;
        for (int w = 0; w < NW; ++w) m = fmax(m, red[w]);
        lam[k] = (float)(sqrt(m) * (1.0 + 1e-5));
    }
    const float* mk = mu + (size_t)3 * k * DP;
    for (int h = warp; h < K; h += NW) {
        const float* mh = mu + (size_t)3 * h * DP;
        for (int i = lane; i < DP; i += 32) dm[warp][i] = (double)mh[i] - (double)mk[i];
        __syncwarp();
        double q = 0;
        for (int j = lane; j < DP; j += 32) {   // z = W_k^T (mu_h - mu_k)
            double z0 = 0, z1 = 0, z2 = 0, z3 = 0;
#pragma unroll
            for (int i = 0; i < DP; i += 4) {
                z0 = fma((double)sW[j * SW + i], dm[warp][i], z0);
                z1 = fma((double)sW[j * SW + i + 1], dm[warp][i + 1], z1);
                z2 = fma((double)sW[j * SW + i + 2], dm[warp][i + 2], z2);
                z3 = fma((double)sW[j * SW + i + 3], dm[warp][i + 3], z3);
            }
            const double z = (z0 + z1) + (z2 + z3);
            zs[warp][j] = z;
            q += z * z;
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
        __syncwarp();
        const double nz = sqrt(q);
        const double inv = nz > 0 ? 1.0 / nz : 0.0;
        float* vh = V + ((size_t)h * K + k) * DP;
        double bsum = 0;
        for (int i = lane; i < DP; i += 32) {    // v = W_k u, u = z / |z|
            double v0 = 0, v1 = 0, v2 = 0, v3 = 0;
#pragma unroll
            for (int j = 0; j < DP; j += 4) {
                v0 = fma((double)sW[j * SW + i], zs[warp][j], v0);
                v1 = fma((double)sW[(j + 1) * SW + i], zs[warp][j + 1], v1);
                v2 = fma((double)sW[(j + 2) * SW + i], zs[warp][j + 2], v2);
                v3 = fma((double)sW[(j + 3) * SW + i], zs[warp][j + 3], v3);
            }
            const double v = ((v0 + v1) + (v2 + v3)) * inv;
            vh[i] = (float)v;
            bsum += (double)(float)v * (double)mk[i];
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) bsum += __shfl_xor_sync(0xffffffffu, bsum, o);
        if (lane == 0) {
            M[(size_t)h * K + k] = (float)(nz * (1.0 - 1e-5));
            beta[(size_t)h * K + k] = (float)bsum;
        }
        __syncwarp();
    }
}

template <int DP>
__device__ __forceinline__ void load_row(const float* __restrict__ x, int64_t pt, float (&xr)[DP])
{
    const float4* src = reinterpret_cast<const float4*>(x + pt * DP);
#pragma unroll
    for (int q = 0; q < DP / 4; ++q) {
        const float4 v = src[q];
        xr[4 * q] = v.x;
        xr[4 * q + 1] = v.y;
        xr[4 * q + 2] = v.z;
        xr[4 * q + 3] = v.w;
    }
}

// pass 1, one block per chunk (chunk length <= kChunkMax): r_h of every point (into rh, permutation
// order), the clusters the bounds cannot leave out (cand[q] = count, then up to kPrMaxCand indices),
// and the totals cnt[0] += count * chunk length, cnt[1] += (count > capacity).
// Dynamic shared memory: kChunkMax + K * (DP + 3) floats + K ints.
template <int DP>
__global__ void __launch_bounds__(kPrTh) k_prune_scan(const float* __restrict__ x, const int32_t* __restrict__ perm,
                                                      const int32_t* __restrict__ chunk,
                                                      const int32_t* __restrict__ nchunks, const float* __restrict__ Wt,
                                                      const float* __restrict__ bvec, const float* __restrict__ cvec,
                                                      const float* __restrict__ mu, const float* __restrict__ lam,
                                                      const float* __restrict__ M, const float* __restrict__ V,
                                                      const float* __restrict__ beta, int K, float margin,
                                                      float* __restrict__ rh, int32_t* __restrict__ cand,
                                                      unsigned long long* __restrict__ cnt)
{
    __shared__ __align__(16) float sW[DP * DP];
    __shared__ float sbv[DP], smu[DP];
    __shared__ float rmin_w[kPrTh / 32], r2_w[kPrTh / 32];
    __shared__ int n_test;
    __shared__ unsigned int keep[(kMaxKForPrune + 31) / 32];
    extern __shared__ __align__(16) float dsm[];
    float* srh = dsm;                          // kChunkMax
    float* sv = srh + kChunkMax;               // n_test * DP
    float* sbeta = sv + (size_t)K * DP;        // n_test
    float* sck = sbeta + K;                    // n_test
    int* sk = reinterpret_cast<int*>(sck + K); // n_test
    const int q = blockIdx.x, t = threadIdx.x, lane = t & 31, warp = t >> 5;
    if (q >= *nchunks) return;
    const int h = chunk[3 * q], start = chunk[3 * q + 1], L = chunk[3 * q + 2];
    {
        const float4* src = reinterpret_cast<const float4*>(Wt + (size_t)3 * h * DP * DP);
        float4* dst = reinterpret_cast<float4*>(sW);
        for (int e = t; e < DP * DP / 4; e += blockDim.x) dst[e] = src[e];
        for (int e = t; e < DP; e += blockDim.x) {
            sbv[e] = bvec[(size_t)3 * h * DP + e];
            smu[e] = mu[(size_t)3 * h * DP + e];
        }
        for (int e = t; e < (K + 31) / 32; e += blockDim.x) keep[e] = 0u;
        if (t == 0) n_test = 0;
    }
    __syncthreads();
    const float ch = cvec[3 * h];
    float tmin = INFINITY, tr2 = 0.f;
    for (int i = start + t; i < start + L; i += blockDim.x) {
        float xr[DP];
        load_row<DP>(x, perm[i], xr);
        const float r = gauss_r_point<DP>(sW, sbv, xr, ch);
        rh[i] = r;
        srh[i - start] = r;
        tmin = fminf(tmin, r);
        float d2 = 0.f;
#pragma unroll
        for (int e = 0; e < DP; ++e) d2 = fmaf(xr[e] - smu[e], xr[e] - smu[e], d2);
        tr2 = fmaxf(tr2, d2);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        tmin = fminf(tmin, __shfl_xor_sync(0xffffffffu, tmin, o));
        tr2 = fmaxf(tr2, __shfl_xor_sync(0xffffffffu, tr2, o));
    }
    if (lane == 0) {
        rmin_w[warp] = tmin;
        r2_w[warp] = tr2;
    }
    __syncthreads();
    float rmin = rmin_w[0], r2 = r2_w[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
        rmin = fminf(rmin, rmin_w[w]);
        r2 = fmaxf(r2, r2_w[w]);
    }
    const float R = sqrtf(r2) * 1.0001f + 1e-4f;
    // chunk bound: clusters it cannot leave out go to the point test
    for (int k = t; k < K; k += blockDim.x) {
        if (k == h) continue;
        const float d = M[(size_t)h * K + k] - lam[k] * R;
        const float ub = cvec[3 * k] - 0.5f * (d > 0.f ? d * d : 0.f);
        if (!(ub < rmin - margin)) sk[atomicAdd(&n_test, 1)] = k;
    }
    __syncthreads();
    const int nt = n_test;
    for (int e = t; e < nt * DP; e += blockDim.x) {
        const int a = e / DP, i = e % DP;
        sv[e] = V[((size_t)h * K + sk[a]) * DP + i];
    }
    for (int a = t; a < nt; a += blockDim.x) {
        sbeta[a] = beta[(size_t)h * K + sk[a]];
        sck[a] = cvec[3 * sk[a]];
    }
    __syncthreads();
    // point bound
    if (nt > 0) {
        for (int i = start + t; i < start + L; i += blockDim.x) {
            float xr[DP];
            load_row<DP>(x, perm[i], xr);
            const float lim = srh[i - start] - margin;
            for (int a = 0; a < nt; ++a) {
                const float* va = sv + (size_t)a * DP;
                float p0 = -sbeta[a], p1 = 0.f;
#pragma unroll
                for (int e = 0; e < DP; e += 2) {
                    p0 = fmaf(va[e], xr[e], p0);
                    p1 = fmaf(va[e + 1], xr[e + 1], p1);
                }
                const float pr = p0 + p1;
                const float ub = sck[a] - 0.5f * pr * pr;
                if (!(ub < lim)) atomicOr(&keep[sk[a] >> 5], 1u << (sk[a] & 31));
            }
        }
    }
    __syncthreads();
    if (t == 0) {
        int n = 0;
        int32_t* cq = cand + (size_t)q * (kPrMaxCand + 1);
        for (int k = 0; k < K; ++k)
            if ((keep[k >> 5] >> (k & 31)) & 1u) {
                if (n < kPrMaxCand) cq[1 + n] = k;
                ++n;
            }
        cq[0] = n;
        atomicAdd(&cnt[0], (unsigned long long)n * (unsigned long long)L);
        if (n > kPrMaxCand) atomicAdd(&cnt[1], 1ull);
    }
}

// The chunks that kept other clusters, in ascending order, and their number (one block).
__global__ void __launch_bounds__(1024) k_prune_list(const int32_t* __restrict__ nchunks,
                                                     const int32_t* __restrict__ cand, int32_t* __restrict__ list,
                                                     int32_t* __restrict__ count)
{
    __shared__ int wc[32];
    const int nc = *nchunks, t = threadIdx.x, lane = t & 31, warp = t >> 5;
    int base = 0;
    for (int q0 = 0; q0 < nc; q0 += 1024) {
        const int qq = q0 + t;
        const bool kept = qq < nc && cand[(size_t)qq * (kPrMaxCand + 1)] > 0;
        const unsigned bal = __ballot_sync(0xffffffffu, kept);
        if (lane == 0) wc[warp] = __popc(bal);
        __syncthreads();
        int off = 0, tot = 0;
        for (int w = 0; w < 32; ++w) {
            off += w < warp ? wc[w] : 0;
            tot += wc[w];
        }
        if (kept) list[base + off + __popc(bal & ((1u << lane) - 1u))] = qq;
        base += tot;
        __syncthreads();
    }
    if (t == 0) *count = base;
}

// Chunks that kept no other cluster: every point takes its current label h + 1 (no draw; a stateful
// per-point stream still advances).  One block per chunk, no shared memory.
__global__ void __launch_bounds__(256) k_prune_settle(const int32_t* __restrict__ perm,
                                                      const int32_t* __restrict__ chunk,
                                                      const int32_t* __restrict__ nchunks,
                                                      const int32_t* __restrict__ cand, int final_, RngArgs rng,
                                                      int32_t* __restrict__ labels)
{
    const int q = blockIdx.x;
    if (q >= *nchunks || cand[(size_t)q * (kPrMaxCand + 1)] != 0) return;
    const int h = chunk[3 * q], start = chunk[3 * q + 1], L = chunk[3 * q + 2];
    for (int i = start + threadIdx.x; i < start + L; i += blockDim.x) {
        const int64_t p0 = perm[i];
        labels[p0] = h + 1;
        if (!final_) skip_uniform2(rng, p0);   // the argmax of final mode draws nothing
    }
}

// pass 2 for the chunks that kept other clusters, one block per tile of kPrTh points (blockIdx.x =
// position in the list, blockIdx.y = tile): r of the kept clusters (r_h from pass 1; every cluster when
// the chunk kept more than kPrMaxCand).  A point whose kept clusters all lie more than the
// margin below r_h takes h + 1 as well (the chunk bound's guarantee, now from the exact r); the others
// get the draw (or argmax) of the dense label phase over all K columns, the left-out clusters at -inf.
// Shared memory: DP*DP + DP + K*kPrTh floats.
template <int DP>
__global__ void __launch_bounds__(kPrTh) k_prune_draw(const float* __restrict__ x, const int32_t* __restrict__ perm,
                                                      const int32_t* __restrict__ chunk,
                                                      const int32_t* __restrict__ nchunks, const float* __restrict__ Wt,
                                                      const float* __restrict__ bvec, const float* __restrict__ cvec,
                                                      int K, int final_, RngArgs rng, const float* __restrict__ rh,
                                                      const int32_t* __restrict__ cand, float margin,
                                                      const int32_t* __restrict__ list, int32_t* __restrict__ labels)
{
    extern __shared__ __align__(16) unsigned char smem[];
    float* sW = reinterpret_cast<float*>(smem);
    float* sbv = sW + DP * DP;
    float* sr = sbv + DP;
    const int q = list[blockIdx.x], t = threadIdx.x;
    const int h = chunk[3 * q], start = chunk[3 * q + 1], L = chunk[3 * q + 2];
    const int base = start + (int)blockIdx.y * kPrTh;
    if (base >= start + L) return;
    const int32_t* cq = cand + (size_t)q * (kPrMaxCand + 1);
    const int n = cq[0];
    const int i = base + t;
    const bool valid = i < start + L;
    const bool all = n > kPrMaxCand;      // over capacity: every cluster
    const int64_t pt = valid ? perm[i] : 0;
    float xr[DP];
    if (valid) load_row<DP>(x, pt, xr);
    else
#pragma unroll
        for (int e = 0; e < DP; ++e) xr[e] = 0.f;
    for (int k = 0; k < K; ++k) sr[k * kPrTh + t] = -INFINITY;
    const float r_own = valid ? rh[i] : 0.f;
    sr[h * kPrTh + t] = r_own;
    const int m = all ? K : n;
    float best_other = -INFINITY;
    for (int a = 0; a < m; ++a) {
        const int k = all ? a : cq[1 + a];
        if (k == h) continue;
        __syncthreads();
        const float4* src = reinterpret_cast<const float4*>(Wt + (size_t)3 * k * DP * DP);
        float4* dst = reinterpret_cast<float4*>(sW);
        for (int e = t; e < DP * DP / 4; e += blockDim.x) dst[e] = src[e];
        for (int e = t; e < DP; e += blockDim.x) sbv[e] = bvec[(size_t)3 * k * DP + e];
        __syncthreads();
        const float r = gauss_r_point<DP>(sW, sbv, xr, cvec[3 * k]);
        sr[k * kPrTh + t] = r;
        best_other = fmaxf(best_other, r);
    }
    if (!valid) return;
    if (best_other < r_own - margin) {
        labels[pt] = h + 1;
        if (!final_) skip_uniform2(rng, pt);
    } else {
        labels[pt] = draw_from_r<kPrTh>(sr, t, K, final_, rng, pt);
    }
}

static size_t prune_draw_smem(int DP, int K) { return sizeof(float) * ((size_t)DP * DP + DP + (size_t)K * kPrTh); }

template <int DP>
static dpmm_status launch_pruned_dp(dpmm_ctx* c, int K, int final_, const float* d_u, bool tc_dense, bool* used)
{
    DPMM_TRY(build_permutation(c, K));
    k_prune_prep<DP><<<K, kPrTh, 0, c->stream>>>(c->d_Wt, c->d_mu, K, c->d_prune_lam, c->d_prune_M, c->d_prune_V,
                                                 c->d_prune_beta);
    DPMM_LAUNCHED();
    DPMM_CUDA_TRY(cudaMemsetAsync(c->d_prune_cnt, 0, 2 * sizeof(unsigned long long), c->stream));
    int32_t* d_err = c->d_aux + 7;
    DPMM_CUDA_TRY(cudaMemsetAsync(d_err, 0, sizeof(int32_t), c->stream));
    if (tc_scan_supported(c, K)) {
        // r_h and the point bounds as tensor-core products (r_h then equals the dense tensor-core r)
        KernelTimer kt(c, PH_PRUNE_SCAN);
        DPMM_TRY(launch_prune_scan_tc(c, K, d_err));
    } else {
        const size_t ssm = sizeof(float) * ((size_t)kChunkMax + (size_t)K * (DP + 3));
        DPMM_CUDA_TRY(cudaFuncSetAttribute(k_prune_scan<DP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ssm));
        KernelTimer kt(c, PH_PRUNE_SCAN);
        k_prune_scan<DP><<<c->max_chunks, kPrTh, ssm, c->stream>>>(
            c->d_x, c->d_perm, c->d_chunk, c->d_nchunks, c->d_Wt, c->d_b, c->d_c, c->d_mu, c->d_prune_lam,
            c->d_prune_M, c->d_prune_V, c->d_prune_beta, K, c->prune_margin, c->d_prune_rh, c->d_prune_cand,
            c->d_prune_cnt);
        DPMM_LAUNCHED();
    }
    int32_t* d_nlist = c->d_aux + 2;
    k_prune_list<<<1, 1024, 0, c->stream>>>(c->d_nchunks, c->d_prune_cand, c->d_prune_list, d_nlist);
    DPMM_LAUNCHED();
    unsigned long long* h = reinterpret_cast<unsigned long long*>(c->h_pinned);
    int32_t* outside = reinterpret_cast<int32_t*>(h + 2);   // points whose label has no chunk
    DPMM_CUDA_TRY(cudaMemcpyAsync(h, c->d_prune_cnt, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                  c->stream));
    DPMM_CUDA_TRY(cudaMemcpyAsync(outside, c->d_aux + 8 + K, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaMemcpyAsync(outside + 1, d_err, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaMemcpyAsync(outside + 2, d_nlist, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (outside[1])
        return fail(DPMM_ERR_TIMEOUT, "tensor-core scan: bounded wait expired (code " + std::to_string(outside[1]) + ")");
    c->prune_tries += 1;
    const double extra = (double)h[0] / (double)c->N;   // kept other clusters per point
    c->prune_last_extra = extra;
    c->prune_last_over = (int64_t)h[1];
    // each kept cluster costs about one more exact r per point (FP32, in k_prune_draw).  Against the
    // SIMT dense phase that is the cheaper path up to about 2 per point; the tensor-core dense phase
    // costs about 1/30 of a kept cluster per point and cluster (N = 1e7, D = 64 on the B200: 0.21 ms
    // per cluster against 3-6 ms per kept cluster per point), so there the limit is K / 30.  Beyond
    // it run the dense phase, and wait before the next attempt
    const double limit = tc_dense ? (double)K / kPruneTcRatio : 2.0;
    if (extra > limit || *outside != 0) {
        c->prune_wait = 2;
        return DPMM_OK;
    }
    const RngArgs r = rng_args(c, d_u);
    const size_t sm = prune_draw_smem(DP, K);
    DPMM_CUDA_TRY(cudaFuncSetAttribute(k_prune_draw<DP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    {
        KernelTimer kt(c, PH_PRUNE_DRAW);
        k_prune_settle<<<c->max_chunks, 256, 0, c->stream>>>(c->d_perm, c->d_chunk, c->d_nchunks, c->d_prune_cand,
                                                             final_, r, c->d_labels);
        DPMM_LAUNCHED();
        const int nlist = outside[2];
        if (nlist > 0) {
            const dim3 grid((unsigned)nlist, (unsigned)((c->chunk_len + kPrTh - 1) / kPrTh));
            k_prune_draw<DP><<<grid, kPrTh, sm, c->stream>>>(c->d_x, c->d_perm, c->d_chunk, c->d_nchunks, c->d_Wt,
                                                            c->d_b, c->d_c, K, final_, r, c->d_prune_rh,
                                                            c->d_prune_cand, c->prune_margin, c->d_prune_list,
                                                            c->d_labels);
            DPMM_LAUNCHED();
        }
    }
    c->prune_used += 1;
    c->prune_extra += extra;
    *used = true;
    return DPMM_OK;
}

dpmm_status launch_cluster_labels_pruned(dpmm_ctx* c, int K, int final_, const float* d_u, bool* used)
{
    *used = false;
    if (c->prior != DPMM_PRIOR_GAUSSIAN || c->Dp > 64 || c->prune_margin <= 0 || K < 2 || K > kMaxKForPrune)
        return DPMM_OK;
    // below kMinKForPruneTc clusters the tensor-core dense phase costs less than the scan alone
    const bool tc_dense = c->ll_mode != DPMM_LL_FP32 && tc_supported(c, K);
    if (tc_dense && K < kMinKForPruneTc) return DPMM_OK;
    if (prune_draw_smem(c->Dp, K) > 220 * 1024) return DPMM_OK;
    if (c->prune_wait > 0) {
        --c->prune_wait;
        return DPMM_OK;
    }
    switch (c->Dp) {
        case 4: return launch_pruned_dp<4>(c, K, final_, d_u, tc_dense, used);
        case 8: return launch_pruned_dp<8>(c, K, final_, d_u, tc_dense, used);
        case 16: return launch_pruned_dp<16>(c, K, final_, d_u, tc_dense, used);
        case 32: return launch_pruned_dp<32>(c, K, final_, d_u, tc_dense, used);
        default: return launch_pruned_dp<64>(c, K, final_, d_u, tc_dense, used);
    }
}

// ----------------------------------------------------------------------------- permutation
// Stable counting sort of the points by label.  Bin K collects labels outside 1..K.
constexpr int kHistBlock = 2048;   // points per histogram block (256 threads x 8)

__device__ __forceinline__ int label_bin(int32_t lab, int K) { return (lab >= 1 && lab <= K) ? lab - 1 : K; }

__global__ void k_hist(const int32_t* __restrict__ labels, int64_t N, int K, int32_t* __restrict__ blk_hist)
{
    extern __shared__ int32_t sh[];
    for (int k = threadIdx.x; k <= K; k += blockDim.x) sh[k] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kHistBlock;
    for (int it = 0; it < kHistBlock / 256; ++it) {
        int64_t pt = base + it * 256 + threadIdx.x;
        if (pt < N) atomicAdd(&sh[label_bin(labels[pt], K)], 1);
    }
    __syncthreads();
    for (int k = threadIdx.x; k <= K; k += blockDim.x) blk_hist[(size_t)blockIdx.x * (K + 1) + k] = sh[k];
}

// one block per bin: exclusive scan over histogram blocks, in place; total into seg_tmp[k]
__global__ void k_scan_bins(int32_t* __restrict__ blk_hist, int nblk, int K, int32_t* __restrict__ total)
{
    const int k = blockIdx.x;
    __shared__ int32_t warp_sums[32];
    __shared__ int32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int b0 = 0; b0 < nblk; b0 += blockDim.x) {
        int b = b0 + threadIdx.x;
        int v = b < nblk ? blk_hist[(size_t)b * (K + 1) + k] : 0;
        // block-wide inclusive scan
        int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        int s = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += t;
        }
        if (lane == 31) warp_sums[w] = s;
        __syncthreads();
        if (w == 0) {
            int ws = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int t = __shfl_up_sync(0xffffffffu, ws, o);
                if (lane >= o) ws += t;
            }
            warp_sums[lane] = ws;
        }
        __syncthreads();
        int incl = s + (w > 0 ? warp_sums[w - 1] : 0);
        if (b < nblk) blk_hist[(size_t)b * (K + 1) + k] = carry + incl - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry += incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) total[k] = carry;
}

// single block: segment starts and the chunk table (cluster, start, len) of <= chunk_len points
__global__ void __launch_bounds__(1024) k_segments(const int32_t* __restrict__ total, int K,
                                                   int32_t* __restrict__ seg, int32_t* __restrict__ chunk,
                                                   int32_t* __restrict__ nchunks, int max_chunks, int chunk_len)
{
    // thread i takes bins [k0, k1); a block scan of the bins' point and chunk totals gives its offsets
    __shared__ int32_t s_t[1024], s_c[1024];
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int items = K + 1;   // cluster bins 0..K-1 and bin K (labels outside 1..K: no chunks)
    const int per = (items + nthr - 1) / nthr;
    const int k0 = min(items, tid * per), k1 = min(items, k0 + per);
    int32_t st = 0, sc = 0;
    for (int k = k0; k < k1; ++k) {
        const int32_t t = total[k];
        st += t;
        if (k < K) sc += (t + chunk_len - 1) / chunk_len;
    }
    s_t[tid] = st;
    s_c[tid] = sc;
    __syncthreads();
    for (int o = 1; o < nthr; o <<= 1) {   // inclusive scan
        const int32_t a = tid >= o ? s_t[tid - o] : 0, c = tid >= o ? s_c[tid - o] : 0;
        __syncthreads();
        s_t[tid] += a;
        s_c[tid] += c;
        __syncthreads();
    }
    int32_t acc = s_t[tid] - st, nc = s_c[tid] - sc;
    for (int k = k0; k < k1; ++k) {
        seg[k] = acc;
        const int32_t t = total[k];
        if (k < K)
            for (int32_t s = 0; s < t; s += chunk_len, ++nc)
                if (nc < max_chunks) {
                    chunk[3 * nc + 0] = k;
                    chunk[3 * nc + 1] = acc + s;
                    chunk[3 * nc + 2] = min(chunk_len, t - s);
                }
        acc += t;
    }
    if (tid == nthr - 1) {
        seg[K + 1] = s_t[nthr - 1];
        *nchunks = min(s_c[nthr - 1], max_chunks);
    }
}

__global__ void k_scatter(const int32_t* __restrict__ labels, int64_t N, int K, const int32_t* __restrict__ blk_off,
                          const int32_t* __restrict__ seg, int32_t* __restrict__ perm)
{
    extern __shared__ int32_t sh[];
    int32_t* run = sh;                 // K+1
    int32_t* wcnt = sh + (K + 1);      // 8 x (K+1)
    for (int k = threadIdx.x; k < 9 * (K + 1); k += blockDim.x) sh[k] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const int64_t base = (int64_t)blockIdx.x * kHistBlock;
    for (int it = 0; it < kHistBlock / 256; ++it) {
        const int64_t pt = base + it * 256 + threadIdx.x;
        const int bin = pt < N ? label_bin(labels[pt], K) : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, bin);
        const int rank = __popc(peers & lt);
        if (rank == 0 && bin >= 0) wcnt[w * (K + 1) + bin] = __popc(peers);
        __syncthreads();
        if (bin >= 0) {
            int before = run[bin];
            for (int v = 0; v < w; ++v) before += wcnt[v * (K + 1) + bin];
            perm[seg[bin] + blk_off[(size_t)blockIdx.x * (K + 1) + bin] + before + rank] = (int32_t)pt;
        }
        __syncthreads();
        if (rank == 0 && bin >= 0) {
            atomicAdd(&run[bin], __popc(peers));
            wcnt[w * (K + 1) + bin] = 0;
        }
        __syncthreads();
    }
}

dpmm_status build_permutation(dpmm_ctx* c, int K)
{
    const int nblk = blocks_for(c->N, kHistBlock);
    if (nblk > c->nblk_hist || K > c->k_max) return fail(DPMM_ERR_INVALID_ARG, "permutation capacity exceeded");
    k_hist<<<nblk, 256, sizeof(int32_t) * (K + 1), c->stream>>>(c->d_labels, c->N, K, c->d_blk_hist);
    DPMM_LAUNCHED();
    int32_t* total = c->d_aux + 8;   // K+1 entries
    k_scan_bins<<<K + 1, 1024, 0, c->stream>>>(c->d_blk_hist, nblk, K, total);
    DPMM_LAUNCHED();
    k_segments<<<1, 1024, 0, c->stream>>>(total, K, c->d_seg, c->d_chunk, c->d_nchunks, c->max_chunks,
                                         c->chunk_len);
    DPMM_LAUNCHED();
    size_t sm = sizeof(int32_t) * 9 * (K + 1);
    if (sm > 48 * 1024) DPMM_CUDA_TRY(cudaFuncSetAttribute(k_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_scatter<<<nblk, 256, sm, c->stream>>>(c->d_labels, c->N, K, c->d_blk_hist, c->d_seg, c->d_perm);
    DPMM_LAUNCHED();
    c->perm_K = K;
    return DPMM_OK;
}

// ----------------------------------------------------------------------------- sub-labels + stats

// Gaussian: one block per chunk of one cluster (points in permutation order).  Draws the
// sub-labels (unless draw == 0, in which case the current sub-labels are used) and accumulates
// per sub-cluster: count, sum(x - s) and the upper triangle of sum (x - s)(x - s)^T, shift
// s = the cluster's mean parameter.  FP32 products, FP32 runs of at most 33 points, FP64 totals.
//
// DP <= 64 ("blocked" form, 128 points per tile):
//   draw  - two threads per point, one per side: warps 0-3 evaluate the l factor, warps 4-7 the r
//           factor, x in registers, factor rows broadcast from shared memory as float4;
//   stats - each thread of a warp-aligned group owns one 4 x 4 block of the upper triangle and
//           does 16 FMAs per point from two float4 loads; G groups take every G-th point of the
//           tile; FP64 totals per thread live in shared memory and are summed over the groups at
//           the end.
// DP = 128: one thread per point for the draw, one matrix entry per thread through a pair table.

template <int DP>
struct SubStatsShape {
    static constexpr bool BLOCKED = DP <= 64;
    static constexpr int TP = 128;                                   // points per tile
    static constexpr int SX = DP + 4;                                // shared row stride (16-byte rows)
    static constexpr int NB = DP / 4;
    static constexpr int NBLK = NB * (NB + 1) / 2;                   // 4 x 4 blocks of the triangle
    static constexpr int GS = (NBLK + 31) / 32 * 32;                 // threads per group (whole warps)
    static constexpr int G = BLOCKED ? 256 / GS : 1;                 // groups
    static constexpr int NTOT = G * NBLK;                            // owners of FP64 totals
    // shared layout in bytes
    static constexpr size_t off_wl = 0;
    static constexpr size_t off_wr = off_wl + sizeof(float) * DP * DP;
    static constexpr size_t off_bl = off_wr + sizeof(float) * DP * DP;
    static constexpr size_t off_br = off_bl + sizeof(float) * DP;
    static constexpr size_t off_s = off_br + sizeof(float) * DP;
    static constexpr size_t off_x = (off_s + sizeof(float) * DP + 15) / 16 * 16;
    static constexpr size_t off_q = off_x + sizeof(float) * TP * SX;
    static constexpr size_t off_sub = off_q + sizeof(float) * 2 * TP;
    static constexpr size_t off_tail = (off_sub + sizeof(int32_t) * TP + 15) / 16 * 16;
    // blocked: FP64 block totals [32][NTOT] then sums [G][2][DP]; DP = 128: pair table
    static constexpr size_t off_tot = off_tail;
    static constexpr size_t off_sum = off_tot + (BLOCKED ? sizeof(double) * 32 * NTOT : 0);
    static constexpr size_t bytes = BLOCKED ? off_sum + sizeof(double) * G * 2 * DP
                                            : off_tail + sizeof(uint16_t) * tri(DP);
};

template <int DP>
__global__ void __launch_bounds__(256, (DP >= 128 ? 1 : 2)) k_gauss_sub_stats(
    const float* __restrict__ x, const int32_t* __restrict__ perm, const int32_t* __restrict__ chunk,
    const int32_t* __restrict__ nchunks, const float* __restrict__ Wt, const float* __restrict__ bvec,
    const float* __restrict__ cvec, const float* __restrict__ lrw, const float* __restrict__ muv, int draw,
    RngArgs rng, int32_t* __restrict__ sub, float* __restrict__ r_out, double* __restrict__ part,
    const uint8_t* __restrict__ mask)
{
    using S = SubStatsShape<DP>;
    constexpr int T = tri(DP);
    constexpr int SL = 1 + DP + T;            // partial record length per sub-cluster
    constexpr int TP = S::TP, SX = S::SX;
    constexpr int E = S::BLOCKED ? 1 : (T + 255) / 256;
    extern __shared__ __align__(16) unsigned char smem[];
    float* sWl = reinterpret_cast<float*>(smem + S::off_wl);
    float* sWr = reinterpret_cast<float*>(smem + S::off_wr);
    float* sbl = reinterpret_cast<float*>(smem + S::off_bl);
    float* sbr = reinterpret_cast<float*>(smem + S::off_br);
    float* ss = reinterpret_cast<float*>(smem + S::off_s);
    float* sx = reinterpret_cast<float*>(smem + S::off_x);
    float* sq = reinterpret_cast<float*>(smem + S::off_q);
    int32_t* ssub = reinterpret_cast<int32_t*>(smem + S::off_sub);
    double* stot = reinterpret_cast<double*>(smem + S::off_tot);
    double* ssum = reinterpret_cast<double*>(smem + S::off_sum);
    uint16_t* spair = reinterpret_cast<uint16_t*>(smem + S::off_tail);

    const int ch = blockIdx.x;
    if (ch >= *nchunks) return;
    const int k = chunk[3 * ch], start = chunk[3 * ch + 1], len = chunk[3 * ch + 2];
    if (mask && !mask[k]) return;
    const int tid = threadIdx.x;

    if (draw) {
        const float4* wl = reinterpret_cast<const float4*>(Wt + (size_t)(3 * k + 1) * DP * DP);
        const float4* wr = reinterpret_cast<const float4*>(Wt + (size_t)(3 * k + 2) * DP * DP);
        for (int e = tid; e < DP * DP / 4; e += 256) {
            reinterpret_cast<float4*>(sWl)[e] = wl[e];
            reinterpret_cast<float4*>(sWr)[e] = wr[e];
        }
        for (int e = tid; e < DP; e += 256) {
            sbl[e] = bvec[(size_t)(3 * k + 1) * DP + e];
            sbr[e] = bvec[(size_t)(3 * k + 2) * DP + e];
        }
    }
    for (int e = tid; e < DP; e += 256) ss[e] = muv[(size_t)(3 * k) * DP + e];
    if (draw) {
        // the points are staged centred on s = the cluster's mean: z = W^T (x - s) - b' with
        // b' = b - W^T s (thread j: row j of the l factor; thread DP + j: of the r factor)
        __syncthreads();
        if (tid < 2 * DP) {
            const int j = tid % DP;
            const float* wrow = (tid < DP ? sWl : sWr) + j * DP;
            float acc = 0.f;
            for (int i = 0; i < DP; ++i) acc = fmaf(wrow[i], ss[i], acc);
            (tid < DP ? sbl : sbr)[j] -= acc;
        }
    }
    if constexpr (!S::BLOCKED) {
        for (int e = tid; e < T; e += 256) {
            int i = 0, rem = e;
            while (rem >= DP - i) { rem -= DP - i; ++i; }
            spair[e] = (uint16_t)((i << 8) | (i + rem));
        }
    }
    const float cl = draw ? cvec[3 * k + 1] : 0.f, cr = draw ? cvec[3 * k + 2] : 0.f;
    const float wl = draw ? lrw[2 * k] : 0.f, wr = draw ? lrw[2 * k + 1] : 0.f;

    // blocked form: this thread's group, 4 x 4 block (bi <= bj) and FP64 total column
    const int grp = tid / S::GS, tb = tid % S::GS;
    const bool has_blk = S::BLOCKED && grp < S::G && tb < S::NBLK;
    int bi = 0, bj = 0;
    if (has_blk) {
        int rem = tb;
        while (rem >= S::NB - bi) { rem -= S::NB - bi; ++bi; }
        bj = bi + rem;
    }
    const bool diag = has_blk && bi == bj;
    const int tcol = grp * S::NBLK + tb;
    if constexpr (S::BLOCKED) {
        if (has_blk)
            for (int m = 0; m < 32; ++m) stot[m * S::NTOT + tcol] = 0.0;
        for (int e = tid; e < S::G * 2 * DP; e += 256) ssum[e] = 0.0;
    }
    float bf[2][16];
    float sf[2][4];
    float accf[2][E];
    double accd[2][E];
#pragma unroll
    for (int s2 = 0; s2 < 2; ++s2) {
#pragma unroll
        for (int m = 0; m < 16; ++m) bf[s2][m] = 0.f;
#pragma unroll
        for (int m = 0; m < 4; ++m) sf[s2][m] = 0.f;
#pragma unroll
        for (int m = 0; m < E; ++m) { accf[s2][m] = 0.f; accd[s2][m] = 0.0; }
    }
    float sumf = 0.f;     // DP = 128: threads [0, DP) -> l sums, [DP, 2DP) -> r sums
    double sumd = 0.0;
    int cnt_l = 0, cnt_r = 0;

    auto flush = [&]() {
        if constexpr (S::BLOCKED) {
            if (has_blk) {
#pragma unroll
                for (int s2 = 0; s2 < 2; ++s2)
#pragma unroll
                    for (int m = 0; m < 16; ++m) {
                        stot[(16 * s2 + m) * S::NTOT + tcol] += (double)bf[s2][m];
                        bf[s2][m] = 0.f;
                    }
                if (diag) {
#pragma unroll
                    for (int s2 = 0; s2 < 2; ++s2)
#pragma unroll
                        for (int a = 0; a < 4; ++a) {
                            ssum[(grp * 2 + s2) * DP + 4 * bi + a] += (double)sf[s2][a];
                            sf[s2][a] = 0.f;
                        }
                }
            }
        } else {
#pragma unroll
            for (int s2 = 0; s2 < 2; ++s2)
#pragma unroll
                for (int m = 0; m < E; ++m) { accd[s2][m] += (double)accf[s2][m]; accf[s2][m] = 0.f; }
            sumd += (double)sumf;
            sumf = 0.f;
        }
    };

    // tile staging: each thread holds NPF float4 of the next tile in registers, loaded while the
    // current tile's statistics accumulate, and stores them centred on s at the next tile's start
    constexpr int NV = TP * DP / 4;                 // float4 per tile
    constexpr int NPF = (NV + 255) / 256;
    float4 pf[NPF];
    auto load_tile = [&](int t0) {
        const int ntn = min(TP, len - t0);
#pragma unroll
        for (int u = 0; u < NPF; ++u) {
            const int e = tid + 256 * u;
            const int pp = e / (DP / 4), i4 = e % (DP / 4);
            pf[u] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (e < NV && pp < ntn)
                pf[u] = __ldg(reinterpret_cast<const float4*>(x + (size_t)__ldg(perm + start + t0 + pp) * DP) + i4);
        }
    };
    constexpr bool PREFETCH = DP <= 64;             // DP = 128: too many registers, load at the tile start
    if (PREFETCH) load_tile(0);
    for (int t0 = 0; t0 < len; t0 += TP) {
        const int nt = min(TP, len - t0);
        if (!PREFETCH) load_tile(t0);
        __syncthreads();
#pragma unroll
        for (int u = 0; u < NPF; ++u) {
            const int e = tid + 256 * u;
            if (e < NV) {
                const int pp = e / (DP / 4), i4 = e % (DP / 4);
                const float4 sv4 = *reinterpret_cast<const float4*>(ss + 4 * i4);
                float4 v = pf[u];
                if (pp < nt) { v.x -= sv4.x; v.y -= sv4.y; v.z -= sv4.z; v.w -= sv4.w; }
                *reinterpret_cast<float4*>(sx + pp * SX + 4 * i4) = v;
            }
        }
        __syncthreads();
        if (draw) {
            if constexpr (S::BLOCKED) {
                // quadratic form of one side for one point
                const int side = tid >> 7, pp = tid & 127;
                const float* W = side ? sWr : sWl;
                const float* bb = side ? sbr : sbl;
                float xr[DP];
#pragma unroll
                for (int i4 = 0; i4 < DP / 4; ++i4) {
                    const float4 v = *reinterpret_cast<const float4*>(sx + pp * SX + 4 * i4);
                    xr[4 * i4] = v.x; xr[4 * i4 + 1] = v.y; xr[4 * i4 + 2] = v.z; xr[4 * i4 + 3] = v.w;
                }
                float q0 = 0.f, q1 = 0.f;
#pragma unroll 2
                for (int j = 0; j < DP; j += 2) {
                    const float4* w0 = reinterpret_cast<const float4*>(W + j * DP);
                    const float4* w1 = reinterpret_cast<const float4*>(W + (j + 1) * DP);
                    float z0 = -bb[j], z1 = -bb[j + 1], z0b = 0.f, z1b = 0.f;
#pragma unroll
                    for (int i4 = 0; i4 < DP / 4; ++i4) {
                        const float4 a = w0[i4], c = w1[i4];
                        z0 = fmaf(a.x, xr[4 * i4 + 0], z0);
                        z1 = fmaf(c.x, xr[4 * i4 + 0], z1);
                        z0b = fmaf(a.y, xr[4 * i4 + 1], z0b);
                        z1b = fmaf(c.y, xr[4 * i4 + 1], z1b);
                        z0 = fmaf(a.z, xr[4 * i4 + 2], z0);
                        z1 = fmaf(c.z, xr[4 * i4 + 2], z1);
                        z0b = fmaf(a.w, xr[4 * i4 + 3], z0b);
                        z1b = fmaf(c.w, xr[4 * i4 + 3], z1b);
                    }
                    z0 += z0b;
                    z1 += z1b;
                    q0 = fmaf(z0, z0, q0);
                    q1 = fmaf(z1, z1, q1);
                }
                sq[side * TP + pp] = q0 + q1;
                __syncthreads();
            } else {
                if (tid < nt) {
                    const float* xp = sx + tid * SX;
                    float ql = 0.f, qr = 0.f;
                    for (int j = 0; j < DP; ++j) {
                        const float* wlp = sWl + j * DP;
                        const float* wrp = sWr + j * DP;
                        float zl = -sbl[j], zr = -sbr[j];
#pragma unroll 8
                        for (int i = 0; i < DP; ++i) {
                            float xv = xp[i];
                            zl = fmaf(wlp[i], xv, zl);
                            zr = fmaf(wrp[i], xv, zr);
                        }
                        ql = fmaf(zl, zl, ql);
                        qr = fmaf(zr, zr, qr);
                    }
                    sq[tid] = ql;
                    sq[TP + tid] = qr;
                }
            }
        }
        int sv = 0;
        if (tid < nt) {
            const int64_t pt = perm[start + t0 + tid];
            if (draw) {
                float rl = cl - 0.5f * sq[tid], rr = cr - 0.5f * sq[TP + tid];
                if (r_out) { r_out[2 * pt] = rl; r_out[2 * pt + 1] = rr; }
                // + log lr_weights, then the 2-way softmax (cudaKernel.cu:352-372)
                rl += wl;
                rr += wr;
                float mx = fmaxf(rl, rr);
                float el = __expf(rl - mx), er = __expf(rr - mx);
                float s = el + er;
                float u1, u2;
                draw_uniform2(rng, pt, u1, u2);
                sv = alias_draw2(el / s, er / s, u1, u2);
                sub[pt] = sv;
            } else {
                sv = sub[pt];
            }
            ssub[tid] = sv;
        }
        cnt_l += __syncthreads_count(sv == 1);
        cnt_r += __syncthreads_count(sv == 2);
        if (PREFETCH && t0 + TP < len) load_tile(t0 + TP);
        if constexpr (S::BLOCKED) {
            if (grp < S::G) {
                // two points per iteration: both points' loads issue before either's FMAs
                auto acc = [&](int sv2, const float4 xi, const float4 xj) {
                    const float vi[4] = {xi.x, xi.y, xi.z, xi.w};
                    const float vj[4] = {xj.x, xj.y, xj.z, xj.w};
                    if (sv2 == 1) {
#pragma unroll
                        for (int a = 0; a < 4; ++a)
#pragma unroll
                            for (int c = 0; c < 4; ++c) bf[0][4 * a + c] = fmaf(vi[a], vj[c], bf[0][4 * a + c]);
                        if (diag) {
#pragma unroll
                            for (int a = 0; a < 4; ++a) sf[0][a] += vi[a];
                        }
                    } else if (sv2 == 2) {
#pragma unroll
                        for (int a = 0; a < 4; ++a)
#pragma unroll
                            for (int c = 0; c < 4; ++c) bf[1][4 * a + c] = fmaf(vi[a], vj[c], bf[1][4 * a + c]);
                        if (diag) {
#pragma unroll
                            for (int a = 0; a < 4; ++a) sf[1][a] += vi[a];
                        }
                    }
                };
                int run = 0;
                for (int pp = grp; pp < nt; pp += 2 * S::G) {
                    const int pq = pp + S::G;
                    const int sa = ssub[pp];
                    const int sb2 = pq < nt ? ssub[pq] : 0;
                    if (has_blk) {
                        const float* xa = sx + pp * SX;
                        const float* xb = sx + (pq < nt ? pq : pp) * SX;
                        const float4 xia = *reinterpret_cast<const float4*>(xa + 4 * bi);
                        const float4 xja = *reinterpret_cast<const float4*>(xa + 4 * bj);
                        const float4 xib = *reinterpret_cast<const float4*>(xb + 4 * bi);
                        const float4 xjb = *reinterpret_cast<const float4*>(xb + 4 * bj);
                        acc(sa, xia, xja);
                        acc(sb2, xib, xjb);
                    }
                    run += ((sa == 1 || sa == 2) ? 1 : 0) + ((sb2 == 1 || sb2 == 2) ? 1 : 0);
                    if (run >= 32) { flush(); run = 0; }   // FP32 runs of at most 33 points
                }
            }
        } else {
            for (int pp = 0; pp < nt; ++pp) {
                const int sv2 = ssub[pp];
                if (sv2 != 1 && sv2 != 2) continue;
                const float* xp = sx + pp * SX;
                const int slot = sv2 - 1;
#pragma unroll
                for (int m = 0; m < E; ++m) {
                    int e = tid + 256 * m;
                    if (e < T) {
                        uint16_t pr = spair[e];
                        int i = pr >> 8, j = pr & 0xff;
                        if (slot == 0) accf[0][m] = fmaf(xp[i], xp[j], accf[0][m]);
                        else accf[1][m] = fmaf(xp[i], xp[j], accf[1][m]);
                    }
                }
                if (slot == 0 && tid < DP) sumf += xp[tid];
                if (slot == 1 && tid >= DP && tid < 2 * DP) sumf += xp[tid - DP];
                if ((pp & 31) == 31) flush();
            }
        }
        flush();
    }
    double* pl = part + (size_t)ch * 2 * SL;
    double* pr = pl + SL;
    if (tid == 0) { pl[0] = (double)cnt_l; pr[0] = (double)cnt_r; }
    if constexpr (S::BLOCKED) {
        __syncthreads();
        // sum the groups' FP64 totals; thread b < NBLK writes block b
        if (tid < S::NBLK) {
            int ri = 0, rem = tid;
            while (rem >= S::NB - ri) { rem -= S::NB - ri; ++ri; }
            const int rj = ri + rem;
#pragma unroll 1
            for (int s2 = 0; s2 < 2; ++s2) {
                double* po = s2 ? pr : pl;
                for (int m = 0; m < 16; ++m) {
                    const int i = 4 * ri + (m >> 2), j = 4 * rj + (m & 3);
                    if (i > j) continue;
                    double v = 0.0;
                    for (int g = 0; g < S::G; ++g) v += stot[(16 * s2 + m) * S::NTOT + g * S::NBLK + tid];
                    po[1 + DP + tri_index(DP, i, j)] = v;
                }
            }
        }
        for (int e = tid; e < 2 * DP; e += 256) {
            double v = 0.0;
            for (int g = 0; g < S::G; ++g) v += ssum[g * 2 * DP + e];
            (e < DP ? pl : pr)[1 + (e % DP)] = v;
        }
    } else {
        if (tid < DP) pl[1 + tid] = sumd;
        else if (tid < 2 * DP) pr[1 + tid - DP] = sumd;
#pragma unroll
        for (int m = 0; m < E; ++m) {
            int e = tid + 256 * m;
            if (e < T) { pl[1 + DP + e] = accd[0][m]; pr[1 + DP + e] = accd[1][m]; }
        }
    }
}

// Statistics only (the sub-labels are given), DP <= 64: one pass per sub-cluster over the
// chunk.  Per tile the points of the pass's sub-cluster are compacted into a list (warp
// ballots), so the accumulation loop has no per-point branch; each thread of a warp-aligned
// group owns a 4 x 4 block of the upper triangle (and the diagonal blocks the sums), adds FP32
// runs of at most 33 points into FP64 totals held in registers, and the groups' totals meet in
// shared memory once per pass.  Same partial records as k_gauss_sub_stats.
template <int DP>
struct SlotStatsShape {
    static constexpr int TP = 128;
    static constexpr int SX = DP + 4;
    static constexpr int NB = DP / 4;
    static constexpr int NBLK = NB * (NB + 1) / 2;
    static constexpr int GS = (NBLK + 31) / 32 * 32;
    static constexpr int G = 256 / GS;
    static constexpr int NTOT = G * NBLK;
    static constexpr size_t off_s = 0;                                           // DP floats (shift)
    static constexpr size_t off_x = (off_s + sizeof(float) * DP + 15) / 16 * 16; // TP x SX floats
    static constexpr size_t off_list = off_x + sizeof(float) * TP * SX;          // TP ints
    static constexpr size_t off_wc = off_list + sizeof(int32_t) * TP;             // 8 warp counts
    static constexpr size_t off_tot = (off_wc + sizeof(int32_t) * 8 + 15) / 16 * 16;   // [20][NTOT] doubles
    static constexpr size_t bytes = off_tot + sizeof(double) * 20 * NTOT;
};

template <int DP>
__global__ void __launch_bounds__(256, 2) k_gauss_slot_stats(
    const float* __restrict__ x, const int32_t* __restrict__ perm, const int32_t* __restrict__ chunk,
    const int32_t* __restrict__ nchunks, const float* __restrict__ muv, const int32_t* __restrict__ sub,
    double* __restrict__ part, const uint8_t* __restrict__ mask)
{
    using S = SlotStatsShape<DP>;
    constexpr int T = tri(DP);
    constexpr int SL = 1 + DP + T;
    constexpr int TP = S::TP, SX = S::SX;
    constexpr int NV = TP * DP / 4;
    constexpr int NPF = (NV + 255) / 256;
    extern __shared__ __align__(16) unsigned char smem[];
    float* ss = reinterpret_cast<float*>(smem + S::off_s);
    float* sx = reinterpret_cast<float*>(smem + S::off_x);
    int32_t* slist = reinterpret_cast<int32_t*>(smem + S::off_list);
    int32_t* swc = reinterpret_cast<int32_t*>(smem + S::off_wc);
    double* stot = reinterpret_cast<double*>(smem + S::off_tot);

    const int ch = blockIdx.x;
    if (ch >= *nchunks) return;
    const int k = chunk[3 * ch], start = chunk[3 * ch + 1], len = chunk[3 * ch + 2];
    if (mask && !mask[k]) return;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int e = tid; e < DP; e += 256) ss[e] = muv[(size_t)(3 * k) * DP + e];

    const int grp = tid / S::GS, tb = tid % S::GS;
    const bool has_blk = grp < S::G && tb < S::NBLK;
    int bi = 0, bj = 0;
    if (has_blk) {
        int rem = tb;
        while (rem >= S::NB - bi) { rem -= S::NB - bi; ++bi; }
        bj = bi + rem;
    }
    const bool diag = has_blk && bi == bj;
    const int tcol = grp * S::NBLK + tb;
    double* out = part + (size_t)ch * 2 * SL;

    float4 pf[NPF];
    int pfs = 0;   // this thread's point's sub-label (threads < TP)
    auto load_tile = [&](int t0) {
        const int ntn = min(TP, len - t0);
#pragma unroll
        for (int u = 0; u < NPF; ++u) {
            const int e = tid + 256 * u;
            const int pp = e / (DP / 4), i4 = e % (DP / 4);
            pf[u] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (e < NV && pp < ntn)
                pf[u] = __ldg(reinterpret_cast<const float4*>(x + (size_t)__ldg(perm + start + t0 + pp) * DP) + i4);
        }
        pfs = tid < ntn ? __ldg(sub + __ldg(perm + start + t0 + tid)) : 0;
    };

    for (int slot = 1; slot <= 2; ++slot) {
        float bf[16], sf[4];
        double bd[16], sd[4];
#pragma unroll
        for (int m = 0; m < 16; ++m) { bf[m] = 0.f; bd[m] = 0.0; }
#pragma unroll
        for (int m = 0; m < 4; ++m) { sf[m] = 0.f; sd[m] = 0.0; }
        auto flush = [&]() {
#pragma unroll
            for (int m = 0; m < 16; ++m) { bd[m] += (double)bf[m]; bf[m] = 0.f; }
#pragma unroll
            for (int m = 0; m < 4; ++m) { sd[m] += (double)sf[m]; sf[m] = 0.f; }
        };
        int cnt = 0;
        __syncthreads();   // ss written / the previous pass's totals read
        load_tile(0);
        for (int t0 = 0; t0 < len; t0 += TP) {
            const int nt = min(TP, len - t0);
            __syncthreads();   // the previous tile's list and rows are no longer read
#pragma unroll
            for (int u = 0; u < NPF; ++u) {
                const int e = tid + 256 * u;
                if (e < NV) {
                    const int pp = e / (DP / 4), i4 = e % (DP / 4);
                    const float4 sv4 = *reinterpret_cast<const float4*>(ss + 4 * i4);
                    float4 v = pf[u];
                    if (pp < nt) { v.x -= sv4.x; v.y -= sv4.y; v.z -= sv4.z; v.w -= sv4.w; }
                    *reinterpret_cast<float4*>(sx + pp * SX + 4 * i4) = v;
                }
            }
            // list of this tile's points in the pass's sub-cluster, in order
            const bool in = tid < nt && pfs == slot;
            const unsigned bal = __ballot_sync(0xffffffffu, in);
            if (lane == 0 && warp < TP / 32) swc[warp] = __popc(bal);
            __syncthreads();
            int off = 0, n_in = 0;
#pragma unroll
            for (int w = 0; w < TP / 32; ++w) {
                const int c = swc[w];
                off += w < warp ? c : 0;
                n_in += c;
            }
            if (in) slist[off + __popc(bal & ((1u << lane) - 1u))] = tid;
            __syncthreads();
            cnt += n_in;
            if (t0 + TP < len) load_tile(t0 + TP);   // the next tile loads during the accumulation
            if (has_blk) {
                auto acc = [&](const float4 xi, const float4 xj) {
                    const float vi[4] = {xi.x, xi.y, xi.z, xi.w};
                    const float vj[4] = {xj.x, xj.y, xj.z, xj.w};
#pragma unroll
                    for (int a = 0; a < 4; ++a)
#pragma unroll
                        for (int c = 0; c < 4; ++c) bf[4 * a + c] = fmaf(vi[a], vj[c], bf[4 * a + c]);
                    if (diag) {
#pragma unroll
                        for (int a = 0; a < 4; ++a) sf[a] += vi[a];
                    }
                };
                // two points per iteration: both points' loads are in flight together
                int run = 0, q = grp;
                for (; q + S::G < n_in; q += 2 * S::G) {
                    const float* xa = sx + slist[q] * SX;
                    const float* xb = sx + slist[q + S::G] * SX;
                    const float4 xia = *reinterpret_cast<const float4*>(xa + 4 * bi);
                    const float4 xja = *reinterpret_cast<const float4*>(xa + 4 * bj);
                    const float4 xib = *reinterpret_cast<const float4*>(xb + 4 * bi);
                    const float4 xjb = *reinterpret_cast<const float4*>(xb + 4 * bj);
                    acc(xia, xja);
                    acc(xib, xjb);
                    run += 2;
                    if (run >= 32) { flush(); run = 0; }   // FP32 runs of at most 33 points
                }
                if (q < n_in) {
                    const float* xa = sx + slist[q] * SX;
                    acc(*reinterpret_cast<const float4*>(xa + 4 * bi), *reinterpret_cast<const float4*>(xa + 4 * bj));
                }
                flush();
            }
        }
        // the groups' totals meet in shared memory; thread b < NBLK writes block b
        if (has_blk) {
#pragma unroll
            for (int m = 0; m < 16; ++m) stot[m * S::NTOT + tcol] = bd[m];
#pragma unroll
            for (int m = 0; m < 4; ++m) stot[(16 + m) * S::NTOT + tcol] = sd[m];
        }
        __syncthreads();
        double* po = out + (size_t)(slot - 1) * SL;
        if (tid == 0) po[0] = (double)cnt;
        if (tid < S::NBLK) {
            int ri = 0, rem = tid;
            while (rem >= S::NB - ri) { rem -= S::NB - ri; ++ri; }
            const int rj = ri + rem;
            for (int m = 0; m < 16; ++m) {
                const int i = 4 * ri + (m >> 2), j = 4 * rj + (m & 3);
                if (i > j) continue;
                double v = 0.0;
                for (int g = 0; g < S::G; ++g) v += stot[m * S::NTOT + g * S::NBLK + tid];
                po[1 + DP + tri_index(DP, i, j)] = v;
            }
            if (ri == rj)
                for (int a = 0; a < 4; ++a) {
                    double v = 0.0;
                    for (int g = 0; g < S::G; ++g) v += stot[(16 + a) * S::NTOT + g * S::NBLK + tid];
                    po[1 + 4 * ri + a] = v;
                }
        }
    }
}

// Multinomial: warp per point; sub-label from two dot products with log theta_l / log theta_r,
// count sums accumulated with shared-memory float atomics (exact for integer counts while a
// chunk's per-category sum stays below 2^24).
__global__ void __launch_bounds__(256) k_mult_sub_stats(
    const float* __restrict__ x, int Dp, const int32_t* __restrict__ perm, const int32_t* __restrict__ chunk,
    const int32_t* __restrict__ nchunks, const float* __restrict__ logtheta, const float* __restrict__ lrw, int draw,
    RngArgs rng, int32_t* __restrict__ sub, float* __restrict__ r_out, double* __restrict__ part, int SL,
    const uint8_t* __restrict__ mask)
{
    extern __shared__ __align__(16) unsigned char smem[];
    float* tl = reinterpret_cast<float*>(smem);   // Dp
    float* tr = tl + Dp;                          // Dp
    float* accl = tr + Dp;                        // Dp
    float* accr = accl + Dp;                      // Dp
    __shared__ int cnt[2];
    const int ch = blockIdx.x;
    if (ch >= *nchunks) return;
    const int k = chunk[3 * ch], start = chunk[3 * ch + 1], len = chunk[3 * ch + 2];
    if (mask && !mask[k]) return;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    for (int e = tid; e < Dp; e += 256) {
        tl[e] = logtheta[(size_t)(3 * k + 1) * Dp + e];
        tr[e] = logtheta[(size_t)(3 * k + 2) * Dp + e];
        accl[e] = 0.f;
        accr[e] = 0.f;
    }
    if (tid < 2) cnt[tid] = 0;
    __syncthreads();
    const float wl = lrw[2 * k], wr = lrw[2 * k + 1];
    for (int pp = w; pp < len; pp += 8) {
        const int64_t pt = perm[start + pp];
        const float* xp = x + (size_t)pt * Dp;
        int sv = 0;
        if (draw) {
            float dl = 0.f, dr = 0.f;
            for (int d = lane; d < Dp; d += 32) {
                float v = xp[d];
                dl = fmaf(v, tl[d], dl);
                dr = fmaf(v, tr[d], dr);
            }
#pragma unroll
            for (int o = 16; o; o >>= 1) {
                dl += __shfl_xor_sync(0xffffffffu, dl, o);
                dr += __shfl_xor_sync(0xffffffffu, dr, o);
            }
            if (lane == 0) {
                float rl = dl + wl, rr = dr + wr;
                if (r_out) { r_out[2 * pt] = dl; r_out[2 * pt + 1] = dr; }
                float mx = fmaxf(rl, rr);
                float el = __expf(rl - mx), er = __expf(rr - mx);
                float s = el + er;
                float u1, u2;
                draw_uniform2(rng, pt, u1, u2);
                sv = alias_draw2(el / s, er / s, u1, u2);
                sub[pt] = sv;
            }
            sv = __shfl_sync(0xffffffffu, lane == 0 ? sv : 0, 0);
        } else {
            sv = sub[pt];
        }
        if (sv == 1 || sv == 2) {
            float* acc = sv == 1 ? accl : accr;
            for (int d = lane; d < Dp; d += 32) atomicAdd(&acc[d], xp[d]);
            if (lane == 0) atomicAdd(&cnt[sv - 1], 1);
        }
    }
    __syncthreads();
    double* pl = part + (size_t)ch * 2 * SL;
    double* pr = pl + SL;
    if (tid == 0) { pl[0] = cnt[0]; pr[0] = cnt[1]; }
    for (int e = tid; e < Dp; e += 256) { pl[1 + e] = accl[e]; pr[1 + e] = accr[e]; }
}

template <int DP>
static dpmm_status launch_gauss_sub_stats_t(dpmm_ctx* c, int draw, RngArgs r, float* d_rout, const uint8_t* d_mask)
{
    if constexpr (DP <= 64) {
        if (!draw && tc_stats_supported(c)) return launch_slot_stats_tc(c, d_mask);
        if (!draw) {
            const size_t sm = SlotStatsShape<DP>::bytes;
            auto kern = k_gauss_slot_stats<DP>;
            DPMM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            KernelTimer kt(d_mask ? nullptr : c, PH_SLOT_STATS);   // full launches only (masked: a few clusters)
            kern<<<c->max_chunks, 256, sm, c->stream>>>(c->d_x, c->d_perm, c->d_chunk, c->d_nchunks, c->d_mu,
                                                        c->d_sub, c->d_part, d_mask);
            DPMM_LAUNCHED();
            return DPMM_OK;
        }
    }
    const size_t sm = SubStatsShape<DP>::bytes;
    auto kern = k_gauss_sub_stats<DP>;
    DPMM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    kern<<<c->max_chunks, 256, sm, c->stream>>>(c->d_x, c->d_perm, c->d_chunk, c->d_nchunks, c->d_Wt, c->d_b, c->d_c,
                                                c->d_lrw, c->d_mu, draw, r, c->d_sub, d_rout, c->d_part, d_mask);
    DPMM_LAUNCHED();
    return DPMM_OK;
}

dpmm_status launch_sub_labels_and_stats(dpmm_ctx* c, int K, const float* d_u, float* d_rout, bool draw,
                                        const uint8_t* d_mask)
{
    if (c->perm_K != K) DPMM_TRY(build_permutation(c, K));
    RngArgs r = rng_args(c, d_u);
    if (draw && !d_mask && tc_sub_stats_supported(c)) {
        // sub-labels and their statistics in one pass over the points (one gather of each row)
        DPMM_TRY(launch_sub_stats_tc(c, r, d_rout));
        return launch_stats_finalize(c, K, d_mask);
    }
    if (draw && !d_mask && tc_sub_supported(c)) {
        // sub-labels on the tensor cores, then the statistics of the drawn sub-labels
        // its error word is read in the statistics launch's sync when that runs on the tensor cores
        DPMM_TRY(launch_sub_labels_tc(c, r, d_rout, c->prior == DPMM_PRIOR_GAUSSIAN && c->Dp <= 64 &&
                                                        tc_stats_supported(c)));
        draw = false;
    }
    if (c->prior == DPMM_PRIOR_GAUSSIAN) {
        switch (c->Dp) {
            case 4: DPMM_TRY(launch_gauss_sub_stats_t<4>(c, draw, r, d_rout, d_mask)); break;
            case 8: DPMM_TRY(launch_gauss_sub_stats_t<8>(c, draw, r, d_rout, d_mask)); break;
            case 16: DPMM_TRY(launch_gauss_sub_stats_t<16>(c, draw, r, d_rout, d_mask)); break;
            case 32: DPMM_TRY(launch_gauss_sub_stats_t<32>(c, draw, r, d_rout, d_mask)); break;
            case 64: DPMM_TRY(launch_gauss_sub_stats_t<64>(c, draw, r, d_rout, d_mask)); break;
            case 128: DPMM_TRY(launch_gauss_sub_stats_t<128>(c, draw, r, d_rout, d_mask)); break;
            default: return fail(DPMM_ERR_INVALID_ARG, "unsupported padded dimension");
        }
    } else {
        size_t sm = sizeof(float) * 4 * c->Dp;
        if (sm > 48 * 1024)
            DPMM_CUDA_TRY(cudaFuncSetAttribute(k_mult_sub_stats, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_mult_sub_stats<<<c->max_chunks, 256, sm, c->stream>>>(c->d_x, c->Dp, c->d_perm, c->d_chunk, c->d_nchunks,
                                                                 c->d_mu, c->d_lrw, draw ? 1 : 0, r, c->d_sub, d_rout,
                                                                 c->d_part, 1 + c->Dp, d_mask);
        DPMM_LAUNCHED();
    }
    return launch_stats_finalize(c, K, d_mask);
}

// Blocks (cluster, share of the scatter triangle): chunk partials summed in chunk order (FP64),
// shifted back to the original coordinates, written as count / sum / full S for slots 3k
// (cluster = l + r), 3k+1 (l), 3k+2 (r).
__global__ void k_stats_finalize(const double* __restrict__ part, const int32_t* __restrict__ chunk,
                                 const int32_t* __restrict__ nchunks, const float* __restrict__ muv,
                                 const double* __restrict__ gshift, int D, int Dp, int gauss, int SL, int out_len,
                                 double* __restrict__ stats, const uint8_t* __restrict__ mask)
{
    const int k = blockIdx.x;
    if (mask && !mask[k]) return;
    const int nc = *nchunks;
    // first chunk of this cluster (chunks are ordered by cluster)
    int lo = 0, hi = nc;
    while (lo < hi) {
        int mid = (lo + hi) / 2;
        if (chunk[3 * mid] < k) lo = mid + 1; else hi = mid;
    }
    const int c0 = lo;
    int c1 = c0;
    while (c1 < nc && chunk[3 * c1] == k) ++c1;
    const int T = gauss ? Dp * (Dp + 1) / 2 : 0;
    extern __shared__ double shd[];
    double* n2 = shd;                 // [2]
    double* sm2 = shd + 2;            // [2][D]
    double* t = sm2 + 2 * D;          // [D] total shift (gauss)
    for (int s = 0; s < 2; ++s) {
        for (int e = threadIdx.x; e < 1 + D; e += blockDim.x) {
            double acc = 0.0;
            for (int q = c0; q < c1; ++q) acc += part[((size_t)q * 2 + s) * SL + e];
            if (e == 0) n2[s] = acc; else sm2[s * D + e - 1] = acc;
        }
    }
    if (gauss)
        for (int e = threadIdx.x; e < D; e += blockDim.x) t[e] = (double)muv[(size_t)3 * k * Dp + e] + gshift[e];
    __syncthreads();
    double* out_c = stats + (size_t)(3 * k) * out_len;
    double* out_l = out_c + out_len;
    double* out_r = out_l + out_len;
    if (blockIdx.y == 0) {
        if (threadIdx.x == 0) {
            out_l[0] = n2[0];
            out_r[0] = n2[1];
            out_c[0] = n2[0] + n2[1];
        }
        for (int e = threadIdx.x; e < D; e += blockDim.x) {
            double sl = sm2[e], sr = sm2[D + e];
            if (gauss) { sl += n2[0] * t[e]; sr += n2[1] * t[e]; }
            out_l[1 + e] = sl;
            out_r[1 + e] = sr;
            out_c[1 + e] = sl + sr;
        }
    }
    if (!gauss) return;
    // S = Sc + t Sc_sum^T + Sc_sum t^T + n t t^T, with Sc_sum = sum (x - t); block y of the
    // cluster takes the y-th share of the upper triangle
    const int per = (T + (int)gridDim.y - 1) / (int)gridDim.y;
    const int e1 = min(T, per * ((int)blockIdx.y + 1));
    for (int e = per * (int)blockIdx.y + threadIdx.x; e < e1; e += blockDim.x) {
        int i = 0, rem = e;
        while (rem >= Dp - i) { rem -= Dp - i; ++i; }
        int j = i + rem;
        if (i >= D || j >= D) continue;
        double v[2];
        for (int s = 0; s < 2; ++s) {
            double acc = 0.0;
            for (int q = c0; q < c1; ++q) acc += part[((size_t)q * 2 + s) * SL + 1 + Dp + e];
            double si = sm2[s * D + i], sj = sm2[s * D + j];
            v[s] = acc + t[i] * sj + si * t[j] + n2[s] * t[i] * t[j];
        }
        size_t ij = 1 + D + (size_t)j * D + i, ji = 1 + D + (size_t)i * D + j;
        out_l[ij] = v[0]; out_l[ji] = v[0];
        out_r[ij] = v[1]; out_r[ji] = v[1];
        out_c[ij] = v[0] + v[1]; out_c[ji] = v[0] + v[1];
    }
}

// masked cluster slots between the statistics and the exchange buffer: to_stats = 0 copies
// src -> dst with zeros in the clusters the mask leaves out; to_stats = 1 copies back the masked ones
__global__ void k_masked_slots(const double* __restrict__ src, double* __restrict__ dst, int64_t n, int per_cluster,
                               const uint8_t* __restrict__ mask, int to_stats)
{
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool on = mask[i / per_cluster] != 0;
    if (to_stats) {
        if (on) dst[i] = src[i];
    } else {
        dst[i] = on ? src[i] : 0.0;
    }
}

dpmm_status launch_stats_finalize(dpmm_ctx* c, int K, const uint8_t* d_mask)
{
    const int gauss = c->prior == DPMM_PRIOR_GAUSSIAN;
    const int SL = gauss ? 1 + c->Dp + tri(c->Dp) : 1 + c->Dp;
    size_t sm = sizeof(double) * (2 + 3 * (size_t)c->D);
    if (sm > 48 * 1024)
        DPMM_CUDA_TRY(cudaFuncSetAttribute(k_stats_finalize, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    const dim3 grid((unsigned)K, gauss ? 8u : 1u);   // the scatter triangle over 8 blocks per cluster
    k_stats_finalize<<<grid, 256, sm, c->stream>>>(c->d_part, c->d_chunk, c->d_nchunks, c->d_mu, c->d_gshift, c->D,
                                                c->Dp, gauss, SL, c->stat_len, c->d_stats, d_mask);
    DPMM_LAUNCHED();
    if (c->shard_world > 1) {
        // this shard's statistics of the slots just finalised -> the sums over all shards.  With a
        // mask only those slots: the others already hold the sums (and the same bookkeeping on every rank)
        const int64_t n = (int64_t)3 * K * c->stat_len;
        if (!d_mask) {
            DPMM_TRY(shard_allreduce(c, c->d_stats, n));
        } else {
            k_masked_slots<<<blocks_for(n, 256), 256, 0, c->stream>>>(c->d_stats, c->d_xchg, n, 3 * c->stat_len, d_mask, 0);
            DPMM_LAUNCHED();
            DPMM_TRY(shard_allreduce(c, c->d_xchg, n));
            k_masked_slots<<<blocks_for(n, 256), 256, 0, c->stream>>>(c->d_xchg, c->d_stats, n, 3 * c->stat_len, d_mask, 1);
            DPMM_LAUNCHED();
        }
    }
    if (!d_mask) {
        c->stats_K = K;
        std::fill(c->stats_ok.begin(), c->stats_ok.end(), 0);
        std::fill(c->stats_ok.begin(), c->stats_ok.begin() + K, 1);
    }
    return DPMM_OK;
}

// ----------------------------------------------------------------------------- relabels
// mode 0 split:  table[l] = new 1-based label (0: not split); sub==2 moves; fresh sub-label
// mode 1 merge:  table[l] = 1: becomes sub 1;  table[l] = -m (m = 1-based target): sub 2, label m
// mode 2 reset:  table[l] != 0: fresh sub-label
// mode 3 remap:  label = table[label]
__global__ void k_relabel(int mode, int64_t N, int tlen, const int32_t* __restrict__ table, RngArgs rng,
                          const uint32_t* __restrict__ bits, int32_t* __restrict__ labels, int32_t* __restrict__ sub)
{
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    int lab = labels[i];
    if (lab < 0 || lab >= tlen) return;
    int t = table[lab];
    switch (mode) {
        case 0:
            if (t != 0) {
                if (sub[i] == 2) labels[i] = t;
                sub[i] = (int)(draw_bits(rng, bits, i) % 2u + 1u);   // cudaKernel.cu:202-212
            }
            break;
        case 1:
            if (t == 1) sub[i] = 1;                                  // cudaKernel.cu:223-237
            else if (t < 0) { sub[i] = 2; labels[i] = -t; }
            break;
        case 2:
            if (t != 0) sub[i] = (int)(draw_bits(rng, bits, i) % 2u + 1u);   // cudaKernel.cu:248-254
            break;
        default:
            labels[i] = t;                                           // cudaKernel.cu:172-178
    }
}

dpmm_status launch_relabel(dpmm_ctx* c, int mode, int K, const int32_t* h_table, int tlen, const uint32_t* d_bits)
{
    (void)K;
    if (tlen > c->k_max + 2) return fail(DPMM_ERR_INVALID_ARG, "relabel table larger than capacity");
    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_remap, h_table, sizeof(int32_t) * tlen, cudaMemcpyHostToDevice, c->stream));
    RngArgs r = rng_args(c, nullptr);
    k_relabel<<<blocks_for(c->N, 256), 256, 0, c->stream>>>(mode, c->N, tlen, c->d_remap, r, d_bits, c->d_labels,
                                                             c->d_sub);
    DPMM_LAUNCHED();
    if (mode != 2) c->perm_K = -1;   // a reset changes sub-labels only
    return DPMM_OK;
}

__global__ void k_sub_count(const int32_t* __restrict__ sub, int64_t N, int32_t* __restrict__ out)
{
    int a = 0, b = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        int s = sub[i];
        a += s == 1;
        b += s == 2;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&out[0], a);
        atomicAdd(&out[1], b);
    }
}

dpmm_status launch_sub_count(dpmm_ctx* c, int32_t* h_l, int32_t* h_r)
{
    DPMM_CUDA_TRY(cudaMemsetAsync(c->d_aux, 0, 2 * sizeof(int32_t), c->stream));
    k_sub_count<<<148 * 4, 256, 0, c->stream>>>(c->d_sub, c->N, c->d_aux);
    DPMM_LAUNCHED();
    int32_t h[2];
    DPMM_CUDA_TRY(cudaMemcpyAsync(h, c->d_aux, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (c->shard_world > 1) {   // counts of the whole data set
        double v[2] = {(double)h[0], (double)h[1]};
        DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_xchg, v, sizeof(v), cudaMemcpyHostToDevice, c->stream));
        DPMM_TRY(shard_allreduce(c, c->d_xchg, 2));
        DPMM_CUDA_TRY(cudaMemcpyAsync(v, c->d_xchg, sizeof(v), cudaMemcpyDeviceToHost, c->stream));
        DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
        h[0] = (int32_t)v[0];
        h[1] = (int32_t)v[1];
    }
    *h_l = h[0];
    *h_r = h[1];
    return DPMM_OK;
}

// ----------------------------------------------------------------------------- FP64 test seams
// cudaKernel_gaussian::log_likelihood_labels for one cluster in FP64 (parameters in d_dbl_scratch:
// mu[D], inv_sigma[D*D] col-major, scalar, log weight)
__global__ void k_loglik_gauss_one(const float* __restrict__ x, int64_t N, int D, int Dp, const double* __restrict__ gshift,
                                   const double* __restrict__ prm, double* __restrict__ r)
{
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= N) return;
    const double* mu = prm;
    const double* is = prm + D;
    const double scalar = prm[D + D * D], logw = prm[D + D * D + 1];
    double z[kMaxGaussDim];
    for (int j = 0; j < D; ++j) z[j] = ((double)x[p * Dp + j] + gshift[j]) - mu[j];
    double sum = 0;
    for (int i = 0; i < D; ++i) {
        double cc = 0;
        for (int j = 0; j < D; ++j) cc += is[(size_t)j * D + i] * z[j];
        sum += z[i] * cc;
    }
    r[p] = scalar - sum / 2 + logw;
}

dpmm_status launch_loglik_gauss_one(dpmm_ctx* c, double* d_r)
{
    k_loglik_gauss_one<<<blocks_for(c->N, 128), 128, 0, c->stream>>>(c->d_x, c->N, c->D, c->Dp, c->d_gshift,
                                                                     c->d_dbl_scratch, d_r);
    DPMM_LAUNCHED();
    return DPMM_OK;
}

__global__ void k_loglik_mult_one(const float* __restrict__ x, int64_t N, int D, int Dp, const double* __restrict__ lt,
                                  double* __restrict__ r)
{
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= N) return;
    double sum = 0;
    for (int i = 0; i < D; ++i) sum += lt[i] * (double)x[p * Dp + i];
    r[p] = sum;
}

dpmm_status launch_loglik_mult_one(dpmm_ctx* c, double* d_r)
{
    k_loglik_mult_one<<<blocks_for(c->N, 128), 128, 0, c->stream>>>(c->d_x, c->N, c->D, c->Dp, c->d_dbl_scratch, d_r);
    DPMM_LAUNCHED();
    return DPMM_OK;
}

constexpr int kSeamMaxK = 64;

// cudaKernel::sample_log_cat_array on a caller matrix (FP64 softmax + alias, as the reference)
__global__ void k_sample_log_cat(const double* __restrict__ r, int64_t N, int K, RngArgs rng, int32_t* __restrict__ labels)
{
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= N) return;
    double y[kSeamMaxK + 2];
    int32_t a[kSeamMaxK + 2], b[kSeamMaxK + 2];
    double mx = 0;
    bool first = true;
    for (int k = 0; k < K; ++k) {
        double v = r[(size_t)k * N + p];
        if (first || v > mx) { first = false; mx = v; }
    }
    double sum = 0;
    for (int k = 0; k < K; ++k) { y[k + 1] = exp(r[(size_t)k * N + p] - mx); sum += y[k + 1]; }
    for (int k = 0; k < K; ++k) y[k + 1] = (y[k + 1] / sum) * K;
    float u1, u2;
    draw_uniform2(rng, p, u1, u2);
    AliasAcc<double, int32_t> acc{y, a, b, 1};
    labels[p] = alias_draw<double, int32_t>(K, acc, u1, u2);
}

dpmm_status launch_sample_log_cat(dpmm_ctx* c, int K, const double* d_r, const float* d_u)
{
    if (K > kSeamMaxK) return fail(DPMM_ERR_INVALID_ARG, "sample_log_cat_array seam supports K <= 64");
    RngArgs r = rng_args(c, d_u);
    k_sample_log_cat<<<blocks_for(c->N, 128), 128, 0, c->stream>>>(d_r, c->N, K, r, c->d_labels);
    DPMM_LAUNCHED();
    return DPMM_OK;
}

// cudaKernel::sample_log_cat_array_sub_cluster: m points given by indices, log-likelihoods m x 2
__global__ void k_sample_log_cat_sub(const double* __restrict__ r, int m, const int32_t* __restrict__ idx,
                                     const double* __restrict__ lrw, RngArgs rng, int64_t N, int32_t* __restrict__ sub)
{
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= m) return;
    int64_t pt = idx[q];
    if (pt < 0 || pt >= N) return;
    double a = r[q] + log(lrw[0]);
    double b = r[q + m] + log(lrw[1]);
    double mx = fmax(a, b);
    a = exp(a - mx);
    b = exp(b - mx);
    double s = a + b;
    double y[4];
    int32_t aa[4], bb[4];
    y[1] = (a / s) * 2;
    y[2] = (b / s) * 2;
    float u1, u2;
    draw_uniform2(rng, pt, u1, u2);
    AliasAcc<double, int32_t> acc{y, aa, bb, 1};
    sub[pt] = alias_draw<double, int32_t>(2, acc, u1, u2);
}

dpmm_status launch_sample_log_cat_sub(dpmm_ctx* c, int m, const double* d_r, const int32_t* d_idx, const double* d_lrw,
                                      const float* d_u)
{
    RngArgs r = rng_args(c, d_u);
    k_sample_log_cat_sub<<<blocks_for(m, 128), 128, 0, c->stream>>>(d_r, m, d_idx, d_lrw, r, c->N, c->d_sub);
    DPMM_LAUNCHED();
    return DPMM_OK;
}

}  // namespace dpmm

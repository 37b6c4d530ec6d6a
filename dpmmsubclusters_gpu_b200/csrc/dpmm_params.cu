// dpmm_params.cu -- cluster parameter draws on the device (NIW prior) and the bookkeeping that keeps
// the device statistics equal to the host's between the statistics phase and the next draw.
//
//   k_draw_niw<DP>     niw::sample_distribution (niw.cpp:82-107) for every statistics slot, as
//                      shared_actions::sample_cluster_params (shared_actions.cpp:9-55) calls it for a
//                      cluster and its two sub-clusters: posterior (niw.cpp:23-49) from the slot's
//                      statistics, precision factor W = (nu' psi')^-T/2 A with A the Bartlett factor
//                      (A_ii = sqrt(chi2(nu' - i)), A_ij ~ N(0, 1) below the diagonal: the draw of
//                      stats::rinvwish2 in factor form), log det Sigma = log det(nu' psi') - 2 sum log
//                      A_ii, mu = m' + L_B A^-T z / sqrt(kappa'), z ~ N(0, I).  The results are written
//                      straight into the label-phase parameters (Wt, b, c, mu - shift), and the slot's
//                      log marginal likelihood (niw.cpp:122-138) is returned for the splittable test.
//   k_merge_stats      merge_clusters_to_splittable (shared_actions.cpp:72-86) on the statistics: the
//                      merged cluster and its l sub-cluster take c_i + c_j, its r sub-cluster c_j
//   k_compact_stats    remove_empty_clusters (local_clusters_actions.cpp:384-419): slot compaction
//
// Random variates: Philox4x32-10 keyed by the run seed, counter (element, slot, draw); normals by
// Box-Muller; chi-square(k) as 2 Gamma(k/2) by Marsaglia & Tsang (ACM TOMS 26(3), 2000), with
// Gamma(a) = Gamma(a + 1) U^(1/a) for a < 1 and at most 64 attempts (then the Wilson-Hilferty
// approximation, which at the degrees of freedom met here is far inside sampling noise).
#include <math.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "dpmm_device.cuh"
#include "dpmm_internal.h"
#include "dpmm_niw.cuh"

namespace dpmm {

// Philox block for (element e, slot s) of draw `draw`
__device__ __forceinline__ Philox4 param_bits(uint64_t seed, uint64_t draw, uint32_t e, uint32_t s)
{
    return philox4x32_10(e, s, (uint32_t)draw, (uint32_t)(draw >> 32) ^ 0xA5A5A5A5u, (uint32_t)seed,
                         (uint32_t)(seed >> 32));
}

// 64 random bits -> double in (0, 1]
__device__ __forceinline__ double u01_53(uint32_t hi, uint32_t lo)
{
    const uint64_t x = (((uint64_t)hi << 32) | lo) >> 11;
    return (double)(x + 1) * (1.0 / 9007199254740992.0);
}

// one standard normal from a Philox block (Box-Muller on its first two 64-bit halves)
__device__ __forceinline__ double normal_from(const Philox4& b)
{
    const double u1 = u01_53(b.v[0], b.v[1]), u2 = u01_53(b.v[2], b.v[3]);
    double sn, cs;
    sincospi(2.0 * u2, &sn, &cs);
    return sqrt(-2.0 * log(u1)) * cs;
}

// chi-square with k > 0 degrees of freedom for diagonal element i
__device__ double chi2_draw(double k, uint64_t seed, uint64_t draw, uint32_t s, uint32_t ebase)
{
    const double a0 = 0.5 * k;
    const bool boost = a0 < 1.0;
    const double a = boost ? a0 + 1.0 : a0;
    const double d = a - 1.0 / 3.0, c = 1.0 / sqrt(9.0 * d);
    double g = -1.0;
    for (int r = 0; r < 64 && g < 0; ++r) {
        const Philox4 b = param_bits(seed, draw, ebase + 2 * r, s);
        const Philox4 b2 = param_bits(seed, draw, ebase + 2 * r + 1, s);
        const double x = normal_from(b);
        const double v1 = 1.0 + c * x;
        if (v1 <= 0) continue;
        const double v = v1 * v1 * v1;
        const double u = u01_53(b2.v[0], b2.v[1]);
        if (log(u) < 0.5 * x * x + d - d * v + d * log(v)) g = d * v;
    }
    if (g < 0) {   // Wilson-Hilferty
        const Philox4 b = param_bits(seed, draw, ebase + 200, s);
        const double z = normal_from(b), h = 2.0 / (9.0 * k);
        const double w = 1.0 - h + z * sqrt(h);
        return fmax(k * w * w * w, 1e-300);
    }
    if (boost) {
        const Philox4 b = param_bits(seed, draw, ebase + 201, s);
        g *= pow(u01_53(b.v[0], b.v[1]), 1.0 / a0);
    }
    return 2.0 * g;
}

// element ids of the random streams of one slot: A(i, j) below the diagonal uses e = j D + i; the
// diagonal i uses 256 ids from D*D + 256 i; z uses D*D + 256 D + i
// Outlier layout (sel != nullptr): the slots of clusters with sel[k] = 1 (the outlier cluster and the
// clusters split from it) use the second prior (k1, v1, ld1, prior1); slots [skip_lo, skip_hi)
// (cluster 1, local_clusters_actions.cpp:348-351) keep their parameters: only their log marginal
// likelihood and the cluster slot's weight term are refreshed (cbase[s] = -log det Sigma / 2 of the
// slot's current parameters, written by every draw).
template <int DP>
__global__ void __launch_bounds__(RegChol<DP>::T) k_draw_niw(const double* __restrict__ stats, int stat_len, int D,
                                                              int Dp, double k0, double v0, double ld0,
                                                              const double* __restrict__ prior, double k1, double v1,
                                                              double ld1, const double* __restrict__ prior1,
                                                              const uint8_t* __restrict__ sel, int skip_lo,
                                                              int skip_hi, double* __restrict__ cbase,
                                                              const double* __restrict__ shift,
                                                              const double* __restrict__ logw, uint64_t seed,
                                                              uint64_t draw, float* __restrict__ Wt,
                                                              float* __restrict__ bv, float* __restrict__ cv,
                                                              float* __restrict__ muv, double* __restrict__ lml,
                                                              int* __restrict__ err)
{
    __shared__ double sh[RegChol<DP>::SMEM];
    __shared__ double mean[DP], yv[DP], zv[DP], uv[DP];
    extern __shared__ double dyn[];
    const int AL = D + 1;                  // leading dimension of A: column reads across lanes are conflict-free
    double* Lm = dyn;                      // D*D: Cholesky factor of psi', later its inverse
    double* Am = Lm + (size_t)D * D;       // D*AL: Bartlett factor (lower)
    double* red = sh + 3 * DP;
    const int s = blockIdx.x, t = threadIdx.x;
    if (sel && sel[s / 3]) {   // the outlier prior
        k0 = k1;
        v0 = v1;
        ld0 = ld1;
        prior = prior1;
    }
    const double* st = stats + (size_t)s * stat_len;
    const double n = st[0];
    const double kp = k0 + n, vp = v0 + n;
    for (int e = t; e < D * D; e += blockDim.x) Lm[e] = 0.0;
    __syncthreads();
    NiwExtras ex;
    const double L = niw_lml_reg<DP>(D, n, st + 1, st + 1 + D, nullptr, nullptr, k0, v0, prior, prior + D, ld0, sh,
                                     &ex, Lm, true);
    if (s >= skip_lo && s < skip_hi) {   // parameters kept (uniform over the block)
        if (t == 0) {
            lml[s] = n > 0 ? L : 0.0;
            if (s % 3 == 0) cv[s] = (float)(cbase[s] + logw[s / 3]);
        }
        return;
    }
    const double* mp = sh + 2 * DP;        // posterior mean, left by niw_lml_reg
    const uint32_t us = (uint32_t)s;
    for (int e = t; e < D * D; e += blockDim.x) {
        const int i = e % D, j = e / D;
        double v = 0.0;
        if (i > j) v = normal_from(param_bits(seed, draw, (uint32_t)e, us));
        else if (i == j) v = sqrt(chi2_draw(vp - i, seed, draw, us, (uint32_t)(D * D + 256 * i)));
        Am[(size_t)j * AL + i] = v;
    }
    for (int i = t; i < D; i += blockDim.x) zv[i] = normal_from(param_bits(seed, draw, (uint32_t)(D * D + 256 * D + i), us));
    __syncthreads();
    // A^T y = z (A^T upper triangular), one warp, rows from the last
    if (t < 32) {
        for (int i = D - 1; i >= 0; --i) {
            double p = 0;
            for (int q = i + 1 + t; q < D; q += 32) p += Am[(size_t)i * AL + q] * yv[q];
            p = warp_sum_d(p);
            if (t == 0) yv[i] = (zv[i] - p) / Am[(size_t)i * AL + i];
            __syncwarp();
        }
    }
    __syncthreads();
    // mu = m' + L_B y / sqrt(kappa'), L_B = sqrt(nu') L (the factor of nu' psi')
    const double sv = sqrt(vp), isk = 1.0 / sqrt(kp);
    for (int i = t; i < D; i += blockDim.x) {
        double acc = 0;
        for (int q = 0; q <= i; ++q) acc += Lm[(size_t)q * D + i] * yv[q];
        mean[i] = mp[i] + sv * acc * isk;
    }
    double la = 0;
    for (int i = t; i < D; i += blockDim.x) la += log(Am[(size_t)i * AL + i]);
    la = block_sum(la, red);               // (its barriers also order mean[] before the inverse)
    const double logdet_sigma = D * log(vp) + ex.ld - 2.0 * la;
    block_tri_inverse(Lm, D);              // Lm = L^-1 (lower)
    // u = L^-1 (mu - shift); b_j = sum_i W(i, j) (mu_i - shift_i) = (1/sqrt(nu')) sum_{k >= j} A(k, j) u_k
    for (int k = t; k < D; k += blockDim.x) {
        double acc = 0;
        for (int i = 0; i <= k; ++i) acc += Lm[(size_t)i * D + k] * (mean[i] - shift[i]);
        uv[k] = acc;
    }
    __syncthreads();
    const float isv = (float)(1.0 / sv);
    float* wt = Wt + (size_t)s * Dp * Dp;
    // W(i, j) = (1/sqrt(nu')) sum_{k >= max(i, j)} L^-1(k, i) A(k, j); Wt[j][i] = W(i, j); lanes take j
    for (int e = t; e < Dp * Dp; e += blockDim.x) {
        const int i = e / Dp, j = e % Dp;
        float w = 0.f;
        if (i < D && j < D) {
            double acc = 0;
            for (int k = max(i, j); k < D; ++k) acc += Lm[(size_t)i * D + k] * Am[(size_t)j * AL + k];
            w = (float)acc * isv;
        }
        wt[(size_t)j * Dp + i] = w;
    }
    for (int j = t; j < Dp; j += blockDim.x) {
        double b = 0;
        if (j < D)
            for (int k = j; k < D; ++k) b += Am[(size_t)j * AL + k] * uv[k];
        bv[(size_t)s * Dp + j] = j < D ? (float)(b / sv) : 0.f;
        muv[(size_t)s * Dp + j] = j < D ? (float)(mean[j] - shift[j]) : 0.f;
    }
    if (t == 0) {
        const double cval = -logdet_sigma / 2 + (s % 3 == 0 ? logw[s / 3] : 0.0);
        if (cbase) cbase[s] = -logdet_sigma / 2;
        cv[s] = (float)cval;
        lml[s] = n > 0 ? L : 0.0;
        if (isnan(cval) || cval == INFINITY || !isfinite(ex.ld)) atomicCAS(err, 0, s + 1);
    }
}

// multinomial_prior::sample_distribution (multinomial_prior.cpp:24-49) for every statistics slot: the
// Dirichlet posterior alpha' = alpha + sum x (multinomial_prior.cpp:12-22), theta = g / sum g with
// g_d ~ Gamma(alpha'_d, 1) (the gamma normalisation of dirichlet.h:39-48), log theta written into the
// label-phase parameters; the slot's log marginal likelihood lnG(sum alpha) - lnG(sum alpha')
// + sum [lnG(alpha'_d) - lnG(alpha_d)] (multinomial_prior.cpp:56-67; 0 for an empty slot, whose
// posterior is the prior) for the splittable test.  One block per slot; element d draws from the
// Philox streams 256 d .. 256 d + 201 of (slot, draw).
__global__ void __launch_bounds__(256) k_draw_dirichlet(const double* __restrict__ stats, int stat_len, int D, int Dp,
                                                        const double* __restrict__ alpha0,
                                                        const double* __restrict__ alpha1,
                                                        const uint8_t* __restrict__ sel, int skip_lo, int skip_hi,
                                                        uint64_t seed, uint64_t draw,
                                                        float* __restrict__ lt, float* __restrict__ cv,
                                                        double* __restrict__ lml)
{
    __shared__ double red[33];
    const int s = blockIdx.x, t = threadIdx.x;
    if (sel && sel[s / 3]) alpha0 = alpha1;   // the outlier prior
    const bool keep = s >= skip_lo && s < skip_hi;   // parameters kept: the marginal likelihood only
    const double* st = stats + (size_t)s * stat_len;
    const double n = st[0];
    double gsum = 0, a0 = 0, ap = 0, lg = 0;
    for (int d = t; d < D; d += blockDim.x) {
        const double a = alpha0[d], a1 = a + st[1 + d];
        if (!keep) {
            const double g = fmax(0.5 * chi2_draw(2.0 * a1, seed, draw, (uint32_t)s, (uint32_t)(256 * d)), 1e-300);
            lt[(size_t)s * Dp + d] = (float)log(g);   // log g for now: the normalisation follows
            gsum += g;
        }
        a0 += a;
        ap += a1;
        lg += lgamma(a1) - lgamma(a);
    }
    gsum = block_sum(gsum, red);
    a0 = block_sum(a0, red);
    ap = block_sum(ap, red);
    lg = block_sum(lg, red);
    if (!keep) {
        const float lz = (float)log(gsum);
        for (int d = t; d < Dp; d += blockDim.x) lt[(size_t)s * Dp + d] = d < D ? lt[(size_t)s * Dp + d] - lz : 0.f;
    }
    if (t == 0) {
        if (!keep) cv[s] = 0.f;   // the multinomial cluster log-likelihood has no weight term (cudaKernel_multinomial.cu:60-76)
        lml[s] = n > 0 ? lgamma(a0) - lgamma(ap) + lg : 0.0;
    }
}

// merge_clusters_to_splittable for disjoint pairs (i, j): slots 3i, 3i+1 <- c_i + c_j, 3i+2 <- c_j
__global__ void k_merge_stats(double* __restrict__ stats, int stat_len, const int32_t* __restrict__ pairs)
{
    const int i = pairs[2 * blockIdx.x], j = pairs[2 * blockIdx.x + 1];
    double* ci = stats + (size_t)(3 * i) * stat_len;
    const double* cj = stats + (size_t)(3 * j) * stat_len;
    for (int e = threadIdx.x; e < stat_len; e += blockDim.x) {
        const double a = ci[e], b = cj[e];
        ci[e] = a + b;
        ci[stat_len + e] = a + b;
        ci[2 * stat_len + e] = b;
    }
}

// dst cluster k takes the three slots of src cluster keep[k]
__global__ void k_compact_stats(const double* __restrict__ src, double* __restrict__ dst, int stat_len,
                                const int32_t* __restrict__ keep)
{
    const int k = blockIdx.x;
    const double* a = src + (size_t)(3 * keep[k]) * stat_len;
    double* b = dst + (size_t)(3 * k) * stat_len;
    for (int e = threadIdx.x; e < 3 * stat_len; e += blockDim.x) b[e] = a[e];
}

static bool device_draws_supported(const dpmm_ctx* c) { return c->prior == DPMM_PRIOR_GAUSSIAN && c->Dp <= 64; }

template <int DP>
static dpmm_status launch_draw_niw(dpmm_ctx* c, int K, uint64_t seed, uint64_t draw)
{
    if constexpr (DP > 64) {
        return fail(DPMM_ERR_INVALID_ARG, "device draws need D <= 64");
    } else {
        const size_t sm = sizeof(double) * ((size_t)c->D * c->D + (size_t)c->D * (c->D + 1));
        DPMM_TRY(allow_smem(k_draw_niw<DP>, sm));
        const bool out = c->outlier_layout != 0;
        k_draw_niw<DP><<<3 * K, RegChol<DP>::T, sm, c->stream>>>(
            c->d_stats, c->stat_len, c->D, c->Dp, c->prior_k, c->prior_v, c->prior_logdet, c->d_prior, c->prior2_k,
            c->prior2_v, c->prior2_logdet, out ? c->d_prior2 : c->d_prior, out ? c->d_prior_sel : nullptr,
            out ? 3 : 0, out && K > 1 ? 6 : 0, c->d_cbase, c->d_gshift, c->d_logw, seed, draw, c->d_Wt, c->d_b, c->d_c, c->d_mu,
            c->d_lml, c->d_aux + 6);
        return DPMM_OK;
    }
}

}  // namespace dpmm

using namespace dpmm;

extern "C" dpmm_status dpmm_sample_gaussian_params(dpmm_ctx* c, int K, uint64_t seed, uint64_t draw,
                                                   const double* weights, const double* lr_weights, double* lml)
{
    if (!c || !weights || !lr_weights) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    if (K < 1 || K > c->k_max) return fail(DPMM_ERR_INVALID_ARG, "K out of range [1, k_max]");
    if (!device_draws_supported(c)) return fail(DPMM_ERR_INVALID_ARG, "device draws need the NIW prior and D <= 64");
    if (!c->prior_set) return fail(DPMM_ERR_STATE, "prior hyper-parameters not set");
    if (c->stats_K < K) return fail(DPMM_ERR_STATE, "statistics of the K clusters are not on the device");
    DPMM_CUDA_TRY(cudaSetDevice(c->device));
    std::vector<double> lw(K);
    std::vector<float> lrw(2 * (size_t)K);
    for (int k = 0; k < K; ++k) {
        lw[k] = std::log(weights[k]);
        if (!std::isfinite(lw[k]) && !(lw[k] < 0)) return fail(DPMM_ERR_NUMERIC, "non-finite cluster weight");
        lrw[2 * k] = (float)std::log(lr_weights[2 * k]);
        lrw[2 * k + 1] = (float)std::log(lr_weights[2 * k + 1]);
    }
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    double* hl = c->h_pinned;
    std::memcpy(hl, lw.data(), sizeof(double) * K);
    {
        PhaseTimer pt(c, PH_PARAMS);
        DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_logw, hl, sizeof(double) * K, cudaMemcpyHostToDevice, c->stream));
        DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_lrw, lrw.data(), sizeof(float) * 2 * K, cudaMemcpyHostToDevice, c->stream));
        DPMM_CUDA_TRY(cudaMemsetAsync(c->d_aux + 6, 0, sizeof(int32_t), c->stream));
        g_h2d_bytes.fetch_add(sizeof(double) * K + sizeof(float) * 2 * K, std::memory_order_relaxed);
        dpmm_status st = DPMM_OK;
        DPMM_WITH_DP(c->Dp, (st = launch_draw_niw<DP>(c, K, seed, draw)));
        DPMM_TRY(st);
        DPMM_LAUNCHED();
        c->K_params = K;
        DPMM_TRY(pack_tc_params(c, K));
    }
    int32_t* herr = reinterpret_cast<int32_t*>(c->h_pinned);
    DPMM_CUDA_TRY(cudaMemcpyAsync(herr, c->d_aux + 6, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    if (lml) DPMM_CUDA_TRY(cudaMemcpyAsync(lml, c->d_lml, sizeof(double) * 3 * K, cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    g_d2h_bytes.fetch_add(sizeof(int32_t) + (lml ? sizeof(double) * 3 * K : 0), std::memory_order_relaxed);
    if (herr[0] != 0) {
        const int s = herr[0] - 1;
        c->K_params = 0;
        return fail(DPMM_ERR_NOT_PD, "posterior scale of cluster " + std::to_string(s / 3) +
                                         (s % 3 ? " (sub)" : "") + " is not positive definite");
    }
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_sample_multinomial_params(dpmm_ctx* c, int K, uint64_t seed, uint64_t draw,
                                                      const double* lr_weights, double* lml)
{
    if (!c || !lr_weights) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    if (c->prior != DPMM_PRIOR_MULTINOMIAL) return fail(DPMM_ERR_INVALID_ARG, "context is not multinomial");
    if (K < 1 || K > c->k_max) return fail(DPMM_ERR_INVALID_ARG, "K out of range [1, k_max]");
    if (!c->prior_set) return fail(DPMM_ERR_STATE, "prior hyper-parameters not set");
    if (c->stats_K < K) return fail(DPMM_ERR_STATE, "statistics of the K clusters are not on the device");
    DPMM_CUDA_TRY(cudaSetDevice(c->device));
    std::vector<float> lrw(2 * (size_t)K);
    for (int k = 0; k < 2 * K; ++k) lrw[k] = (float)std::log(lr_weights[k]);
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    float* hl = reinterpret_cast<float*>(c->h_pinned);
    std::memcpy(hl, lrw.data(), sizeof(float) * 2 * K);
    {
        PhaseTimer pt(c, PH_PARAMS);
        DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_lrw, hl, sizeof(float) * 2 * K, cudaMemcpyHostToDevice, c->stream));
        g_h2d_bytes.fetch_add(sizeof(float) * 2 * K, std::memory_order_relaxed);
        const bool out = c->outlier_layout != 0;
        k_draw_dirichlet<<<3 * K, 256, 0, c->stream>>>(c->d_stats, c->stat_len, c->D, c->Dp, c->d_prior,
                                                        out ? c->d_prior2 : c->d_prior,
                                                        out ? c->d_prior_sel : nullptr, out ? 3 : 0,
                                                        out && K > 1 ? 6 : 0, seed, draw,
                                                       c->d_mu, c->d_c, c->d_lml);
        DPMM_LAUNCHED();
        c->K_params = K;
        c->mult_tc_K = -1;
    }
    if (lml) DPMM_CUDA_TRY(cudaMemcpyAsync(lml, c->d_lml, sizeof(double) * 3 * K, cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (lml) g_d2h_bytes.fetch_add(sizeof(double) * 3 * K, std::memory_order_relaxed);
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_merge_statistics(dpmm_ctx* c, int n, const int32_t* index, const int32_t* new_index)
{
    if (!c || n < 0 || (n > 0 && (!index || !new_index))) return fail(DPMM_ERR_INVALID_ARG, "bad pair list");
    if (n == 0) return DPMM_OK;
    std::vector<int32_t> pairs(2 * (size_t)n);
    std::vector<uint8_t> used(c->k_max, 0);
    for (int t = 0; t < n; ++t) {
        const int i = index[t], j = new_index[t];
        if (i < 0 || j < 0 || i >= c->k_max || j >= c->k_max || i == j)
            return fail(DPMM_ERR_INVALID_ARG, "cluster index out of range");
        if (used[i] || used[j]) return fail(DPMM_ERR_INVALID_ARG, "merge pairs must be disjoint");
        used[i] = used[j] = 1;
        pairs[2 * t] = i;
        pairs[2 * t + 1] = j;
    }
    DPMM_CUDA_TRY(cudaSetDevice(c->device));
    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_remap, pairs.data(), sizeof(int32_t) * 2 * n, cudaMemcpyHostToDevice, c->stream));
    g_h2d_bytes.fetch_add(sizeof(int32_t) * 2 * n, std::memory_order_relaxed);
    k_merge_stats<<<n, 256, 0, c->stream>>>(c->d_stats, c->stat_len, c->d_remap);
    DPMM_LAUNCHED();
    // the slots now hold the host's bookkeeping, which the next draw reads as they are
    for (int t = 0; t < n; ++t) c->stats_ok[index[t]] = c->stats_ok[new_index[t]] = 1;
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_compact_statistics(dpmm_ctx* c, int n_keep, const int32_t* keep)
{
    if (!c || n_keep < 0 || n_keep > c->k_max || (n_keep > 0 && !keep)) return fail(DPMM_ERR_INVALID_ARG, "bad keep list");
    for (int k = 0; k < n_keep; ++k)
        if (keep[k] < 0 || keep[k] >= c->k_max || (k > 0 && keep[k] <= keep[k - 1]))
            return fail(DPMM_ERR_INVALID_ARG, "keep list must be increasing cluster indices");
    if (n_keep == 0) return DPMM_OK;
    DPMM_CUDA_TRY(cudaSetDevice(c->device));
    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_remap, keep, sizeof(int32_t) * n_keep, cudaMemcpyHostToDevice, c->stream));
    g_h2d_bytes.fetch_add(sizeof(int32_t) * n_keep, std::memory_order_relaxed);
    k_compact_stats<<<n_keep, 256, 0, c->stream>>>(c->d_stats, c->d_stats_tmp, c->stat_len, c->d_remap);
    DPMM_LAUNCHED();
    std::swap(c->d_stats, c->d_stats_tmp);
    if (c->outlier_layout && n_keep > 1 && keep[1] != 1 && c->K_params > keep[1]) {
        // cluster 1's parameters are not redrawn (local_clusters_actions.cpp:348-351): the cluster that
        // moves into index 1 brings its current ones (device to device, the 3 slots are contiguous)
        const size_t s0 = 3 * (size_t)keep[1], s1 = 3;
        if (c->prior == DPMM_PRIOR_GAUSSIAN) {
            const size_t m = (size_t)c->Dp * c->Dp;
            DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_Wt + s1 * m, c->d_Wt + s0 * m, sizeof(float) * 3 * m,
                                          cudaMemcpyDeviceToDevice, c->stream));
            DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_b + s1 * c->Dp, c->d_b + s0 * c->Dp, sizeof(float) * 3 * c->Dp,
                                          cudaMemcpyDeviceToDevice, c->stream));
            if (c->d_cbase)
                DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_cbase + s1, c->d_cbase + s0, sizeof(double) * 3,
                                              cudaMemcpyDeviceToDevice, c->stream));
        }
        DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_mu + s1 * c->Dp, c->d_mu + s0 * c->Dp, sizeof(float) * 3 * c->Dp,
                                      cudaMemcpyDeviceToDevice, c->stream));
        DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_c + s1, c->d_c + s0, sizeof(float) * 3, cudaMemcpyDeviceToDevice,
                                      c->stream));
        DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_lrw + 2, c->d_lrw + 2 * (size_t)keep[1], sizeof(float) * 2,
                                      cudaMemcpyDeviceToDevice, c->stream));
    }
    std::vector<uint8_t> ok(c->k_max, 0);
    for (int k = 0; k < n_keep; ++k) ok[k] = c->stats_ok[keep[k]];
    c->stats_ok = ok;
    c->stats_K = n_keep;
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_statistics_counts(dpmm_ctx* c, int n, const int32_t* indices, int64_t* count)
{
    if (!c || n < 0 || (n > 0 && (!indices || !count))) return fail(DPMM_ERR_INVALID_ARG, "bad index list");
    if (!c->points_ready) return fail(DPMM_ERR_STATE, "points not uploaded");
    if (n == 0) return DPMM_OK;
    int K = 0;
    for (int i = 0; i < n; ++i) {
        if (indices[i] < 0 || indices[i] >= c->k_max) return fail(DPMM_ERR_INVALID_ARG, "cluster index out of range");
        K = std::max(K, indices[i] + 1);
    }
    DPMM_CUDA_TRY(cudaSetDevice(c->device));
    const int Keff = std::min(c->k_max, std::max(K, c->K_params));
    DPMM_TRY(ensure_stats(c, Keff));
    double* h = c->h_pinned;
    // the count is the first value of every slot: one strided copy of 3K values
    DPMM_CUDA_TRY(cudaMemcpy2DAsync(h, sizeof(double), c->d_stats, sizeof(double) * c->stat_len, sizeof(double),
                                    3 * (size_t)K, cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    g_d2h_bytes.fetch_add(sizeof(double) * 3 * K, std::memory_order_relaxed);
    for (int q = 0; q < n; ++q)
        for (int s = 0; s < 3; ++s) count[3 * q + s] = (int64_t)llround(h[3 * indices[q] + s]);
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_get_gaussian_params(dpmm_ctx* c, int K, float* wt, float* b, float* cv, float* mu)
{
    if (!c) return fail(DPMM_ERR_INVALID_ARG, "null context");
    if (c->prior != DPMM_PRIOR_GAUSSIAN) return fail(DPMM_ERR_STATE, "context is not Gaussian");
    if (K < 1 || K > c->K_params) return fail(DPMM_ERR_STATE, "parameters of K clusters are not set");
    DPMM_CUDA_TRY(cudaSetDevice(c->device));
    const size_t S = 3 * (size_t)K, Dp = c->Dp;
    if (wt) DPMM_CUDA_TRY(cudaMemcpyAsync(wt, c->d_Wt, sizeof(float) * S * Dp * Dp, cudaMemcpyDeviceToHost, c->stream));
    if (b) DPMM_CUDA_TRY(cudaMemcpyAsync(b, c->d_b, sizeof(float) * S * Dp, cudaMemcpyDeviceToHost, c->stream));
    if (cv) DPMM_CUDA_TRY(cudaMemcpyAsync(cv, c->d_c, sizeof(float) * S, cudaMemcpyDeviceToHost, c->stream));
    if (mu) DPMM_CUDA_TRY(cudaMemcpyAsync(mu, c->d_mu, sizeof(float) * S * Dp, cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_get_multinomial_params(dpmm_ctx* c, int K, float* log_theta)
{
    if (!c || !log_theta) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    if (c->prior != DPMM_PRIOR_MULTINOMIAL) return fail(DPMM_ERR_STATE, "context is not multinomial");
    if (K < 1 || K > c->K_params) return fail(DPMM_ERR_STATE, "parameters of K clusters are not set");
    DPMM_CUDA_TRY(cudaSetDevice(c->device));
    DPMM_CUDA_TRY(cudaMemcpy2DAsync(log_theta, sizeof(float) * c->D, c->d_mu, sizeof(float) * c->Dp, sizeof(float) * c->D,
                                    3 * (size_t)K, cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return DPMM_OK;
}

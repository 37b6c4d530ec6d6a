/*
 * dpmm_capi.h -- C ABI of the B200 (sm_100a) implementation of the per-iteration
 * data-parallel path of the Chang & Fisher sub-cluster DPMM sampler.
 *
 * Two layers, both plain C (pointers, sizes, status codes; no C++ or torch types):
 *
 *  1. Device back-end (dpmm_ctx).  One entry point per method of the reference's
 *     device back-end class `cudaKernel` (DPMMSubClusters/cudaKernel.cuh:31-138) and
 *     its Gaussian / multinomial subclasses, so a C++ adapter deriving from
 *     `cudaKernel` can forward every call here and `prior::get_cuda()`,
 *     `local_clusters_actions::group_step` and `dp_parallel` stay unchanged.
 *     Each declaration names the reference method it replaces (file:line).
 *
 *  2. Whole sampler (dpmm_model_info).  dpmm_dp_parallel / dpmm_dp_parallel_from_file
 *     run the reference's iteration loop (dp_parallel_sampling.cpp:89-206) with this
 *     back-end and return what `ModelInfo` holds (labels, weights, iter_count, ...).
 *
 * Conventions (same as the reference):
 *   - points are point-major: the reference's Eigen D x N column-major matrix, i.e.
 *     point n occupies points[n*D .. n*D+D-1];
 *   - labels are 1-based int32; sub-labels are in {1, 2};
 *   - square matrices (inv_sigma, psi, S) are D x D column-major (Eigen's default);
 *   - uniforms are float in (0, 1], two per point per draw (u[2n], u[2n+1]), playing
 *     the role of the two curand_uniform() calls of the reference's alias draw
 *     (cudaKernel.cu:115-116).  A NULL uniforms pointer means "draw them on the device"
 *     with the context's generator (Philox4x32-10, or cuRAND XORWOW in compat mode).
 *
 * Error convention: every function returns a dpmm_status; nothing calls exit().  The
 * reference instead printf()s and exit(EXIT_FAILURE)s on any CUDA error
 * (cudaKernel.cu:1492-1508).  dpmm_last_error() gives a message for the calling thread.
 *
 * Threading: a context is used by one host thread at a time; separate contexts may be
 * driven from separate threads.  All device memory is allocated at dpmm_create (at
 * capacity k_max); the phase calls do not allocate.
 */
#ifndef DPMM_CAPI_H
#define DPMM_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DPMM_CAPI_VERSION 1

typedef enum dpmm_status {
    DPMM_OK = 0,
    DPMM_ERR_INVALID_ARG = 1,
    DPMM_ERR_OOM = 2,
    DPMM_ERR_CUDA = 3,
    DPMM_ERR_NOT_PD = 4,       /* a matrix that must be positive definite is not */
    DPMM_ERR_TIMEOUT = 5,      /* a bounded device wait gave up */
    DPMM_ERR_NUMERIC = 6,      /* NaN / Inf in inputs or results */
    DPMM_ERR_STATE = 7,        /* call out of order (e.g. no points uploaded) */
    DPMM_ERR_IO = 8,           /* file could not be read / parsed */
    DPMM_ERR_NO_DEVICE = 9,
    DPMM_ERR_EXCHANGE = 10     /* a sharded context's allreduce reported a failure */
} dpmm_status;

/* prior_type (global_params.h:11-15) */
typedef enum dpmm_prior_type { DPMM_PRIOR_GAUSSIAN = 0, DPMM_PRIOR_MULTINOMIAL = 1 } dpmm_prior_type;

/* device random generator for draws whose uniforms the caller does not supply */
typedef enum dpmm_rng_kind {
    DPMM_RNG_PHILOX = 0,        /* counter-based Philox4x32-10: stateless, (seed, point, draw) */
    DPMM_RNG_CURAND_XORWOW = 1  /* per-point curandStateXORWOW, curand_init(seed, point, 0):
                                   the reference's stream and call order (cudaKernel.cu:19-25) */
} dpmm_rng_kind;

/* how the N x K log-likelihood contraction is computed */
typedef enum dpmm_loglik_mode {
    DPMM_LL_FP32 = 0,           /* SIMT FP32 ("plain FP32 form") */
    DPMM_LL_TC_BF16X3 = 1,      /* tcgen05 tensor cores, split-BF16 (hi*hi + lo*hi + hi*lo), FP32 accumulate */
    DPMM_LL_AUTO = 2            /* tensor cores where the shape allows, else FP32 */
} dpmm_loglik_mode;

typedef struct dpmm_desc {
    int64_t n_points;     /* N */
    int32_t dim;          /* D */
    int32_t prior_type;   /* dpmm_prior_type */
    int32_t k_max;        /* capacity for clusters (0 -> 256) */
    int32_t rng_kind;     /* dpmm_rng_kind */
    uint64_t seed;        /* device generator seed */
    int32_t loglik_mode;  /* dpmm_loglik_mode */
    int32_t device;       /* CUDA device ordinal */
    int32_t verbose;
    int32_t reserved[7];
} dpmm_desc;

typedef struct dpmm_ctx dpmm_ctx;

const char* dpmm_status_string(dpmm_status s);
/* message of the last failing call on this host thread ("" if none) */
const char* dpmm_last_error(void);
int dpmm_capi_version(void);

/* ------------------------------------------------------------------ sharding by points
 * No counterpart in the reference (its multi-device code is inactive, cudaKernel.cu:553-554).
 * A context may hold one shard of a data set split by points over `world` ranks.  Per-point work
 * (labels, sub-labels, relabels, the pruned label phase) stays on the shard; every aggregate the
 * context returns or keeps -- the statistics of every cluster slot, the sub-label counts, the
 * all-points statistics, the label-agreement contingency table, and the mean the points are
 * shifted by -- is summed over the ranks through `allreduce`, so it is the whole data set's.
 * Random numbers are keyed by the global point index (point_offset + local index), so a sharded
 * run draws what one context over all points draws. */

/* In-place sum over all ranks of `count` doubles in device memory at `buf`, which the context has
 * written on `stream` (a cudaStream_t).  On return buf must hold the sums, identical on every rank,
 * and work the context queues on `stream` afterwards must see them.  Every rank calls it the same
 * number of times in the same order.  Returns 0 on success. */
typedef int (*dpmm_allreduce_fn)(void* user, double* buf, int64_t count, void* stream);

typedef struct dpmm_shard {
    int32_t rank;               /* 0 .. world-1 */
    int32_t world;              /* ranks holding shards of the data set */
    int64_t point_offset;       /* global index of this shard's first point */
    int64_t n_total;            /* points of all shards together */
    dpmm_allreduce_fn allreduce;
    void* user;                 /* passed to allreduce */
} dpmm_shard;

/* ------------------------------------------------------------------ device back-end */

/* cudaKernel::init (cudaKernel.cu:537-635).  Unlike the reference it does not call
 * cudaDeviceReset, so several contexts (samplers) can share a device. */
dpmm_status dpmm_create(const dpmm_desc* desc, dpmm_ctx** out);
/* cudaKernel::release (cudaKernel.cu:720-749) */
dpmm_status dpmm_destroy(dpmm_ctx* ctx);

/* The H2D copy of the points inside cudaKernel::init (cudaKernel.cu:622-626).
 * points: N*D values, point-major, in host (pageable or pinned) or device memory.  The device keeps
 * them as FP32 relative to a shift (NIW prior: the mean of every (n_total / 65536)-th point by global
 * index, rounded to 20 significant bits); pageable host points are converted on host threads, so
 * only the FP32 rows cross PCIe.  NaN or Inf in the points gives DPMM_ERR_NUMERIC. */
dpmm_status dpmm_upload_points(dpmm_ctx* ctx, const double* points);
dpmm_status dpmm_upload_points_f32(dpmm_ctx* ctx, const float* points);
/* Makes the context one shard of a data set split by points (see dpmm_shard); call it before the
 * points are uploaded.  In a sharded context dpmm_set_ground_truth takes values in [0, 65536). */
dpmm_status dpmm_set_shard(dpmm_ctx* ctx, const dpmm_shard* shard);

/* cudaKernel::sample_labels (cudaKernel.cu:1103-1111): labels uniform in
 * [1 + o, initial_clusters + o], o = (outlier_mod > 0). */
dpmm_status dpmm_sample_labels(dpmm_ctx* ctx, int initial_clusters, double outlier_mod,
                               const float* uniforms /* N or NULL */);
/* cudaKernel::sample_sub_labels (cudaKernel.cu:1093-1101) */
dpmm_status dpmm_sample_sub_labels(dpmm_ctx* ctx, const float* uniforms /* N or NULL */);
/* The two uniforms per point that the next label or sub-label draw would take from the
 * context's generator (the pair of curand_uniform() calls of cudaKernel.cu:115-116 in
 * cuRAND-compatible mode), written to uniforms[2N]; the generator advances as that draw
 * would.  Lets a caller replay the reference's random stream through the caller-uniform
 * paths. */
dpmm_status dpmm_draw_uniforms(dpmm_ctx* ctx, float* uniforms /* 2N */);

/* cudaKernel::update_labels (cudaKernel.cu:1145-1148); the set_labels / set_sub_labels
 * seams of the reference's test double (test/myCudaKernel.h). */
dpmm_status dpmm_set_labels(dpmm_ctx* ctx, const int32_t* labels);
dpmm_status dpmm_set_sub_labels(dpmm_ctx* ctx, const int32_t* sub_labels);
/* cudaKernel::get_labels / get_sub_labels (cudaKernel.cu:1113-1143) */
dpmm_status dpmm_get_labels(dpmm_ctx* ctx, int32_t* labels);
dpmm_status dpmm_get_sub_labels(dpmm_ctx* ctx, int32_t* sub_labels);
/* cudaKernel::get_sub_labels_count (cudaKernel.cu:1237-1257) */
dpmm_status dpmm_get_sub_labels_count(dpmm_ctx* ctx, int32_t* l, int32_t* r);

/* cudaKernel::inverse_matrix (cudaKernel.cu:1558-1598), used by niw::sample_distribution
 * (priors/niw.cpp:61-107): B = A^-1 for an n x n FP64 matrix, 1 <= n <= 2048, host arrays in either
 * layout (column-major in, column-major out; row-major likewise), computed on the device.  The
 * reference inverts by Gauss-Jordan without pivoting; this uses partial pivoting (the same inverse to
 * FP64 rounding) and returns DPMM_ERR_NUMERIC for a singular matrix or a non-finite inverse. */
dpmm_status dpmm_inverse_matrix(dpmm_ctx* ctx, int n, const double* A, double* B);

/* cudaKernel::multiplie_matrix_for_inverseWishart (cudaKernel.cu:980-1016), used by
 * niw::sample_distribution: C = (A B)(A B)^T with A m x n, B n x k, C m x m, FP64 column-major host
 * arrays (sizes 1 .. 2048), computed on the device (C exactly symmetric). */
dpmm_status dpmm_multiply_for_inverse_wishart(dpmm_ctx* ctx, int m, int n, int k, const double* A,
                                              const double* B, double* C);

/* Cluster parameters for the next label / sub-label phase: the thin_cluster_params
 * broadcast (local_clusters_actions.cpp:373-382, 449-458) plus the per-cluster H2D copies
 * the reference makes inside cudaKernel_gaussian::log_likelihood_labels / _sub_labels
 * (cudaKernel_gaussian.cu:43-113).
 *   mu[K*D], inv_sigma[K*D*D] (col-major), logdet_sigma[K], weights[K]: cluster k;
 *   mu_lr[2K*D], inv_sigma_lr[2K*D*D], logdet_sigma_lr[2K], lr_weights[2K]: sub-cluster
 *   (k, s) at index 2k+s, s = 0 (l) / 1 (r).
 * The precision matrices are factored on the host (FP64 Cholesky, inv_sigma = W W^T);
 * a matrix that is not positive definite gives DPMM_ERR_NOT_PD. */
dpmm_status dpmm_set_gaussian_params(dpmm_ctx* ctx, int K, const double* mu,
                                     const double* inv_sigma, const double* logdet_sigma,
                                     const double* weights, const double* mu_lr,
                                     const double* inv_sigma_lr, const double* logdet_sigma_lr,
                                     const double* lr_weights);
/* Same, given precision square-root factors W (inv_sigma = W W^T, D x D col-major, any such
 * factor), as the Bartlett draw of niw::sample_distribution (niw.cpp:61-107) produces directly;
 * no host factorisation is done. */
dpmm_status dpmm_set_gaussian_factors(dpmm_ctx* ctx, int K, const double* mu, const double* w,
                                      const double* logdet_sigma, const double* weights,
                                      const double* mu_lr, const double* w_lr,
                                      const double* logdet_sigma_lr, const double* lr_weights);
/* multinomial_dist{alpha = log theta} per cluster / sub-cluster (cudaKernel_multinomial.cu:37-76);
 * weights are accepted but, as in the reference, do not enter the label log-likelihood. */
dpmm_status dpmm_set_multinomial_params(dpmm_ctx* ctx, int K, const double* log_theta,
                                        const double* weights, const double* log_theta_lr,
                                        const double* lr_weights);

/* cudaKernel::create_clusters_labels (cudaKernel.cu:1400-1490): N x K log-likelihood,
 * softmax and Walker-alias draw per point (argmax when final != 0), fused in one kernel;
 * the N x K matrix never reaches memory.
 *   uniforms: 2N or NULL.  loglik_out (test seam, nullable): N x K point-major, each
 *   value WITHOUT the cluster-independent constant -D*D*log(2*pi)/2 (Gaussian). */
dpmm_status dpmm_create_clusters_labels(dpmm_ctx* ctx, int K, int final_, const float* uniforms,
                                        float* loglik_out);
/* cudaKernel::create_subclusters_labels (cudaKernel.cu:1299-1398): for every point its two
 * sub-cluster log-likelihoods (+ log lr_weights), 2-way softmax and alias draw, using the
 * labels of the last label phase.  Fused with the sufficient-statistic reduction of
 * dpmm_create_sufficient_statistics (results kept on the device and returned by it).
 *   loglik_out (nullable): N x 2 point-major, without the -D*D*log(2*pi)/2 constant. */
dpmm_status dpmm_create_subclusters_labels(dpmm_ctx* ctx, int K, const float* uniforms,
                                           float* loglik_out);
/* cudaKernel::create_sufficient_statistics (cudaKernel.cu:844-941): for each of the n
 * listed clusters (0-based indices) the statistics of the cluster (slot 3i), its l (3i+1)
 * and r (3i+2) sub-clusters: count, sum x (D) and, Gaussian only, the uncentred scatter
 * S = sum x x^T (D x D).  Any output pointer may be NULL.  Computed from the current labels
 * and sub-labels with a deterministic segmented reduction (FP32 within a chunk of points,
 * shifted; FP64 across chunks). */
dpmm_status dpmm_create_sufficient_statistics(dpmm_ctx* ctx, int n, const int32_t* indices,
                                              int64_t* count, double* sum, double* S);

/* cudaKernel::split_cluster_local_worker (cudaKernel.cu:1204-1214), applied for each pair in
 * order: in cluster index[i], sub==2 points move to new_index[i]; every point of it gets a
 * fresh random sub-label (curand()%2+1).  bits (nullable, N values) stands for curand(). */
dpmm_status dpmm_split_clusters(dpmm_ctx* ctx, int n, const int32_t* index, const int32_t* new_index,
                                const uint32_t* bits);
/* cudaKernel::merge_clusters_worker (cudaKernel.cu:1215-1225), each pair in order */
dpmm_status dpmm_merge_clusters(dpmm_ctx* ctx, int n, const int32_t* index, const int32_t* new_index);
/* cudaKernel::reset_bad_clusters_worker (cudaKernel.cu:1226-1236), each index in order */
dpmm_status dpmm_reset_bad_clusters(dpmm_ctx* ctx, int n, const int32_t* index, const uint32_t* bits);
/* cudaKernel::remove_empty_clusters_worker (cudaKernel.cu:1194-1203) called once per limit,
 * in order (labels > limit are decremented); applied as one relabel pass. */
dpmm_status dpmm_remove_empty_clusters(dpmm_ctx* ctx, int n, const int32_t* limits);

/* Test seams of the reference's test double (test/myCudaKernel.h):
 * cudaKernel_gaussian::log_likelihood_labels (cudaKernel_gaussian.cu:82-113) for one cluster,
 * r_out[N] in FP64 INCLUDING the -D*D*log(2*pi)/2 constant; */
dpmm_status dpmm_log_likelihood_labels_gaussian(dpmm_ctx* ctx, const double* mu,
                                                const double* inv_sigma, double logdet_sigma,
                                                double weight, double* r_out);
/* cudaKernel_multinomial::log_likelihood_labels (cudaKernel_multinomial.cu:60-76) */
dpmm_status dpmm_log_likelihood_labels_multinomial(dpmm_ctx* ctx, const double* log_theta,
                                                   double* r_out);
/* cudaKernel::sample_log_cat_array (cudaKernel.cu:805-829): softmax + alias draw of labels
 * from a caller-given N x K column-major log-likelihood matrix (FP64 arithmetic). */
dpmm_status dpmm_sample_log_cat_array(dpmm_ctx* ctx, int K, const double* loglik,
                                      const float* uniforms);
/* cudaKernel::sample_log_cat_array_sub_cluster (cudaKernel.cu:775-803): m points with
 * indices[m], loglik m x 2 column-major, lr_weights[2]; writes their sub-labels. */
dpmm_status dpmm_sample_log_cat_array_sub_cluster(dpmm_ctx* ctx, int m, const double* loglik,
                                                  const int32_t* indices, const double* lr_weights,
                                                  const float* uniforms);

/* ---- split / merge Hastings in one launch each (FP64 on the device) -------------------- */

/* Prior hyper-parameters: niw_hyperparams{k, m, v, psi} (priors/niw_hyperparams.h:9-43) or
 * multinomial_hyper{alpha} (priors/multinomial_hyper.h:9-29). */
dpmm_status dpmm_set_prior_niw(dpmm_ctx* ctx, double k, const double* m, double v, const double* psi);
dpmm_status dpmm_set_prior_multinomial(dpmm_ctx* ctx, const double* alpha);
/* Runs with an outlier cluster (outlier_mod > 0: create_outlier_local_cluster and sample_clusters,
 * local_clusters_actions.cpp:48-79, 341-371) with device draws: the outlier cluster's own prior
 * (outlier_hyper_params) for the clusters that carry it, chosen per cluster by
 * dpmm_set_cluster_priors (second[k] != 0: cluster k uses it; the outlier cluster and the clusters
 * split from it), in the device draws and the device marginal likelihoods; and, as the reference,
 * cluster 1's parameters are not redrawn (its marginal likelihood and weight term are refreshed),
 * and move with it when dpmm_compact_statistics renumbers the clusters. */
dpmm_status dpmm_set_outlier_prior_niw(dpmm_ctx* ctx, double k, const double* m, double v, const double* psi);
dpmm_status dpmm_set_outlier_prior_multinomial(dpmm_ctx* ctx, const double* alpha);
dpmm_status dpmm_set_cluster_priors(dpmm_ctx* ctx, int K, const uint8_t* second);

/* For the K clusters whose statistics the last dpmm_create_subclusters_labels /
 * dpmm_create_sufficient_statistics left on the device: the posterior of the cluster and
 * of its two sub-clusters (niw.cpp:23-49 / multinomial_prior.cpp:12-22), their log
 * marginal likelihoods (niw.cpp:122-138 / multinomial_prior.cpp:56-67) into lml[3K]
 * (slots 3k, 3k+1, 3k+2), and the split log Hastings ratio of each cluster
 * (local_clusters_actions.cpp:222-233) into split_log_hr[K] (NaN where N_l or N_r is 0). */
dpmm_status dpmm_split_hastings(dpmm_ctx* ctx, int K, double alpha, double* lml, double* split_log_hr);
/* Merge log Hastings ratio (shared_actions.cpp:88-111) of every pair i < j of the K clusters
 * in one launch: merge_log_hr[i*K + j] (row-major; entries with i >= j or an empty cluster
 * are NaN).  Uses the cluster-level statistics on the device. */
dpmm_status dpmm_merge_hastings(dpmm_ctx* ctx, int K, double alpha, double* merge_log_hr);

/* Allocation-free form of dpmm_merge_hastings, with no counterpart in the reference.  For callers
 * that cannot call cudaMalloc: host programs whose device memory is owned by another framework's
 * pool or fixed budget, and latency-critical loops that cannot afford cudaMalloc's implicit device
 * synchronisation.  It needs no dpmm_ctx: the caller passes device pointers to the inputs
 *   prior  NIW: m[D] then psi[D*D] (col-major); multinomial: alpha[D]   (k0, v0: NIW kappa, nu)
 *   stats  3K slots of (count, sum[D], S[D*D]) (NIW) or (count, sum[D]) (multinomial), FP64, in the
 *          layout dpmm_create_sufficient_statistics returns; slot 3k is cluster k
 * and the output merge_log_hr[K*K] (row-major; entries i >= j or with an empty cluster are NaN), and
 * the work is queued on `stream` (a cudaStream_t; NULL = the default stream) without waiting for it.
 * The kernels' scratch is a file-scope device array for at most 1024 clusters (K > 1024 is rejected
 * with DPMM_ERR_INVALID_ARG); every device that loads the library holds it (8 KB) until exit.  The
 * first call in a context (on a device, and again after cudaDeviceReset or when another context is
 * made current) looks up the array's device address, so make that first call before any stream
 * capture.  All calls on a device share the array: calls that overlap on the GPU race.
 * A NaN entry means an empty cluster, or a psi that is not positive definite (its log determinant,
 * and so every ratio, is NaN); dpmm_create / dpmm_set_prior reject such a psi with DPMM_ERR_NOT_PD.
 * It calls no cudaMalloc, cudaFree or other allocating routine. */
dpmm_status dpmm_merge_hastings_static(int32_t prior_type, int32_t D, int32_t K, double alpha, double k0, double v0,
                                       const double* prior, const double* stats, double* merge_log_hr,
                                       void* stream);

/* ---- learned split/merge screen (no counterpart in the reference) ----------------------------
 * The reference computes the exact ratio of every split candidate and every cluster pair each
 * iteration (local_clusters_actions.cpp:244-321).  The screen ranks the candidates with a small MLP
 * over 32 features derived from the statistics on the device, so the exact FP64 ratio
 * (dpmm_split_hastings_list / dpmm_merge_hastings_list, the same arithmetic as dpmm_split_hastings /
 * dpmm_merge_hastings) is needed for the best-ranked few only; the accept test stays exact.
 * Candidate rows: split row k = cluster k (K rows); merge row = pair i < j, row-major over the
 * strict upper triangle (K(K-1)/2 rows). */
#define DPMM_SCREEN_FEATURES 32
#define DPMM_SCREEN_HIDDEN 64
/* parameters, one FP32 vector: W1[64][32], b1[64], W2[64][64], b2[64], w3[64], b3 */
#define DPMM_SCREEN_PARAMS 6337
#define DPMM_SCREEN_MAX_TOP 256
typedef enum dpmm_screen_kind { DPMM_SCREEN_SPLIT = 0, DPMM_SCREEN_MERGE = 1 } dpmm_screen_kind;

/* MLP parameters of the context's screen (inference rounds the weights to BF16, biases stay FP32) */
dpmm_status dpmm_screen_set_params(dpmm_ctx* ctx, const float* params);
/* features (rows x 32, nullable) and proxy log ratios (rows, nullable) of every candidate of `kind`
 * for the K clusters whose statistics are on the device; rows with an empty slot are zero */
dpmm_status dpmm_screen_features(dpmm_ctx* ctx, int K, int kind, double alpha, float* features, double* proxy);
/* features + MLP scores + selection: the `top` (<= DPMM_SCREEN_MAX_TOP) best-scored candidate rows
 * whose clusters are all eligible (eligible[K], nonzero = eligible), in ascending row order, into
 * selected[n_selected]; scores (rows, nullable) receives every row's score */
dpmm_status dpmm_screen_select(dpmm_ctx* ctx, int K, int kind, double alpha, const uint8_t* eligible, int top,
                               int32_t* selected, int32_t* n_selected, float* scores);
/* exact split ratios of n (<= DPMM_SCREEN_MAX_TOP) listed clusters / merge ratios of n listed pairs
 * (pairs[2t], pairs[2t+1]); values equal those of dpmm_split_hastings / dpmm_merge_hastings */
dpmm_status dpmm_split_hastings_list(dpmm_ctx* ctx, int K, double alpha, int n, const int32_t* clusters,
                                     double* split_log_hr);
dpmm_status dpmm_merge_hastings_list(dpmm_ctx* ctx, int K, double alpha, int n, const int32_t* pairs,
                                     double* merge_log_hr);
/* MLP on the device without a context (host arrays in and out):
 *   forward: scores[rows] of features[rows x 32] with the deployed (BF16-weight) parameters;
 *   loss_grad: mean squared error (1/rows) sum (z - t)^2 of the FP32 parameters and its gradient;
 *   train: `epochs` passes of shuffled minibatches (the last partial batch of an epoch is dropped),
 *          Adam (beta 0.9 / 0.999, eps 1e-8) at rate lr from the given parameters, updated in place;
 *          epoch_loss[epochs] (nullable) = mean minibatch loss of each epoch. */
dpmm_status dpmm_screen_forward(const float* features, int64_t rows, const float* params, float* scores,
                                int32_t device);
dpmm_status dpmm_screen_loss_grad(const float* features, const float* targets, int32_t rows, const float* params,
                                  float* loss, float* grad, int32_t device);
dpmm_status dpmm_screen_train(const float* features, const float* targets, int64_t rows, int32_t epochs,
                              int32_t batch, float lr, uint64_t seed, float* params, float* epoch_loss,
                              int32_t device);

/* ---- cluster parameter draws on the device (NIW prior, D <= 64) -------------------------------
 * shared_actions::sample_cluster_params (shared_actions.cpp:9-55) with niw::sample_distribution
 * (niw.cpp:82-107) for the cluster and both sub-clusters of each of the K clusters, from the
 * statistics on the device (as the statistics phase, dpmm_merge_statistics and
 * dpmm_compact_statistics leave them); the draws become the label / sub-label parameters directly
 * (what dpmm_set_gaussian_factors would upload).  weights[K]: mixture weights; lr_weights[2K]: the
 * sub-cluster weights; (seed, draw): the Philox stream of this draw; lml (nullable, 3K): each slot's
 * log marginal likelihood (niw.cpp:122-138).  A posterior that is not positive definite gives
 * DPMM_ERR_NOT_PD. */
dpmm_status dpmm_sample_gaussian_params(dpmm_ctx* ctx, int K, uint64_t seed, uint64_t draw, const double* weights,
                                        const double* lr_weights, double* lml);
/* The same for the multinomial prior: multinomial_prior::sample_distribution (multinomial_prior.cpp:
 * 24-49) for every slot, log theta = log of a Dirichlet(alpha + sum x) draw made on the device from
 * the slot's statistics; lr_weights[2K]: the sub-cluster weights (the cluster label phase has no
 * weight term, cudaKernel_multinomial.cu:60-76); lml (nullable, 3K): each slot's log marginal
 * likelihood (multinomial_prior.cpp:56-67). */
dpmm_status dpmm_sample_multinomial_params(dpmm_ctx* ctx, int K, uint64_t seed, uint64_t draw,
                                           const double* lr_weights, double* lml);
/* merge_clusters_to_splittable (shared_actions.cpp:72-86) applied to the device statistics for each
 * (disjoint) pair: cluster index[t] and its l sub-cluster take c_i + c_j, its r sub-cluster c_j. */
dpmm_status dpmm_merge_statistics(dpmm_ctx* ctx, int n, const int32_t* index, const int32_t* new_index);
/* the slot compaction of remove_empty_clusters (local_clusters_actions.cpp:384-419): cluster k takes
 * the statistics of cluster keep[k] (increasing indices) */
dpmm_status dpmm_compact_statistics(dpmm_ctx* ctx, int n_keep, const int32_t* keep);
/* counts of the listed clusters' three slots (as dpmm_create_sufficient_statistics, counts only) */
dpmm_status dpmm_statistics_counts(dpmm_ctx* ctx, int n, const int32_t* indices, int64_t* count);
/* Test seam (no counterpart in the reference): the label-phase parameters of the 3K slots as they are
 * on the device, FP32, with the padded dimension Dp (the next power of two >= max(D, 4)):
 * wt[3K][Dp][Dp] (wt[s][j][i] = W(i, j)), b[3K][Dp] = W^T (mu - shift), c[3K] = -log det Sigma / 2
 * (+ log w for cluster slots), mu[3K][Dp] = mu - shift, where shift is the data mean the points are
 * stored relative to.  Any output may be NULL. */
dpmm_status dpmm_get_gaussian_params(dpmm_ctx* ctx, int K, float* wt, float* b, float* c, float* mu);
/* Test seam (no counterpart in the reference) for the bounded device waits: with stall nonzero every
 * tensor-core kernel issues no tensor-core products (the dense Gaussian and multinomial label kernels,
 * the pruned phase's scans, the sub-label and statistics kernels and their fused pass), so every wait
 * for them runs out after its limit (2 s); the call then returns DPMM_ERR_TIMEOUT after the kernel has
 * waited for the copies it issued and freed its tensor memory, and the context stays usable. */
dpmm_status dpmm_set_wait_test(dpmm_ctx* ctx, int32_t stall);
/* Sub-cluster labels and their statistics in one pass over the points (no counterpart in the
 * reference, whose create_subclusters_labels and statistics are separate passes): with on nonzero the
 * NIW contexts at D = 17 .. 64 that run both on the tensor cores gather each point once for both
 * (k_sub_stats_tc); with on = 0 (the default: on the B200 the two kernels are faster) they run as
 * k_sub_labels_tc and then k_slot_stats_tc.  The sub-cluster log-likelihoods and sub-labels are
 * bit-identical either way; the statistics agree to FP32 rounding (the same products accumulated in
 * 16- instead of 32-point tiles). */
dpmm_status dpmm_set_fused_sub_stats(dpmm_ctx* ctx, int32_t on);
/* Test seam (no counterpart in the reference): log theta[3K][D] of the 3K slots of a multinomial context
 * as the label phases use them (FP32). */
dpmm_status dpmm_get_multinomial_params(dpmm_ctx* ctx, int K, float* log_theta);

/* ---- pruned label phase (NIW prior, D <= 64; no counterpart in the reference) -----------------
 * dpmm_create_clusters_labels (without loglik_out) evaluates, for each chunk of points of one current
 * cluster, only the clusters that an upper bound cannot put more than `margin` nats below the chunk's
 * own cluster; the left-out clusters carry less than K e^-margin of each point's probability and get
 * probability 0 in the same draw.  When the bound keeps more than 2 other clusters per point (early
 * iterations) the dense phase runs and the next 2 label phases stay dense.  margin <= 0 switches it
 * off (default 30).
 * stats: out[0] attempts, out[1] label phases run pruned, out[2] mean kept other clusters per point
 * in those, out[3] the margin, out[4] the last attempt's kept other clusters per point, out[5] its
 * chunks that kept more than 16 (their points are evaluated against every cluster). */
dpmm_status dpmm_set_label_pruning(dpmm_ctx* ctx, double margin);
dpmm_status dpmm_label_pruning_stats(const dpmm_ctx* ctx, double* out);

/* ---- agreement of the labels with a ground truth (verbose mode; replaces the label download and
 * MIToolbox scoring of dp_parallel_sampling.cpp:161-179) ----------------------------------------
 * dpmm_set_ground_truth uploads N int32 ground-truth values once (any values: mapped to dense
 * classes in order of first appearance; NULL clears them).  dpmm_label_agreement counts the (label
 * 1..K, class) pairs of the current labels on the device and scores the K x classes table on the
 * host: nmi = 2 I / (H(ground truth) + H(labels)) (1 when both entropies are 0), vi = H + H - 2 I in
 * nats; either output may be NULL.  dpmm_nmi_from_table is that host part for a caller's K x G
 * row-major table of counts. */
dpmm_status dpmm_set_ground_truth(dpmm_ctx* ctx, const int32_t* gt);
dpmm_status dpmm_label_agreement(dpmm_ctx* ctx, int K, double* nmi, double* vi);
dpmm_status dpmm_nmi_from_table(const int64_t* table, int K, int G, double* nmi, double* vi);

/* Synchronise the context's stream; returns any pending device error. */
dpmm_status dpmm_synchronize(dpmm_ctx* ctx);

/* Diagnostics (no counterpart in the reference, which prints per-iteration wall times only):
 * kernels this library has launched in this process; bytes it copied host->device and
 * device->host; device time per phase of a context (ms[11], calls[11]: labels, sub-labels +
 * statistics, statistics only, split ratios, merge ratios, relabels, parameters, then single kernels
 * inside those phases: the tensor-core label kernel, the pruned label phase's scan and draw kernels,
 * and the sub-cluster statistics kernel over all clusters; its re-launches for a few clusters after
 * moves are not timed) accumulated while timing is on.  enable = 1 / 0 switches
 * timing on / off and clears the counters, -1 only reads them.  Timing adds one event
 * synchronisation per phase and per timed kernel. */
uint64_t dpmm_kernel_launch_count(void);
void dpmm_transfer_bytes(uint64_t* h2d, uint64_t* d2h);
dpmm_status dpmm_phase_times(dpmm_ctx* ctx, int enable, double* ms, int64_t* calls);

/* ------------------------------------------------------------------ whole sampler */

/* Arguments of dp_parallel_sampling_class::dp_parallel (dp_parallel_sampling.h:17-29) and the
 * --params_path JSON keys (global_params.cpp:25-65). */
typedef struct dpmm_run_desc {
    int32_t prior_type;          /* dpmm_prior_type */
    int32_t iterations;          /* iters (default 100) */
    int32_t initial_clusters;    /* init_clusters (default 1) */
    int32_t burnout;             /* burnout_period (default 15 via dp_parallel, 20 via JSON) */
    double alpha;                /* concentration */
    double max_clusters;         /* max_num_of_clusters (<= 0 -> unlimited) */
    double outlier_weight;       /* outlier_mod */
    uint64_t seed;               /* randomSeed (0 -> time based, as the reference) */
    int32_t verbose;             /* use_verbose: log posterior (+ NMI with gt) per iteration */
    int32_t loglik_mode;         /* dpmm_loglik_mode */
    int32_t rng_kind;            /* dpmm_rng_kind */
    int32_t k_max;               /* cluster capacity (0 -> 256) */
    /* hyper_params: NIW (k, m[D], v, psi[D*D]) or multinomial alpha[D]; NULL -> defaults */
    double niw_k, niw_v;
    const double* niw_m;
    const double* niw_psi;
    const double* mult_alpha;
    /* outlier_hyper_params (same layout); NULL -> defaults */
    double out_niw_k, out_niw_v;
    const double* out_niw_m;
    const double* out_niw_psi;
    const double* out_mult_alpha;
    const int32_t* gt;           /* ground-truth labels for NMI (nullable) */
    int32_t device;
    /* learned split/merge screen (no counterpart in the reference; 0 = every candidate exact) */
    int32_t screen_mode;         /* dpmm_screen_mode */
    int32_t screen_top;          /* candidates of each kind sent to the exact ratio (0 -> 16) */
    int32_t screen_sweep_every;  /* every this many iterations all candidates are exact (0 -> 10) */
    float screen_min_recall;     /* the screen is switched off for the rest of the run when the full
                                    sweeps' recall of accepted moves falls below this (0 -> 0.5) */
    const float* screen_params;  /* DPMM_SCREEN_PARAMS floats; required by DPMM_SCREEN_ON */
    int32_t screen_split_min;    /* split candidates are screened only above this many (0 -> 256): the
                                    exact split ratios of K clusters cost one launch of 3K blocks */
    int32_t host_param_draws;    /* nonzero: draw the cluster parameters on the host (FP64, OpenMP) even
                                    where the device draws them (NIW prior, D <= 64, no outlier cluster) */
    float label_prune_margin;    /* pruned label phase margin in nats (0 -> 30; negative -> off) */
    int32_t reserved[1];
} dpmm_run_desc;

typedef enum dpmm_screen_mode {
    DPMM_SCREEN_OFF = 0,         /* every candidate exact (the reference's behaviour) */
    DPMM_SCREEN_ON = 1,          /* exact ratio for the screen's top candidates only */
    DPMM_SCREEN_LOG = 2          /* every candidate exact, and its features + exact ratio logged */
} dpmm_screen_mode;

typedef struct dpmm_model_info dpmm_model_info;

/* Step-wise form of the same run: dpmm_sampler_create does what the constructor, init_model and
 * init_first_clusters do (dp_parallel_sampling.cpp:19-23, 48-87); each dpmm_sampler_step runs
 * n iterations of run_model's loop (dp_parallel_sampling.cpp:139-200), counting iterations from
 * 1 to run->iterations exactly as the reference does (argmax labels and no more split / merge
 * moves in the last 5).  points: N*D point-major, in host or device memory (any address the
 * CUDA runtime can copy from); points_f32 selects float instead of double. */
typedef struct dpmm_sampler dpmm_sampler;
dpmm_status dpmm_sampler_create(const dpmm_run_desc* run, int64_t n, int32_t d, const void* points,
                                int32_t points_f32, dpmm_sampler** out);
/* The same sampler over one shard of a data set split by points across `shard->world` ranks
 * (one process or thread per GPU), all ranks calling with the same run descriptor and seed.  The
 * reference's multi-device code is inactive (cudaKernel.cu:553-554 keeps one device); this is the
 * data-parallel form of its path: per-point work stays on each rank, the per-cluster statistics are
 * summed over the ranks through shard->allreduce, and every host decision (split / merge tests,
 * parameter draws, weights) is then taken identically on every rank from the same numbers with the
 * same seeded generators.  n and points are this rank's shard; labels in the model info are its
 * shard's labels. */
dpmm_status dpmm_sampler_create_sharded(const dpmm_run_desc* run, int64_t n, int32_t d, const void* points,
                                        int32_t points_f32, const dpmm_shard* shard, dpmm_sampler** out);
dpmm_status dpmm_sampler_step(dpmm_sampler* s, int32_t n_iters);
dpmm_status dpmm_sampler_num_clusters(const dpmm_sampler* s, int32_t* k);
/* stream of the sampler's device work (cudaStream_t), for timing with events */
void* dpmm_sampler_stream(const dpmm_sampler* s);
/* the device back-end context the sampler drives (for dpmm_phase_times) */
dpmm_ctx* dpmm_sampler_context(const dpmm_sampler* s);
/* ModelInfo of the iterations run so far (labels copied from the device) */
dpmm_status dpmm_sampler_model_info(dpmm_sampler* s, dpmm_model_info** out);
dpmm_status dpmm_sampler_destroy(dpmm_sampler* s);

/* dp_parallel_sampling_class(N, x, seed, prior) + dp_parallel(...) (dp_parallel_sampling.cpp:19-23,
 * 89-117).  points: N*D point-major. */
dpmm_status dpmm_dp_parallel(const dpmm_run_desc* run, int64_t n, int32_t d, const double* points,
                             dpmm_model_info** out);
/* dp_parallel_sampling_class(npy, json, prior) + dp_parallel_from_file() (dp_parallel_sampling.cpp:25-31,
 * 119-122): reads an N x D .npy (float64 / float32 / int32 / int64 / uint8 / uint16 / bf16 counts
 * read exactly) and the params JSON (accepts // comments). */
dpmm_status dpmm_dp_parallel_from_file(const char* npy_path, const char* params_path, int32_t prior_type,
                                       const dpmm_run_desc* overrides /* nullable */,
                                       dpmm_model_info** out);
/* ---- batches of samplers (no counterpart in the reference, which runs one sampler per process:
 * its init calls cudaDeviceReset, cudaKernel.cu:615) ------------------------------------------------
 * count independent data sets (uneven N, D, K; runs[i], n[i] points of d[i] dimensions at
 * points[i], host FP64 point-major, all on runs[0].device) advanced together one iteration at a
 * time: the host stages of all samplers on a thread pool; the label phase of all NIW data sets of one
 * padded dimension as ONE launch (work list of (data set, block of points) items, replayed from a
 * CUDA graph; the points per block chosen by timing 32 / 64 / 128 on the first iteration).  NIW data
 * sets use the FP32 SIMT label kernel.  Each data set's result is what dpmm_dp_parallel returns. */
typedef struct dpmm_batch dpmm_batch;
dpmm_status dpmm_batch_create(int32_t count, const dpmm_run_desc* runs, const int64_t* n, const int32_t* d,
                              const double* const* points, dpmm_batch** out);
dpmm_status dpmm_batch_step(dpmm_batch* b, int32_t n_iters);
/* out[0] data sets, out[1] padded-dimension groups, out[2] batched label launches, out[3] of them
 * replayed from a CUDA graph, out[4..9] block size chosen for padded dimension 4, 8, 16, 32, 64, 128
 * (0: no such group / not tuned yet) */
dpmm_status dpmm_batch_info(const dpmm_batch* b, int64_t* out);
dpmm_status dpmm_batch_model_info(dpmm_batch* b, int32_t index, dpmm_model_info** out);
dpmm_status dpmm_batch_destroy(dpmm_batch* b);

/* ModelInfo accessors (modelInfo.h:45-56).  Arrays stay valid until dpmm_model_info_free. */
int64_t dpmm_model_info_n(const dpmm_model_info* mi);
const int32_t* dpmm_model_info_labels(const dpmm_model_info* mi);
int32_t dpmm_model_info_num_weights(const dpmm_model_info* mi);
const double* dpmm_model_info_weights(const dpmm_model_info* mi);
int32_t dpmm_model_info_iterations(const dpmm_model_info* mi);
const double* dpmm_model_info_iter_count(const dpmm_model_info* mi);
const double* dpmm_model_info_likelihood_history(const dpmm_model_info* mi);
const double* dpmm_model_info_nmi_history(const dpmm_model_info* mi);  /* NULL without gt */
const int32_t* dpmm_model_info_cluster_count_history(const dpmm_model_info* mi);
/* screen counters of the run (all 0 with the screen off): out[0] split candidates, out[1] split
 * candidates evaluated exactly, out[2] merge candidates (pairs), out[3] pairs evaluated exactly,
 * out[4] full sweeps run, out[5] moves accepted in them, out[6] of those, moves the screen's
 * selection of the same iteration held, out[7] iteration at which the screen was switched off (0:
 * never) */
dpmm_status dpmm_model_info_screen_stats(const dpmm_model_info* mi, int64_t* out);
/* the DPMM_SCREEN_LOG record: rows of (features[32], exact log ratio, kind 0 split / 1 merge,
 * iteration) */
int64_t dpmm_model_info_screen_log_rows(const dpmm_model_info* mi);
const float* dpmm_model_info_screen_log_features(const dpmm_model_info* mi);
const double* dpmm_model_info_screen_log_hr(const dpmm_model_info* mi);
const int8_t* dpmm_model_info_screen_log_kind(const dpmm_model_info* mi);
const int32_t* dpmm_model_info_screen_log_iter(const dpmm_model_info* mi);
/* write {"labels": [...], "weights": [...], "iter_count": [...]} as main.cpp:72-87 does */
dpmm_status dpmm_model_info_write_json(const dpmm_model_info* mi, const char* path);
void dpmm_model_info_free(dpmm_model_info* mi);

#ifdef __cplusplus
}
#endif
#endif /* DPMM_CAPI_H */

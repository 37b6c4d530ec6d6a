// dpmm_internal.h -- context layout shared by the CUDA translation units and the C++ host
// driver.  Not part of the public ABI (include/dpmm_capi.h is).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>
#include <vector>

#include "../../include/dpmm_capi.h"

struct curandStateXORWOW;

namespace dpmm {

// Largest padded dimension of the Gaussian kernels (x held in registers per thread).
constexpr int kMaxGaussDim = 128;
// Largest dimension of the multinomial kernels (count vectors).
constexpr int kMaxMultDim = 4096;
// Points per chunk of the segmented (per-cluster) passes: a multiple of kChunkUnit between
// kChunkUnit and kChunkMax, the smallest that still gives about four waves of blocks.
constexpr int kChunkUnit = 1024;
constexpr int kChunkMax = 4096;
// Pruned label phase: at most kMaxKForPrune clusters; a chunk keeps at most kPrMaxCand other
// clusters before it is evaluated against every cluster.
constexpr int kMaxKForPrune = 256;
// Pruned label phase against the tensor-core dense phase (N = 1e7, D = 64 on the B200): the scan alone
// costs about as much as the dense phase at 7 clusters, and a kept cluster per point about as much as
// 30 clusters of the dense phase.
constexpr int kMinKForPruneTc = 8;
constexpr double kPruneTcRatio = 30.0;
constexpr int kPrMaxCand = 16;

// Learned split/merge screen (dpmm_screen.cu): 32 features per candidate, a 32 -> 64 -> 64 -> 1 MLP
// whose parameters are one FP32 vector W1[64][32], b1[64], W2[64][64], b2[64], w3[64], b3.
constexpr int kScrF = 32;
constexpr int kScrH = 64;
constexpr int kScrOffW1 = 0;
constexpr int kScrOffB1 = kScrOffW1 + kScrH * kScrF;
constexpr int kScrOffW2 = kScrOffB1 + kScrH;
constexpr int kScrOffB2 = kScrOffW2 + kScrH * kScrH;
constexpr int kScrOffW3 = kScrOffB2 + kScrH;
constexpr int kScrOffB3 = kScrOffW3 + kScrH;
constexpr int kScrParams = kScrOffB3 + 1;
constexpr int kScrRec = 10;         // FP64 values per statistics slot
constexpr int kScrMaxTop = 256;     // largest candidate list of one selection / exact-ratio call
static_assert(kScrParams == DPMM_SCREEN_PARAMS, "screen parameter count");
static_assert(kScrF == DPMM_SCREEN_FEATURES, "screen feature count");
static_assert(kScrMaxTop == DPMM_SCREEN_MAX_TOP, "screen list capacity");

int padded_dim(int d);  // 4, 8, 16, 32, 64, 128 (Gaussian); d rounded up to 32 (multinomial)

// Thread-local error message for dpmm_last_error().
void set_error(const std::string& msg);
dpmm_status fail(dpmm_status s, const std::string& msg);
dpmm_status cuda_status(cudaError_t e, const char* what);

#define DPMM_CUDA_TRY(expr)                                              \
    do {                                                                 \
        cudaError_t _e = (expr);                                         \
        if (_e != cudaSuccess) return ::dpmm::cuda_status(_e, #expr);    \
    } while (0)

// process-wide diagnostics: kernels launched, bytes copied host->device / device->host
extern std::atomic<uint64_t> g_launches, g_h2d_bytes, g_d2h_bytes;

#define DPMM_LAUNCHED()                                                        \
    do {                                                                       \
        ::dpmm::g_launches.fetch_add(1, std::memory_order_relaxed);            \
        DPMM_CUDA_TRY(cudaGetLastError());                                     \
    } while (0)

enum Phase { PH_LABELS = 0, PH_SUB_STATS = 1, PH_STATS = 2, PH_SPLIT_HR = 3, PH_MERGE_HR = 4, PH_RELABEL = 5,
             PH_PARAMS = 6, PH_LABEL_KERNEL = 7, PH_PRUNE_SCAN = 8, PH_PRUNE_DRAW = 9, PH_SLOT_STATS = 10,
             PH_COUNT = 11 };

#define DPMM_TRY(expr)                         \
    do {                                       \
        dpmm_status _s = (expr);               \
        if (_s != DPMM_OK) return _s;          \
    } while (0)

// How a phase obtains its uniforms.
struct RngArgs {
    int kind;                      // dpmm_rng_kind
    uint64_t seed;
    uint64_t ctr;                  // Philox draw counter (one per phase call)
    curandStateXORWOW* states;     // per point (compat mode)
    const float* ucaller;          // device copy of caller uniforms (or nullptr)
    int64_t offset;                // global index of the context's first point (sharded data sets)
};

}  // namespace dpmm

// Device-side state of one sampler.  All buffers are allocated at dpmm_create at capacity.
struct dpmm_ctx {
    int device = 0;
    int64_t N = 0;
    int D = 0;
    int Dp = 0;                    // padded dimension used by the kernels
    int prior = 0;
    int k_max = 0;
    int rng_kind = 0;
    uint64_t seed = 0;
    uint64_t philox_ctr = 0;
    int ll_mode = 0;
    int verbose = 0;
    bool points_ready = false;
    bool tc_ok = false;            // tensor-core kernel usable for this shape
    cudaStream_t stream = nullptr;
    int num_sms = 0;               // streaming multiprocessors of the device (persistent grids)

    // points: N x Dp row-major FP32.  Gaussian points are stored shifted by `shift`
    // (their FP64 mean), which leaves every log-likelihood unchanged and keeps the FP32
    // contraction and the scatter accumulation away from cancellation.
    float* d_x = nullptr;
    std::vector<double> shift;
    double* d_gshift = nullptr;    // shift on the device (D doubles)

    int32_t* d_labels = nullptr;
    int32_t* d_sub = nullptr;
    curandStateXORWOW* d_curand = nullptr;

    // cluster parameters: 3 slots per cluster (3k: cluster, 3k+1: l, 3k+2: r)
    int K_params = 0;
    float* d_Wt = nullptr;         // [3*k_max][Dp][Dp], Wt[j][i] = W(i, j)  (Gaussian)
    float* d_b = nullptr;          // [3*k_max][Dp], b = W^T (mu - shift)   (Gaussian)
    float* d_c = nullptr;          // [3*k_max]: -logdet/2 + log w (slot 3k), -logdet/2 (sub slots);
                                   // 0 for the multinomial prior (no weight term)
    float* d_lrw = nullptr;        // [2*k_max] log lr_weights
    float* d_mu = nullptr;         // [3*k_max][Dp], mu - shift (Gaussian) / log theta (multinomial)
    uint8_t* d_Btc = nullptr;      // tensor-core B operand: per pair of clusters a 32 KB split-bf16,
                                   // K-major 128-byte-swizzled tile (Gaussian, Dp = 32 or 64)
    uint8_t* d_Atc = nullptr;      // tensor-core A operand: per 128 points the same 32 KB split-bf16
                                   // swizzled tile, packed once when the points are uploaded
    uint8_t* d_Bsub = nullptr;     // tensor-core sub-label phase: per cluster its two sub-cluster
                                   // factors as one 32 KB split-bf16 swizzled B tile
    uint8_t* d_Amult = nullptr;    // multinomial tensor-core label phase: the counts as BF16, per
                                   // (128-point tile, 64-category block) one 16 KB swizzled tile
    uint8_t* d_Bmult = nullptr;    // ... log theta of the clusters as three BF16 parts per block
    bool mult_tc_ok = false;       // every count is held exactly by BF16 (checked at upload)
    int mult_tc_K = -1;            // clusters packed in d_Bmult (-1: stale)
    float* d_rbuf = nullptr;       // tensor-core label phase: r cluster-major [k_max][N]
    float* d_rpart = nullptr;      // per point and half: running max, sum of exp (or best, arg) [4][N]
    std::vector<float> h_param_stage;

    // label-ordered permutation of the points and the per-cluster chunk table
    int nblk_hist = 0;
    int32_t* d_perm = nullptr;
    int32_t* d_blk_hist = nullptr; // [nblk_hist][k_max]
    int32_t* d_seg = nullptr;      // [k_max + 1] segment starts
    int32_t* d_chunk = nullptr;    // [max_chunks][3] (cluster, start, len)
    int32_t* d_nchunks = nullptr;
    int max_chunks = 0;
    int chunk_len = dpmm::kChunkMax;   // points per chunk (see kChunkUnit)
    int perm_K = -1;               // K the permutation was built for (-1: stale)

    // statistics: chunk partials (FP64) and per-slot results in original coordinates
    double* d_part = nullptr;      // [max_chunks][2][stat_len]
    double* d_stats = nullptr;     // [3*k_max][stat_len]: count, sum[D], S[D*D] (col-major)
    double* d_stats_tmp = nullptr; // same size: the target of a compaction (then swapped)
    double* d_logw = nullptr;      // [k_max] log mixture weights of the device parameter draw
    int stat_len = 0;              // 1 + D + D*D (Gaussian) / 1 + D (multinomial)
    int stats_K = -1;              // clusters 0..stats_K-1 have statistics on the device ...
    std::vector<uint8_t> stats_ok; // ... and stats_ok[k] says whether they are still current
    uint8_t* d_mask = nullptr;     // [k_max] clusters selected for a partial recompute

    // uniforms / random bits supplied by the caller, staged on the device
    float* d_u = nullptr;          // 2N
    uint32_t* d_bits = nullptr;    // N
    int32_t* d_remap = nullptr;    // [k_max + 2] relabel table
    int32_t* d_aux = nullptr;      // small scratch (counts)
    double* d_r64 = nullptr;       // N doubles (FP64 test seams)
    double* d_dbl_scratch = nullptr; // k_max-sized FP64 scratch

    // priors + Hastings (FP64)
    bool prior_set = false;
    double prior_k = 0, prior_v = 0;
    double prior_logdet = 0;       // log det psi0 (NIW)
    bool prior_identity = false;   // NIW prior with m0 = 0 and psi0 = I
    double* d_prior = nullptr;     // NIW: m[D], psi[D*D]; multinomial: alpha[D]
    // runs with an outlier cluster (local_clusters_actions.cpp:48-79, 341-371): cluster 0 has its own
    // prior (its slots are drawn from this one's posterior), cluster 1's parameters are not redrawn
    int outlier_layout = 0;
    double prior2_k = 0, prior2_v = 0, prior2_logdet = 0;
    double* d_prior2 = nullptr;    // like d_prior
    uint8_t* d_prior_sel = nullptr;  // [k_max] 1: the cluster's slots use the second prior
    double* d_cbase = nullptr;     // [3*k_max] -log det Sigma / 2 of each slot's current parameters (NIW)
    double* d_linalg = nullptr;    // scratch of dpmm_inverse_matrix / dpmm_multiply_for_inverse_wishart
    size_t linalg_bytes = 0;       // (grown on demand)
    double* d_lml = nullptr;       // [3*k_max]
    double* d_split_hr = nullptr;  // [k_max]
    double* d_merge_hr = nullptr;  // [k_max*k_max]
    double* d_post_logdet = nullptr; // [3*k_max]
    // learned split/merge screen (dpmm_screen.cu)
    double* d_scr_rec = nullptr;   // [3*k_max][kScrRec] per-slot posterior quantities
    double* d_scr_vec = nullptr;   // [3*k_max][2][D]: NIW m', diag(psi'); Dirichlet a'/sum a', a'
    float* d_scr_linv = nullptr;   // [k_max][D][D] inverse Cholesky factor of each cluster's psi' (NIW)
    float* d_scr_feat = nullptr;   // [rows][kScrF], rows = max(k_max, k_max (k_max - 1) / 2)
    double* d_scr_prox = nullptr;  // [rows] proxy log Hastings ratio (feature 2 before scaling)
    float* d_scr_score = nullptr;  // [rows] MLP scores
    float* d_scr_w = nullptr;      // [kScrParams] FP32 parameters
    float* d_scr_wdep = nullptr;   // [kScrParams] deployed: weights rounded to BF16, biases FP32
    uint8_t* d_scr_elig = nullptr; // [k_max] eligible clusters
    int32_t* d_scr_sel = nullptr;  // [kScrMaxTop + 1] selected rows, then their count
    int32_t* d_scr_list = nullptr; // [2 * kScrMaxTop] clusters / pairs of an exact-ratio list
    int32_t* d_scr_slots = nullptr;// [3 * kScrMaxTop] slots whose lml the list needs
    double* d_scr_hr = nullptr;    // [kScrMaxTop] exact ratios of the list
    bool scr_params_set = false;

    // pruned label phase (dpmm_kernels.cu: k_prune_*): NIW prior, padded dimension <= 64
    float prune_margin = 30.f;     // nats; <= 0 switches the pruned phase off
    int prune_wait = 0;            // label phases to run dense before the next attempt
    int64_t prune_tries = 0, prune_used = 0;
    double prune_extra = 0;        // sum over used phases of kept other clusters per point
    double prune_last_extra = 0;   // the last attempt's kept other clusters per point
    int64_t prune_last_over = 0;   // ... and its chunks over the candidate-list capacity
    float* d_prune_rh = nullptr;   // [N] r of each point's current cluster, permutation order
    int32_t* d_prune_cand = nullptr; // [max_chunks][17] kept clusters per chunk
    int32_t* d_prune_list = nullptr; // [max_chunks] the chunks that kept other clusters, ascending
    float* d_prune_lam = nullptr;  // [KP], KP = min(k_max, 256) (the pruned phase takes K <= 256)
    float* d_prune_M = nullptr;    // [KP][KP]
    float* d_prune_V = nullptr;    // [KP][KP][Dp] point-bound directions
    float* d_prune_beta = nullptr; // [KP][KP]
    // ground truth for the label agreement scores (dpmm_set_ground_truth)
    int32_t* d_gt = nullptr;       // [N] dense ground-truth ids 0..gt_G-1
    int gt_G = 0;
    bool sub_err_pending = false;  // the sub-label kernel's error word awaits the statistics launch's sync
    unsigned long long* d_ctab = nullptr;   // [k_max][gt_G] contingency counts
    unsigned long long* d_prune_cnt = nullptr;   // [2]
    double* h_pinned = nullptr;    // pinned staging for D2H of results
    size_t h_pinned_bytes = 0;

    int stall_tc_mma = 0;          // test seam (dpmm_set_wait_test): tensor-core kernels issue no products
    int fuse_sub_stats = 0;        // sub-labels and statistics in one pass (dpmm_set_fused_sub_stats)

    // sharding by points (dpmm_set_shard): the aggregates are summed over the ranks by `allreduce`
    int shard_world = 1, shard_rank = 0;
    int64_t pt_offset = 0;         // global index of this shard's first point
    int64_t n_total = 0;           // points of all shards (N when not sharded)
    dpmm_allreduce_fn allreduce = nullptr;
    void* allreduce_user = nullptr;
    double* d_xchg = nullptr;      // staging of the exchanges: [3*k_max*stat_len] doubles (sharded only)
    size_t xchg_len = 0;

    // events for phase timing (bench): device time per phase while `timing` is set
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t kev0 = nullptr, kev1 = nullptr;   // one kernel inside a phase (PH_LABEL_KERNEL)
    bool timing = false;
    double phase_ms[dpmm::PH_COUNT] = {0};
    int64_t phase_calls[dpmm::PH_COUNT] = {0};
};

namespace dpmm {
// Records device time of one phase on the context's stream when timing is enabled.
struct PhaseTimer {
    dpmm_ctx* c;
    int ph;
    PhaseTimer(dpmm_ctx* ctx, int phase) : c(ctx), ph(phase)
    {
        if (c && c->timing) cudaEventRecord(c->ev0, c->stream);
    }
    ~PhaseTimer()
    {
        if (!c || !c->timing) return;
        cudaEventRecord(c->ev1, c->stream);
        if (cudaEventSynchronize(c->ev1) == cudaSuccess) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, c->ev0, c->ev1);
            c->phase_ms[ph] += ms;
            c->phase_calls[ph] += 1;
        }
    }
};

// The same for one kernel launch inside a phase, with its own events.
struct KernelTimer {
    dpmm_ctx* c;
    int ph;
    KernelTimer(dpmm_ctx* ctx, int phase) : c(ctx), ph(phase)
    {
        if (c && c->timing) cudaEventRecord(c->kev0, c->stream);
    }
    ~KernelTimer()
    {
        if (!c || !c->timing) return;
        cudaEventRecord(c->kev1, c->stream);
        if (cudaEventSynchronize(c->kev1) == cudaSuccess) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, c->kev0, c->kev1);
            c->phase_ms[ph] += ms;
            c->phase_calls[ph] += 1;
        }
    }
};
}  // namespace dpmm

namespace dpmm {
// One data set's share of a batched label phase (see launch_labels_batched)
struct LabelJob {
    const float* x;
    int64_t N;
    const float* Wt;
    const float* b;
    const float* c;
    int K;
    int final_;
    RngArgs rng;
    int32_t* labels;
};

// kernel launchers (dpmm_kernels.cu)
// label phase of several Gaussian data sets of padded dimension Dp in one launch: nitems blocks of
// P points, item (job, block); kmax: the largest K of the jobs
dpmm_status launch_labels_batched(int Dp, int P, const LabelJob* d_jobs, const int2* d_items, int nitems, int kmax,
                                  cudaStream_t st);
size_t gauss_label_smem_bytes(int DP, int P, int K);
// a context's label phase as a batch job (dpmm_capi.cu)
dpmm_status make_label_job(dpmm_ctx* c, int K, int final_, LabelJob* job);
dpmm_status launch_init_curand(dpmm_ctx* c);
dpmm_status launch_labels_init(dpmm_ctx* c, int initial_clusters, double outlier_mod, const float* d_u);
dpmm_status launch_sub_labels_init(dpmm_ctx* c, const float* d_u);
dpmm_status launch_draw_uniforms(dpmm_ctx* c, float* d_u);   // 2N uniforms of the next draw
dpmm_status launch_cluster_labels(dpmm_ctx* c, int K, int final_, const float* d_u, float* d_rout);
// the pruned label phase; *used = false when it declined (the caller then runs the dense phase)
dpmm_status launch_cluster_labels_pruned(dpmm_ctx* c, int K, int final_, const float* d_u, bool* used);
dpmm_status build_permutation(dpmm_ctx* c, int K);
dpmm_status launch_sub_labels_and_stats(dpmm_ctx* c, int K, const float* d_u, float* d_rout, bool draw,
                                        const uint8_t* d_mask = nullptr);
dpmm_status launch_stats_finalize(dpmm_ctx* c, int K, const uint8_t* d_mask);
// recompute the statistics of every cluster k < K that is not current (all of them if none is)
dpmm_status ensure_stats(dpmm_ctx* c, int K);
void invalidate_stats(dpmm_ctx* c);
void invalidate_stats(dpmm_ctx* c, int k);
dpmm_status launch_relabel(dpmm_ctx* c, int mode, int K, const int32_t* h_table, int table_len,
                           const uint32_t* d_bits);
dpmm_status launch_sub_count(dpmm_ctx* c, int32_t* h_l, int32_t* h_r);
dpmm_status launch_loglik_gauss_one(dpmm_ctx* c, double* d_r);
dpmm_status launch_loglik_mult_one(dpmm_ctx* c, double* d_r);
dpmm_status launch_sample_log_cat(dpmm_ctx* c, int K, const double* d_r, const float* d_u);
dpmm_status launch_sample_log_cat_sub(dpmm_ctx* c, int m, const double* d_r, const int32_t* d_idx,
                                      const double* d_lrw, const float* d_u);
// Hastings (dpmm_hastings.cu)
dpmm_status launch_split_hastings(dpmm_ctx* c, int K, double alpha);
dpmm_status launch_merge_hastings(dpmm_ctx* c, int K, double alpha);
// log marginal likelihood of the 3K slots of the statistics as they are on the device (no
// recompute from the labels), copied to lml[3K]
dpmm_status slot_lml_as_is(dpmm_ctx* c, int K, double* lml);
// learned screen (dpmm_screen.cu)
dpmm_status launch_screen_features(dpmm_ctx* c, int K, int kind, double alpha);
dpmm_status launch_screen_select(dpmm_ctx* c, int K, int kind, double alpha, int top);
// tensor-core label kernel (dpmm_tc.cu); returns DPMM_ERR_INVALID_ARG when the shape is unsupported
bool tc_supported(const dpmm_ctx* c, int K);
dpmm_status launch_cluster_labels_tc(dpmm_ctx* c, int K, int final_, const float* d_u, float* d_rout);
dpmm_status pack_tc_params(dpmm_ctx* c, int K);
dpmm_status pack_tc_points(dpmm_ctx* c);   // A operand from the uploaded points
// multinomial label phase on the tensor cores (dpmm_tc.cu)
bool tc_mult_supported(const dpmm_ctx* c, int K);
size_t mult_tc_a_bytes(int64_t N, int D);
size_t mult_tc_b_bytes(int k_max, int D);
dpmm_status pack_mult_tc_points(dpmm_ctx* c);          // the counts as BF16 tiles (at upload)
dpmm_status pack_mult_tc_params(dpmm_ctx* c, int K);   // log theta as three BF16 parts
dpmm_status launch_mult_labels_tc(dpmm_ctx* c, int K, int final_, const float* d_u, float* d_rout);
size_t tc_param_bytes(int k_max);          // B tiles + bias records for k_max clusters
// tensor-core sub-label kernel (dpmm_tc.cu): draws the sub-labels only (statistics separately)
bool tc_sub_supported(const dpmm_ctx* c);
// defer_check: its error word is read by the statistics launch that follows (one sync for both)
dpmm_status launch_sub_labels_tc(dpmm_ctx* c, RngArgs r, float* d_rout, bool defer_check = false);
// pass 1 of the pruned label phase on the tensor cores (dpmm_tc.cu; Dp = 32 or 64, packed B tiles)
bool tc_scan_supported(const dpmm_ctx* c, int K);
dpmm_status launch_prune_scan_tc(dpmm_ctx* c, int K, int32_t* d_err);
// sub-cluster statistics (sub-labels given) on the tensor cores (dpmm_tc.cu; Dp = 32 or 64)
bool tc_stats_supported(const dpmm_ctx* c);
dpmm_status launch_slot_stats_tc(dpmm_ctx* c, const uint8_t* d_mask);
bool tc_sub_stats_supported(const dpmm_ctx* c);
dpmm_status launch_sub_stats_tc(dpmm_ctx* c, RngArgs r, float* d_rout);

RngArgs rng_args(dpmm_ctx* c, const float* d_ucaller);
// In-place sum over the shards of `count` doubles at d_buf (device, written on the context's stream);
// nothing to do for a context that is not sharded.
dpmm_status shard_allreduce(dpmm_ctx* c, double* d_buf, int64_t count);
// statistics of all points together (niw::create_sufficient_statistics over the whole data set)
dpmm_status all_points_stats(dpmm_ctx* c, int64_t* count, double* sum, double* S);
dpmm_status launch_fill_labels(dpmm_ctx* c, int32_t value);
}  // namespace dpmm

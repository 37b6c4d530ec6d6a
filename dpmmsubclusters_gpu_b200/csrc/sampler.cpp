// sampler.cpp -- host driver of the Chang & Fisher sub-cluster split/merge sampler running
// on the device back-end of dpmm_capi.  It keeps the reference's iteration semantics:
//   dp_parallel_sampling_class::dp_parallel / init_model / init_first_clusters / run_model
//                                                   (dp_parallel_sampling.cpp:19-206)
//   local_clusters_actions::group_step and the steps it calls (local_clusters_actions.cpp:14-490)
//   shared_actions::sample_cluster_params / create_splittable_from_params /
//                   merge_clusters_to_splittable / should_merge (shared_actions.cpp:9-111)
//   niw / multinomial_prior posterior, lml, sampling (priors/niw.cpp, priors/multinomial_prior.cpp)
//   global_params JSON keys and defaults (global_params.h:37-78, global_params.cpp:8-106)
// What moved to the device: label / sub-label draws, sufficient statistics, the split ratios of
// all clusters (one launch) and the merge ratios of all pairs (one launch).  Host FP64 keeps the
// per-cluster bookkeeping, parameter draws and the sequential accept/reject decisions.
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <ctime>
#include <fstream>
#include <map>
#include <memory>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "dpmm_internal.h"
#include "io.h"
#include "linalg.h"

namespace dpmm {
namespace host {

struct Hyper {               // niw_hyperparams {k, m, v, psi} / multinomial_hyper {alpha}
    bool outlier = false;        // the outlier cluster's prior (outlier_hyper_params)
    double k = 0, v = 0;
    std::vector<double> m, psi;
    std::vector<double> chol;    // lower Cholesky factor of psi (NIW)
    double logdet = 0;           // log det psi (NIW)
    std::vector<double> alpha;
};

struct Stats {               // niw_sufficient_statistics / multinomial_sufficient_statistics
    int64_t N = 0;
    std::vector<double> sum, S;
};

struct Dist {                // mv_gaussian (precision factor form) / multinomial_dist
    std::vector<double> mu, W;   // inv_sigma = W W^T
    double logdet_sigma = 0;
    std::vector<double> log_theta;
};

struct ClusterParams {       // cluster_parameters (ds.h:39-118)
    Hyper prior, post;
    Dist dist;
    Stats stats;
};

struct Splittable {          // splittable_cluster_params (ds.h:122-214) + local_cluster counts
    ClusterParams c, l, r;
    double lrw[2] = {0.5, 0.5};
    bool splittable = false;
    std::vector<std::pair<bool, double>> hist;
    int64_t points_count = 0;
};

struct Config {
    int prior = DPMM_PRIOR_GAUSSIAN;
    int iterations = 100, initial_clusters = 1, burnout = 15;
    int argmax_sample_stop = 5, split_stop = 5;
    double alpha = 10.0, max_clusters = 1e300, outlier_mod = 0.0;
    uint64_t seed = 0;
    bool verbose = false;
    Hyper hyper, outlier_hyper;
    std::vector<int32_t> gt;
    int loglik_mode = DPMM_LL_AUTO, rng_kind = DPMM_RNG_PHILOX, k_max = 0, device = 0;
    // learned split/merge screen (no counterpart in the reference)
    int screen_mode = DPMM_SCREEN_OFF, screen_top = 16, screen_sweep = 10, screen_split_min = 256;
    double screen_min_recall = 0.5;
    std::vector<float> screen_params;
    bool host_param_draws = false;   // draw the NIW parameters on the host even where the device can
    double label_prune_margin = 30.0;  // pruned label phase margin (<= 0: off)
};

// screen counters and the DPMM_SCREEN_LOG record of a run
struct ScreenRecord {
    int64_t split_cand = 0, split_exact = 0, merge_cand = 0, merge_exact = 0;
    int64_t sweeps = 0, sweep_accepts = 0, sweep_hits = 0, disabled_at = 0;
    std::vector<float> log_features;
    std::vector<double> log_hr;
    std::vector<int8_t> log_kind;
    std::vector<int32_t> log_iter;
};

class Sampler {
public:
    // N: this context's points; the data set's total is ctx->n_total (larger for a shard)
    Sampler(const Config& cfg, dpmm_ctx* ctx, int64_t N, int D)
        : cfg_(cfg), ctx_(ctx), N_(N), Ntot_(ctx->n_total), D_(D), gen_((unsigned long)cfg.seed)
    {
        // device-resident parameters: the draws run on the device from the device statistics, the
        // host keeps counts only (and the outlier cluster's full statistics, for its split ratio)
        dev_ = device_draws(cfg, D);
        cfg_.outlier_hyper.outlier = true;
    }

    // device draws for NIW at D <= 64 and the multinomial prior; runs with an outlier cluster draw on
    // the host (the device supports them -- dpmm_set_outlier_prior_*, dpmm_set_cluster_priors -- but
    // whole runs were not shown to match the host draws' outcomes: their course is dominated by the
    // reference's never-redrawn cluster 1)
    static bool device_draws(const Config& cfg, int D)
    {
        return !cfg.host_param_draws && !(cfg.outlier_mod > 0) && (cfg.prior == DPMM_PRIOR_MULTINOMIAL || D <= 64);
    }

    // init_model + init_first_clusters, then iterations first..first+n-1 of run_model
    dpmm_status init() { return init_first_clusters(); }
    dpmm_status step(int n, dpmm_model_info* mi);
    dpmm_status finish(dpmm_model_info* mi);
    int num_clusters() const { return (int)clusters_.size(); }
    bool running() const { return iter_ < cfg_.iterations; }
    dpmm_ctx* context() const { return ctx_; }

    // one iteration in stages, for drivers that run the label phase of many samplers together
    struct IterState {
        int i = 0;
        bool final_ = false, no_more_splits = false;
        std::chrono::steady_clock::time_point t0;
    };
    IterState begin_iteration();
    dpmm_status stage_params();
    dpmm_status stage_rest(bool no_more_splits, bool final_);
    dpmm_status end_iteration(const IterState& st, dpmm_model_info* mi);
    const ScreenRecord& screen_record() const { return scr_; }
    int iteration() const { return iter_; }

private:
    // ----------------------------------------------------------------- prior maths
    void finish_hyper(Hyper& h) const
    {
        if (cfg_.prior != DPMM_PRIOR_GAUSSIAN) return;
        if (la::cholesky(h.psi.data(), D_, h.chol)) h.logdet = la::logdet_from_chol(h.chol, D_);
        else h.logdet = NAN;
    }

    Hyper posterior(const Hyper& p, const Stats& s) const   // niw.cpp:23-49, multinomial_prior.cpp:12-22
    {
        if (s.N == 0) return p;
        Hyper h;
        if (cfg_.prior == DPMM_PRIOR_MULTINOMIAL) {
            h.alpha.resize(D_);
            for (int d = 0; d < D_; ++d) h.alpha[d] = p.alpha[d] + s.sum[d];
            return h;
        }
        const int D = D_;
        h.k = p.k + (double)s.N;
        h.v = p.v + (double)s.N;
        h.m.resize(D);
        for (int i = 0; i < D; ++i) h.m[i] = (p.m[i] * p.k + s.sum[i]) / h.k;
        h.psi.resize((size_t)D * D);
        for (int j = 0; j < D; ++j)
            for (int i = 0; i <= j; ++i) {      // upper triangle, mirrored (selfadjointView<Upper>)
                size_t ij = (size_t)j * D + i;
                double tm = p.v * p.psi[ij] + p.k * p.m[i] * p.m[j];
                double v = (tm - h.k * h.m[i] * h.m[j] + s.S[ij]) / h.v;
                h.psi[ij] = v;
                h.psi[(size_t)i * D + j] = v;
            }
        finish_hyper(h);
        return h;
    }

    static double lmvgamma(double x, int D)    // utils.cpp:94-102
    {
        double r = D * (D - 1) / 4.0 * std::log(M_PI);
        for (int d = 1; d <= D; ++d) r += std::lgamma(x + (1 - d) / 2.0);
        return r;
    }

    double lml(const Hyper& p, const Hyper& q, const Stats& s) const   // niw.cpp:122-138 / multinomial_prior.cpp:56-67
    {
        if (cfg_.prior == DPMM_PRIOR_MULTINOMIAL) {
            double s0 = 0, sp = 0, v = 0;
            for (int d = 0; d < D_; ++d) {
                s0 += p.alpha[d];
                sp += q.alpha[d];
                v += std::lgamma(q.alpha[d]) - std::lgamma(p.alpha[d]);
            }
            return std::lgamma(s0) - std::lgamma(sp) + v;
        }
        const int D = D_;
        return -(double)s.N * D * 0.5 * std::log(M_PI) + lmvgamma(q.v / 2.0, D) - lmvgamma(p.v / 2.0, D) +
               (p.v / 2.0) * (D * std::log(p.v) + p.logdet) - (q.v / 2.0) * (D * std::log(q.v) + q.logdet) +
               (D / 2.0) * std::log(p.k / q.k);
    }

    Stats aggregate(const Stats& a, const Stats& b) const   // niw.cpp:140-148
    {
        Stats o;
        o.N = a.N + b.N;
        o.sum.resize(a.sum.size());
        for (size_t i = 0; i < a.sum.size(); ++i) o.sum[i] = a.sum[i] + b.sum[i];
        o.S.resize(a.S.size());
        for (size_t i = 0; i < a.S.size(); ++i) o.S[i] = a.S[i] + b.S[i];
        return o;
    }

    Stats empty_stats() const
    {
        Stats s;
        s.sum.assign(D_, 0.0);
        if (cfg_.prior == DPMM_PRIOR_GAUSSIAN) s.S.assign((size_t)D_ * D_, 0.0);
        return s;
    }

    // niw::sample_distribution (niw.cpp:82-107) in factor form: with v psi = L L^T and A the
    // Bartlett factor (A_ii = sqrt(chi2(v - i)), A_ij ~ N(0,1) below the diagonal, the draw of
    // stats::rinvwish2), the precision is W W^T with W = L^-T A ~ Wishart(v, (v psi)^-1); then
    // Sigma = (L A^-T)(L A^-T)^T, log det Sigma = 2 sum log L_ii - 2 sum log A_ii, and
    // mu = m + L A^-T z / sqrt(k), z ~ N(0, I).  multinomial_prior::sample_distribution
    // (multinomial_prior.cpp:24-49): log of a Dirichlet(alpha) draw.
    Dist sample(const Hyper& h, std::mt19937_64& g) const
    {
        Dist d;
        if (cfg_.prior == DPMM_PRIOR_MULTINOMIAL) {
            std::vector<double> x(D_);
            double s = 0;
            for (int i = 0; i < D_; ++i) {
                std::gamma_distribution<double> ga(h.alpha[i], 1.0);
                x[i] = ga(g);
                s += x[i];
            }
            d.log_theta.resize(D_);
            for (int i = 0; i < D_; ++i) d.log_theta[i] = std::log(x[i] / s);
            return d;
        }
        const int D = D_;
        std::vector<double> L((size_t)D * D);
        const double sv = std::sqrt(h.v);
        for (size_t e = 0; e < L.size(); ++e) L[e] = h.chol[e] * sv;
        std::normal_distribution<double> nd(0.0, 1.0);
        std::vector<double> A((size_t)D * D, 0.0);
        for (int i = 1; i < D; ++i)
            for (int j = 0; j < i; ++j) A[(size_t)j * D + i] = nd(g);
        for (int i = 0; i < D; ++i) {
            std::chi_squared_distribution<double> cs(h.v - i);
            A[(size_t)i * D + i] = std::sqrt(cs(g));
        }
        // W = L^-T A: solve L^T W = A by back substitution over rows, all columns at once (A is
        // lower-triangular); each update is a contiguous AXPY over a row of W, with the terms
        // subtracted in the same order (q ascending) as a per-column solve
        std::vector<double> Wr((size_t)D * D);   // row-major: Wr[i * D + c] = W(i, c)
        for (int i = D - 1; i >= 0; --i) {
            double* wi = &Wr[(size_t)i * D];
            for (int c = 0; c < D; ++c) wi[c] = i >= c ? A[(size_t)c * D + i] : 0.0;
            for (int q = i + 1; q < D; ++q) {
                const double f = L[(size_t)i * D + q];   // L(q, i)
                const double* wq = &Wr[(size_t)q * D];
                for (int c = 0; c < D; ++c) wi[c] -= f * wq[c];
            }
            const double dii = L[(size_t)i * D + i];
            for (int c = 0; c < D; ++c) wi[c] /= dii;
        }
        d.W.resize((size_t)D * D);
        for (int c = 0; c < D; ++c)
            for (int i = 0; i < D; ++i) d.W[(size_t)c * D + i] = Wr[(size_t)i * D + c];
        double ldl = 0, lda = 0;
        for (int i = 0; i < D; ++i) {
            ldl += std::log(L[(size_t)i * D + i]);
            lda += std::log(A[(size_t)i * D + i]);
        }
        d.logdet_sigma = 2 * ldl - 2 * lda;
        // mu = m + L y / sqrt(k) with A^T y = z
        std::vector<double> z(D), y(D);
        for (int i = 0; i < D; ++i) z[i] = nd(g);
        for (int i = D - 1; i >= 0; --i) {
            double s = z[i];
            for (int q = i + 1; q < D; ++q) s -= A[(size_t)i * D + q] * y[q];
            y[i] = s / A[(size_t)i * D + i];
        }
        d.mu.resize(D);
        const double isk = 1.0 / std::sqrt(h.k);
        for (int i = 0; i < D; ++i) {
            double s = 0;
            for (int q = 0; q <= i; ++q) s += L[(size_t)q * D + i] * y[q];
            d.mu[i] = h.m[i] + s * isk;
        }
        return d;
    }

    // per-draw generator: seeded from (seed, draw counter) so draws can run in parallel and
    // stay reproducible for a given seed
    std::mt19937_64 draw_gen(uint64_t id) const
    {
        std::seed_seq sq{(uint32_t)cfg_.seed, (uint32_t)(cfg_.seed >> 32), (uint32_t)id, (uint32_t)(id >> 32)};
        return std::mt19937_64(sq);
    }

    std::vector<double> dirichlet(const std::vector<double>& a)   // distributions_util/dirichlet.h:39-48
    {
        std::vector<double> x(a.size());
        double s = 0;
        for (size_t i = 0; i < a.size(); ++i) {
            std::gamma_distribution<double> g(a[i], 1.0);
            x[i] = g(gen_);
            s += x[i];
        }
        for (double& v : x) v /= s;
        return x;
    }

    double uniform()
    {
        std::uniform_real_distribution<double> u(0, 1);
        return u(gen_);
    }

    std::vector<std::pair<bool, double>> fresh_hist() const
    {
        return std::vector<std::pair<bool, double>>(cfg_.burnout + 5, std::make_pair(false, 0.0));
    }

    // ----------------------------------------------------------------- device glue
    dpmm_status upload_params(const std::vector<double>& weights);
    dpmm_status update_suff_stats_posterior(const std::vector<int32_t>& indices);
    dpmm_status host_stats_posterior(const std::vector<int32_t>& indices);
    dpmm_status sync_prior_select();
    void sample_cluster_params_all();
    dpmm_status sample_clusters();
    dpmm_status sample_clusters_device();
    void mixture_weights();
    dpmm_status reset_bad_clusters();
    dpmm_status check_and_split(bool final_, std::vector<int32_t>& all_indices);
    dpmm_status check_and_merge(bool final_);
    dpmm_status remove_empty_clusters();
    dpmm_status group_step(bool no_more_splits, bool final_);
    dpmm_status init_first_clusters();
    dpmm_status calculate_posterior(double* out);
    Config cfg_;
    dpmm_ctx* ctx_;
    int64_t N_;      // points of this context (its shard)
    int64_t Ntot_;   // points of the whole data set
    int D_;
    int iter_ = 0;
    std::mt19937 gen_;
    uint64_t draw_ctr_ = 0;
    std::vector<Splittable> clusters_;
    std::vector<double> weights_;

    // ----------------------------------------------------------------- learned screen
    enum ScreenUse { USE_FULL, USE_SCREEN, USE_SWEEP };
    bool dev_ = false;            // parameters drawn on the device (see the constructor)
    ScreenRecord scr_;
    bool scr_disabled_ = false;
    bool scr_swept_ = false;     // a full sweep ran in this iteration
    // min_cand: fewer candidates than this are all evaluated exactly (the screen would cost more)
    ScreenUse screen_use(int64_t ncand, int64_t min_cand = 0) const
    {
        if (cfg_.screen_mode != DPMM_SCREEN_ON || scr_disabled_) return USE_FULL;
        if (cfg_.screen_sweep > 0 && iter_ % cfg_.screen_sweep == 0) return USE_SWEEP;
        return ncand > cfg_.screen_top && ncand >= min_cand ? USE_SCREEN : USE_FULL;
    }
    dpmm_status screen_log(int K, int kind, const std::vector<uint8_t>& row_ok, const double* hr_of_row);
    void screen_assess();

};

}  // namespace host
}  // namespace dpmm

struct dpmm_model_info {
    int64_t n = 0;
    std::vector<int32_t> labels;
    std::vector<double> weights, iter_count, likelihood_history, nmi_history;
    std::vector<int32_t> cluster_count_history;
    dpmm::host::ScreenRecord screen;
};

namespace dpmm {
namespace host {

// thin_cluster_params broadcast + per-cluster parameter copies (local_clusters_actions.cpp:373-382)
dpmm_status Sampler::upload_params(const std::vector<double>& weights)
{
    const int K = (int)clusters_.size();
    const int D = D_;
    std::vector<double> w(K, 1.0), lrw(2 * (size_t)K);
    for (int k = 0; k < K; ++k) {
        w[k] = k < (int)weights.size() ? weights[k] : 0.0;
        lrw[2 * k] = clusters_[k].lrw[0];
        lrw[2 * k + 1] = clusters_[k].lrw[1];
    }
    if (cfg_.prior == DPMM_PRIOR_MULTINOMIAL) {
        std::vector<double> lt((size_t)K * D), lt_lr((size_t)2 * K * D);
        for (int k = 0; k < K; ++k) {
            std::memcpy(&lt[(size_t)k * D], clusters_[k].c.dist.log_theta.data(), sizeof(double) * D);
            std::memcpy(&lt_lr[(size_t)(2 * k) * D], clusters_[k].l.dist.log_theta.data(), sizeof(double) * D);
            std::memcpy(&lt_lr[(size_t)(2 * k + 1) * D], clusters_[k].r.dist.log_theta.data(), sizeof(double) * D);
        }
        return dpmm_set_multinomial_params(ctx_, K, lt.data(), w.data(), lt_lr.data(), lrw.data());
    }
    std::vector<double> mu((size_t)K * D), W((size_t)K * D * D), ld(K), mu_lr((size_t)2 * K * D),
        W_lr((size_t)2 * K * D * D), ld_lr(2 * (size_t)K);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < K; ++k) {
        const Dist* ds[3] = {&clusters_[k].c.dist, &clusters_[k].l.dist, &clusters_[k].r.dist};
        std::memcpy(&mu[(size_t)k * D], ds[0]->mu.data(), sizeof(double) * D);
        std::memcpy(&W[(size_t)k * D * D], ds[0]->W.data(), sizeof(double) * D * D);
        ld[k] = ds[0]->logdet_sigma;
        for (int s = 0; s < 2; ++s) {
            std::memcpy(&mu_lr[(size_t)(2 * k + s) * D], ds[1 + s]->mu.data(), sizeof(double) * D);
            std::memcpy(&W_lr[(size_t)(2 * k + s) * D * D], ds[1 + s]->W.data(), sizeof(double) * D * D);
            ld_lr[2 * k + s] = ds[1 + s]->logdet_sigma;
        }
    }
    return dpmm_set_gaussian_factors(ctx_, K, mu.data(), W.data(), ld.data(), w.data(), mu_lr.data(), W_lr.data(),
                                     ld_lr.data(), lrw.data());
}

// runs with an outlier cluster: which clusters carry the outlier prior (the outlier cluster and the
// clusters split from it, as their host bookkeeping does), before every device launch that reads the
// priors (draws, marginal likelihoods, split and merge ratios: each cluster's own prior, as
// should_split_local and should_merge use, local_clusters_actions.cpp:215-239, shared_actions.cpp:88-95)
dpmm_status Sampler::sync_prior_select()
{
    if (!(cfg_.outlier_mod > 0) || clusters_.empty()) return DPMM_OK;
    std::vector<uint8_t> sel(clusters_.size());
    for (size_t k = 0; k < clusters_.size(); ++k) sel[k] = clusters_[k].c.prior.outlier ? 1 : 0;
    return dpmm_set_cluster_priors(ctx_, (int)sel.size(), sel.data());
}

// local_clusters_actions::update_suff_stats_posterior (local_clusters_actions.cpp:103-168)
dpmm_status Sampler::update_suff_stats_posterior(const std::vector<int32_t>& indices)
{
    const int n = (int)indices.size();
    if (n == 0) return DPMM_OK;
    if (dev_) {   // the statistics stay on the device; the host bookkeeping needs the counts
        std::vector<int64_t> cnt(3 * (size_t)n);
        DPMM_TRY(dpmm_statistics_counts(ctx_, n, indices.data(), cnt.data()));
        bool outlier_listed = false;
        for (int q = 0; q < n; ++q) {
            Splittable& sc = clusters_[indices[q]];
            sc.c.stats.N = cnt[3 * (size_t)q];
            sc.l.stats.N = cnt[3 * (size_t)q + 1];
            sc.r.stats.N = cnt[3 * (size_t)q + 2];
            sc.points_count = sc.c.stats.N;
            outlier_listed |= cfg_.outlier_mod > 0 && indices[q] == 0;
        }
        // the outlier cluster's split ratio is evaluated on the host (its own prior): its full
        // statistics and posteriors
        if (outlier_listed) return host_stats_posterior({0});
        return DPMM_OK;
    }
    return host_stats_posterior(indices);
}

// the statistics of the listed clusters downloaded, and their posteriors
dpmm_status Sampler::host_stats_posterior(const std::vector<int32_t>& indices)
{
    const int n = (int)indices.size();
    const int D = D_;
    const bool gauss = cfg_.prior == DPMM_PRIOR_GAUSSIAN;
    std::vector<int64_t> cnt(3 * (size_t)n);
    std::vector<double> sum(3 * (size_t)n * D), S(gauss ? 3 * (size_t)n * D * D : 0);
    DPMM_TRY(dpmm_create_sufficient_statistics(ctx_, n, indices.data(), cnt.data(), sum.data(),
                                               gauss ? S.data() : nullptr));
#pragma omp parallel for schedule(dynamic)
    for (int q = 0; q < n; ++q) {
        Splittable& sc = clusters_[indices[q]];
        ClusterParams* cp[3] = {&sc.c, &sc.l, &sc.r};
        for (int s = 0; s < 3; ++s) {
            Stats st;
            st.N = cnt[3 * (size_t)q + s];
            st.sum.assign(&sum[(3 * (size_t)q + s) * D], &sum[(3 * (size_t)q + s) * D] + D);
            if (gauss) st.S.assign(&S[(3 * (size_t)q + s) * D * D], &S[(3 * (size_t)q + s) * D * D] + (size_t)D * D);
            cp[s]->stats = std::move(st);
            cp[s]->post = posterior(cp[s]->prior, cp[s]->stats);
        }
        sc.points_count = sc.c.stats.N;
    }
    return DPMM_OK;
}

// shared_actions::sample_cluster_params (shared_actions.cpp:9-55) for every cluster, with the
// three distribution draws of all clusters done in parallel
void Sampler::sample_cluster_params_all()
{
    const int K = (int)clusters_.size();
    std::vector<int> todo;
    for (int i = 0; i < K; ++i)
        if (!(cfg_.outlier_mod > 0 && i == 1)) todo.push_back(i);   // local_clusters_actions.cpp:348-351
    const uint64_t base = draw_ctr_;
    draw_ctr_ += 3 * (uint64_t)K;
    std::vector<double> lml_lr(K, 0.0);
    // one task per draw (3 per cluster) and per sub-cluster marginal likelihood: the tasks of a
    // cluster are independent, so they balance over the threads better than whole clusters
    const int nt = (int)todo.size();
    std::vector<double> lml_s(2 * (size_t)nt, 0.0);
#pragma omp parallel for schedule(dynamic)
    for (int q = 0; q < 5 * nt; ++q) {
        const int t = q / 5, s = q % 5;
        const int i = todo[t];
        Splittable& sc = clusters_[i];
        if (s < 3) {
            ClusterParams* cp = s == 0 ? &sc.c : (s == 1 ? &sc.l : &sc.r);
            std::mt19937_64 g = draw_gen(base + 3 * (uint64_t)i + s);
            cp->dist = sample(cp->post, g);
        } else {
            const ClusterParams& cp = s == 3 ? sc.l : sc.r;
            lml_s[2 * (size_t)t + (s - 3)] = lml(cp.prior, cp.post, cp.stats);
        }
    }
    for (int t = 0; t < nt; ++t) lml_lr[todo[t]] = lml_s[2 * (size_t)t] + lml_s[2 * (size_t)t + 1];
    const int B = cfg_.burnout;
    for (int i : todo) {
        Splittable& sc = clusters_[i];
        std::vector<double> pc = {(double)sc.l.stats.N + cfg_.alpha / 2, (double)sc.r.stats.N + cfg_.alpha / 2};
        std::vector<double> w = dirichlet(pc);
        sc.lrw[0] = w[0];
        sc.lrw[1] = w[1];
        for (int q = 0; q < B - 1; ++q) sc.hist[q] = sc.hist[q + 1];
        sc.hist[B - 1] = std::make_pair(true, lml_lr[i]);
        double now = 0.0;
        bool ready = true;
        for (int q = 0; q < B; ++q) {
            if (sc.hist[q].first) now += sc.hist[q].second * (1 / (B - 0.1));
            else ready = false;
        }
        if (ready && now - sc.hist[B - 1].second < 1e-2) sc.splittable = true;
        sc.points_count = sc.c.stats.N;
    }
}

// local_clusters_actions::sample_clusters (local_clusters_actions.cpp:341-371)
dpmm_status Sampler::sample_clusters()
{
    if (dev_) return sample_clusters_device();
    sample_cluster_params_all();
    mixture_weights();
    return DPMM_OK;
}

// the cluster weights: Dir(N_1 .. N_K, alpha) without its last entry (local_clusters_actions.cpp:341-371)
void Sampler::mixture_weights()
{
    std::vector<double> pc;
    for (size_t i = 0; i < clusters_.size(); ++i) {
        if (cfg_.outlier_mod > 0 && i == 1) continue;
        pc.push_back((double)clusters_[i].points_count);
    }
    pc.push_back(cfg_.alpha);
    std::vector<double> d;
    if (pc.size() == 2 && pc[0] == 0.0) d = {0.0, 1.0};   // local_clusters_actions.cpp:323-339
    else d = dirichlet(pc);
    weights_.clear();
    for (size_t i = 0; i + 1 < d.size(); ++i) weights_.push_back(d[i] * (1 - cfg_.outlier_mod));
    if (cfg_.outlier_mod > 0) weights_.insert(weights_.begin(), cfg_.outlier_mod);
}

// sample_clusters with the NIW draws on the device: the host draws the Dirichlet weights (same
// generator order as the host path: sub-cluster weights cluster by cluster, then the mixture
// weights), the device draws every slot's parameters into the label-phase buffers and returns each
// slot's log marginal likelihood for the splittable history (shared_actions.cpp:30-54)
dpmm_status Sampler::sample_clusters_device()
{
    const int K = (int)clusters_.size();
    const bool outlier = cfg_.outlier_mod > 0;
    DPMM_TRY(sync_prior_select());
    std::vector<double> lrw(2 * (size_t)K);
    for (int i = 0; i < K; ++i) {
        Splittable& sc = clusters_[i];
        if (!(outlier && i == 1)) {   // cluster 1 is not redrawn with an outlier cluster (:348-351)
            std::vector<double> w =
                dirichlet({(double)sc.l.stats.N + cfg_.alpha / 2, (double)sc.r.stats.N + cfg_.alpha / 2});
            sc.lrw[0] = w[0];
            sc.lrw[1] = w[1];
        }
        lrw[2 * i] = sc.lrw[0];
        lrw[2 * i + 1] = sc.lrw[1];
    }
    mixture_weights();
    std::vector<double> w(K, 0.0), lml(3 * (size_t)K);
    for (int k = 0; k < K && k < (int)weights_.size(); ++k) w[k] = weights_[k];
    if (cfg_.prior == DPMM_PRIOR_MULTINOMIAL)
        DPMM_TRY(dpmm_sample_multinomial_params(ctx_, K, cfg_.seed, draw_ctr_, lrw.data(), lml.data()));
    else
        DPMM_TRY(dpmm_sample_gaussian_params(ctx_, K, cfg_.seed, draw_ctr_, w.data(), lrw.data(), lml.data()));
    draw_ctr_ += 3 * (uint64_t)K;
    const int B = cfg_.burnout;
    for (int i = 0; i < K; ++i) {
        if (outlier && i == 1) continue;
        Splittable& sc = clusters_[i];
        for (int q = 0; q < B - 1; ++q) sc.hist[q] = sc.hist[q + 1];
        sc.hist[B - 1] = std::make_pair(true, lml[3 * (size_t)i + 1] + lml[3 * (size_t)i + 2]);
        double now = 0.0;
        bool ready = true;
        for (int q = 0; q < B; ++q) {
            if (sc.hist[q].first) now += sc.hist[q].second * (1 / (B - 0.1));
            else ready = false;
        }
        if (ready && now - sc.hist[B - 1].second < 1e-2) sc.splittable = true;
        sc.points_count = sc.c.stats.N;
    }
    return DPMM_OK;
}

// local_clusters_actions::reset_bad_clusters (local_clusters_actions.cpp:429-447)
dpmm_status Sampler::reset_bad_clusters()
{
    std::vector<int32_t> bad;
    for (size_t i = 0; i < clusters_.size(); ++i) {
        Splittable& sc = clusters_[i];
        if (sc.l.stats.N == 0 || sc.r.stats.N == 0) {
            bad.push_back((int32_t)i);
            sc.hist = fresh_hist();
            sc.splittable = false;
        }
    }
    if (bad.empty()) return DPMM_OK;
    DPMM_TRY(dpmm_reset_bad_clusters(ctx_, (int)bad.size(), bad.data(), nullptr));
    return update_suff_stats_posterior(bad);
}

// local_clusters_actions::check_and_split + should_split_local + split_cluster_local
// (local_clusters_actions.cpp:183-194, 215-285), split ratios from one device launch.  With the
// learned screen on, only the screen's top candidates are proposed (and evaluated exactly).
dpmm_status Sampler::check_and_split(bool final_, std::vector<int32_t>& all_indices)
{
    const int K = (int)clusters_.size();
    all_indices.clear();
    std::vector<int> split(K, 0);
    bool any_candidate = false;
    for (int i = 0; i < K; ++i)
        if (clusters_[i].splittable && clusters_[i].c.stats.N > 1 && !(cfg_.outlier_mod > 0 && i == 1))
            any_candidate = true;
    if (!any_candidate || final_) return DPMM_OK;
    // candidates whose ratio the device computes (the outlier cluster's is computed on the host)
    std::vector<uint8_t> elig(K, 0);
    int64_t ncand = 0;
    for (int i = 0; i < K; ++i) {
        const Splittable& sc = clusters_[i];
        if (sc.splittable && sc.c.stats.N > 1 && sc.l.stats.N > 0 && sc.r.stats.N > 0 && !(cfg_.outlier_mod > 0 && i <= 1)) {
            elig[i] = 1;
            ++ncand;
        }
    }
    std::vector<double> hr(K, NAN);
    std::vector<uint8_t> in_sel(K, 0);
    const ScreenUse use = screen_use(ncand, cfg_.screen_split_min);
    DPMM_TRY(sync_prior_select());
    if (use != USE_FULL && ncand > 0) {
        std::vector<int32_t> sel(kScrMaxTop);
        int32_t nsel = 0;
        DPMM_TRY(dpmm_screen_select(ctx_, K, DPMM_SCREEN_SPLIT, cfg_.alpha, elig.data(), cfg_.screen_top, sel.data(),
                                    &nsel, nullptr));
        for (int t = 0; t < nsel; ++t) in_sel[sel[t]] = 1;
        if (use == USE_SCREEN) {
            std::vector<double> out(nsel);
            DPMM_TRY(dpmm_split_hastings_list(ctx_, K, cfg_.alpha, nsel, sel.data(), out.data()));
            for (int t = 0; t < nsel; ++t) hr[sel[t]] = out[t];
            scr_.split_exact += nsel;
        }
    }
    if (use != USE_SCREEN) {
        DPMM_TRY(dpmm_split_hastings(ctx_, K, cfg_.alpha, nullptr, hr.data()));
        scr_.split_exact += ncand;
        if (cfg_.screen_mode == DPMM_SCREEN_LOG) DPMM_TRY(screen_log(K, DPMM_SCREEN_SPLIT, elig, hr.data()));
    }
    scr_.split_cand += ncand;
    for (int i = 0; i < K; ++i) {
        if (cfg_.outlier_mod > 0 && i == 1) continue;
        Splittable& sc = clusters_[i];
        if (!(sc.splittable && sc.c.stats.N > 1)) continue;
        if (sc.l.stats.N == 0 || sc.r.stats.N == 0) continue;
        const bool outlier0 = cfg_.outlier_mod > 0 && i == 0;
        if (use == USE_SCREEN && !outlier0 && !in_sel[i]) continue;   // not proposed this iteration
        double log_hr = hr[i];
        if (outlier0) {
            // the outlier cluster has its own prior: evaluate its ratio on the host
            Hyper p = posterior(sc.c.prior, sc.c.stats), pl = posterior(sc.c.prior, sc.l.stats),
                  pr = posterior(sc.c.prior, sc.r.stats);
            log_hr = std::log(cfg_.alpha) + std::lgamma((double)sc.l.stats.N) + lml(sc.l.prior, pl, sc.l.stats) +
                     std::lgamma((double)sc.r.stats.N) + lml(sc.r.prior, pr, sc.r.stats) -
                     (std::lgamma((double)sc.c.stats.N) + lml(sc.c.prior, p, sc.c.stats));
        }
        const double u = uniform();
        if (log_hr > std::log(u)) {
            split[i] = 1;
            if (use == USE_SWEEP && elig[i]) {
                ++scr_.sweep_accepts;
                scr_.sweep_hits += in_sel[i];
            }
        }
    }
    int n_split = std::accumulate(split.begin(), split.end(), 0);
    // capacity guard: the device tables hold k_max clusters
    while (n_split > 0 && K + n_split > ctx_->k_max) {
        for (int i = K - 1; i >= 0; --i)
            if (split[i]) { split[i] = 0; --n_split; break; }
    }
    if (n_split == 0) return DPMM_OK;
    std::vector<int32_t> idx, nidx;
    int new_index = K;
    clusters_.resize(K + n_split);
    for (int i = 0; i < K; ++i) {
        if (!split[i]) continue;
        idx.push_back(i);
        nidx.push_back(new_index);
        // split_cluster_local: the new cluster takes r, cluster i keeps l.  Every field of both is
        // rewritten here, so the parameters move rather than copy (a D x D NIW cluster holds several
        // D x D matrices per sub-cluster)
        Splittable& sc = clusters_[i];
        Splittable ns;
        auto make = [&](ClusterParams&& p, Splittable& out) {   // create_splittable_from_params
            out.l = p;
            out.r = p;
            if (!dev_) {   // (device mode: every slot is drawn on the device before the next label phase)
                std::mt19937_64 g1 = draw_gen(draw_ctr_++), g2 = draw_gen(draw_ctr_++);
                out.l.dist = sample(p.post, g1);
                out.r.dist = sample(p.post, g2);
            }
            std::vector<double> w = dirichlet({cfg_.alpha / 2, cfg_.alpha / 2});
            out.lrw[0] = w[0];
            out.lrw[1] = w[1];
            out.c = std::move(p);
            out.hist = fresh_hist();
            out.splittable = false;
        };
        ClusterParams r = std::move(sc.r), l = std::move(sc.l);
        make(std::move(r), ns);
        make(std::move(l), sc);
        ns.points_count = ns.c.stats.N;
        sc.points_count = sc.c.stats.N;
        clusters_[new_index] = std::move(ns);
        ++new_index;
    }
    all_indices = idx;
    all_indices.insert(all_indices.end(), nidx.begin(), nidx.end());
    return dpmm_split_clusters(ctx_, (int)idx.size(), idx.data(), nidx.data(), nullptr);
}

// local_clusters_actions::check_and_merge + shared_actions::should_merge + merge_clusters
// (local_clusters_actions.cpp:204-213, 287-321; shared_actions.cpp:72-111); all pair ratios
// from one device launch, accepted greedily in (i, j) order.  With the learned screen on, only the
// screen's top pairs are proposed (and evaluated exactly), still greedily in (i, j) order.
dpmm_status Sampler::check_and_merge(bool final_)
{
    const int K = (int)clusters_.size();
    int n_split = 0;
    for (auto& c : clusters_) n_split += c.splittable && c.c.stats.N > 0;
    if (n_split < 2) return DPMM_OK;
    std::vector<uint8_t> elig(K, 0);
    int64_t m = 0;
    for (int i = 0; i < K; ++i) {
        const Splittable& a = clusters_[i];
        elig[i] = !(cfg_.outlier_mod > 0 && i == 0) && a.splittable && a.c.stats.N > 0;
        m += elig[i];
    }
    const int64_t ncand = m * (m - 1) / 2;
    DPMM_TRY(sync_prior_select());
    const ScreenUse use = screen_use(ncand);
    // proposals in (i, j) order with their ratios
    struct Prop {
        int i, j;
        double hr;
        bool sel;
    };
    std::vector<Prop> props;
    std::vector<uint8_t> in_sel;
    std::vector<int32_t> sel_pairs;
    if (use != USE_FULL && ncand > 0) {
        std::vector<int32_t> sel(kScrMaxTop);
        int32_t nsel = 0;
        DPMM_TRY(dpmm_screen_select(ctx_, K, DPMM_SCREEN_MERGE, cfg_.alpha, elig.data(), cfg_.screen_top, sel.data(),
                                    &nsel, nullptr));
        in_sel.assign((size_t)K * K, 0);
        for (int t = 0; t < nsel; ++t) {
            int64_t b = sel[t];
            int i = 0, rowlen = K - 1;
            while (b >= rowlen) {
                b -= rowlen;
                ++i;
                --rowlen;
            }
            const int j = i + 1 + (int)b;
            in_sel[(size_t)i * K + j] = 1;
            sel_pairs.push_back(i);
            sel_pairs.push_back(j);
        }
        if (use == USE_SCREEN) {
            std::vector<double> out(nsel);
            DPMM_TRY(dpmm_merge_hastings_list(ctx_, K, cfg_.alpha, nsel, sel_pairs.data(), out.data()));
            for (int t = 0; t < nsel; ++t) props.push_back({sel_pairs[2 * t], sel_pairs[2 * t + 1], out[t], true});
            scr_.merge_exact += nsel;
        }
    }
    if (use != USE_SCREEN) {
        std::vector<double> hr((size_t)K * K);
        DPMM_TRY(dpmm_merge_hastings(ctx_, K, cfg_.alpha, hr.data()));
        scr_.merge_exact += ncand;
        if (cfg_.screen_mode == DPMM_SCREEN_LOG) {
            std::vector<uint8_t> row_ok;
            std::vector<double> hr_rows;
            for (int i = 0; i < K; ++i)
                for (int j = i + 1; j < K; ++j) {
                    row_ok.push_back(elig[i] && elig[j]);
                    hr_rows.push_back(hr[(size_t)i * K + j]);
                }
            DPMM_TRY(screen_log(K, DPMM_SCREEN_MERGE, row_ok, hr_rows.data()));
        }
        for (int i = 0; i < K; ++i)
            for (int j = i + 1; j < K; ++j)
                props.push_back({i, j, hr[(size_t)i * K + j], !in_sel.empty() && in_sel[(size_t)i * K + j]});
    }
    scr_.merge_cand += ncand;
    std::vector<int32_t> idx, nidx;
    for (const Prop& pr : props) {
        const int i = pr.i, j = pr.j;
        if (cfg_.outlier_mod > 0 && i == 0) continue;
        Splittable& a = clusters_[i];
        Splittable& b = clusters_[j];
        if (!(a.splittable && b.splittable && a.c.stats.N > 0 && b.c.stats.N > 0)) continue;
        const double log_hr = pr.hr;
        const double u = uniform();
        if (!((log_hr > std::log(u)) || (final_ && log_hr > std::log(0.1)))) continue;
        if (use == USE_SWEEP) {
            ++scr_.sweep_accepts;
            scr_.sweep_hits += pr.sel;
        }
        // merge_clusters_to_splittable(a, b.c) then local bookkeeping
        a.c.stats = aggregate(a.c.stats, b.c.stats);
        if (!dev_) a.c.post = posterior(a.c.prior, a.c.stats);
        std::vector<double> w = dirichlet({(double)a.c.stats.N + cfg_.alpha / 2, (double)b.c.stats.N + cfg_.alpha / 2});
        a.lrw[0] = w[0];
        a.lrw[1] = w[1];
        a.l = a.c;
        a.r = std::move(b.c);   // b is emptied below and skipped by every later candidate
        a.splittable = false;
        a.hist = fresh_hist();
        a.points_count += b.points_count;
        b.points_count = 0;
        b.c.stats.N = 0;
        b.splittable = false;
        idx.push_back(i);
        nidx.push_back(j);
    }
    if (idx.empty()) return DPMM_OK;
    DPMM_TRY(dpmm_merge_clusters(ctx_, (int)idx.size(), idx.data(), nidx.data()));
    if (dev_) DPMM_TRY(dpmm_merge_statistics(ctx_, (int)idx.size(), idx.data(), nidx.data()));
    return DPMM_OK;
}

// features + exact ratio of every loggable candidate row (DPMM_SCREEN_LOG)
dpmm_status Sampler::screen_log(int K, int kind, const std::vector<uint8_t>& row_ok, const double* hr_of_row)
{
    const size_t rows = row_ok.size();
    if (rows == 0) return DPMM_OK;
    std::vector<float> f(rows * kScrF);
    DPMM_TRY(dpmm_screen_features(ctx_, K, kind, cfg_.alpha, f.data(), nullptr));
    for (size_t r = 0; r < rows; ++r) {
        if (!row_ok[r] || !std::isfinite(hr_of_row[r])) continue;
        scr_.log_features.insert(scr_.log_features.end(), &f[r * kScrF], &f[r * kScrF] + kScrF);
        scr_.log_hr.push_back(hr_of_row[r]);
        scr_.log_kind.push_back((int8_t)kind);
        scr_.log_iter.push_back(iter_);
    }
    return DPMM_OK;
}

// after an iteration with a full sweep: switch the screen off when its recall is too low
void Sampler::screen_assess()
{
    if (!scr_swept_) return;
    scr_swept_ = false;
    ++scr_.sweeps;
    if (scr_.sweep_accepts >= 8 && (double)scr_.sweep_hits < cfg_.screen_min_recall * (double)scr_.sweep_accepts) {
        scr_disabled_ = true;
        scr_.disabled_at = iter_;
    }
}

// local_clusters_actions::remove_empty_clusters (local_clusters_actions.cpp:384-419)
dpmm_status Sampler::remove_empty_clusters()
{
    std::vector<Splittable> keep;
    std::vector<int32_t> limits, kept;
    int removed = 0;
    const size_t K = clusters_.size();
    for (size_t i = 0; i < K; ++i) {
        const int64_t pc = clusters_[i].points_count;
        if (pc == 0) {
            limits.push_back((int32_t)(i - removed + 1));
            ++removed;
        }
        if (pc > 0 || (cfg_.outlier_mod > 0 && i == 0) || (cfg_.outlier_mod > 0 && i == 1 && K == 2)) {
            keep.push_back(std::move(clusters_[i]));
            kept.push_back((int32_t)i);
        }
    }
    clusters_ = std::move(keep);
    if (limits.empty()) return DPMM_OK;
    DPMM_TRY(dpmm_remove_empty_clusters(ctx_, (int)limits.size(), limits.data()));
    if (dev_) DPMM_TRY(dpmm_compact_statistics(ctx_, (int)kept.size(), kept.data()));
    return DPMM_OK;
}

// local_clusters_actions::group_step (local_clusters_actions.cpp:460-490)
dpmm_status Sampler::group_step(bool no_more_splits, bool final_)
{
    DPMM_TRY(stage_params());
    DPMM_TRY(dpmm_create_clusters_labels(ctx_, (int)clusters_.size(), final_ ? 1 : 0, nullptr, nullptr));
    return stage_rest(no_more_splits, final_);
}

// the stages of group_step: parameters for the label phase ...
dpmm_status Sampler::stage_params()
{
    DPMM_TRY(sample_clusters());
    if (!dev_) DPMM_TRY(upload_params(weights_));
    return DPMM_OK;
}

// ... and everything after it (sub-labels, statistics, reset, split, merge, compaction)
dpmm_status Sampler::stage_rest(bool no_more_splits, bool final_)
{
    const int K = (int)clusters_.size();
    DPMM_TRY(dpmm_create_subclusters_labels(ctx_, K, nullptr, nullptr));
    std::vector<int32_t> all(K);
    std::iota(all.begin(), all.end(), 0);
    DPMM_TRY(update_suff_stats_posterior(all));
    DPMM_TRY(reset_bad_clusters());
    if (!no_more_splits) {
        std::vector<int32_t> idx;
        scr_swept_ = screen_use(0) == USE_SWEEP;
        DPMM_TRY(check_and_split(final_, idx));
        DPMM_TRY(update_suff_stats_posterior(idx));
        DPMM_TRY(check_and_merge(final_));
        screen_assess();
    }
    return remove_empty_clusters();
}

// dp_parallel_sampling_class::init_model + init_first_clusters (dp_parallel_sampling.cpp:48-87)
dpmm_status Sampler::init_first_clusters()
{
    DPMM_TRY(dpmm_sample_labels(ctx_, cfg_.initial_clusters, cfg_.outlier_mod, nullptr));
    DPMM_TRY(dpmm_sample_sub_labels(ctx_, nullptr));
    clusters_.clear();
    if (cfg_.outlier_mod > 0) {   // create_outlier_local_cluster (local_clusters_actions.cpp:48-79)
        Splittable sc;
        sc.c.prior = cfg_.outlier_hyper;
        sc.c.stats = empty_stats();
        DPMM_TRY(all_points_stats(ctx_, &sc.c.stats.N, sc.c.stats.sum.data(),
                                  cfg_.prior == DPMM_PRIOR_GAUSSIAN ? sc.c.stats.S.data() : nullptr));
        sc.c.post = posterior(cfg_.outlier_hyper, sc.c.stats);
        std::mt19937_64 g = draw_gen(draw_ctr_++);
        sc.c.dist = sample(sc.c.post, g);
        sc.l = sc.c;
        sc.r = sc.c;
        sc.hist = fresh_hist();
        int32_t l = 0, r = 0;
        DPMM_TRY(dpmm_get_sub_labels_count(ctx_, &l, &r));
        sc.l.stats.N = l;
        sc.r.stats.N = r;
        sc.points_count = sc.c.stats.N;
        clusters_.push_back(std::move(sc));
    }
    for (int i = 0; i < cfg_.initial_clusters; ++i) {   // create_first_local_cluster (:14-46)
        Splittable sc;
        sc.c.prior = cfg_.hyper;
        sc.c.stats = empty_stats();
        std::mt19937_64 g = draw_gen(draw_ctr_++);
        sc.c.dist = sample(cfg_.hyper, g);
        sc.c.post = cfg_.hyper;
        sc.c.stats.N = Ntot_;
        sc.l = sc.c;
        sc.r = sc.c;
        sc.hist = fresh_hist();
        sc.l.stats.N = 0;
        sc.r.stats.N = 0;
        int32_t l = 0, r = 0;
        DPMM_TRY(dpmm_get_sub_labels_count(ctx_, &l, &r));
        sc.l.stats.N = l;
        sc.r.stats.N = r;
        sc.points_count = sc.c.stats.N;
        clusters_.push_back(std::move(sc));
        DPMM_TRY(dpmm_sample_sub_labels(ctx_, nullptr));   // split_first_cluster_worker
    }
    std::vector<int32_t> all(clusters_.size());
    std::iota(all.begin(), all.end(), 0);
    DPMM_TRY(update_suff_stats_posterior(all));
    if (dev_ && cfg_.outlier_mod > 0) {
        // cluster 1 keeps its initial draw (it is not redrawn with an outlier cluster): the host's
        // initial parameters go to the device once, the device draws then replace the others
        std::vector<double> w(clusters_.size(), 1.0 / (double)clusters_.size());
        DPMM_TRY(upload_params(w));
    }
    return sample_clusters();
}

// dp_parallel_sampling_class::calculate_posterior (dp_parallel_sampling.cpp:218-236); with device
// draws the clusters' marginal likelihoods come from the device statistics
dpmm_status Sampler::calculate_posterior(double* out)
{
    double lp = std::lgamma(cfg_.alpha) - std::lgamma((double)Ntot_ + cfg_.alpha);
    std::vector<double> dl;
    if (dev_ && !clusters_.empty()) {
        dl.resize(3 * clusters_.size());
        DPMM_TRY(sync_prior_select());
        DPMM_TRY(slot_lml_as_is(ctx_, (int)clusters_.size(), dl.data()));
    }
    for (size_t k = 0; k < clusters_.size(); ++k) {
        const Splittable& sc = clusters_[k];
        if (sc.c.stats.N == 0) continue;
        lp += dev_ ? dl[3 * k] : lml(sc.c.prior, sc.c.post, sc.c.stats);
        lp += std::log(cfg_.alpha) + std::lgamma((double)sc.c.stats.N);
    }
    *out = lp;
    return DPMM_OK;
}

// dp_parallel_sampling_class::run_model (dp_parallel_sampling.cpp:132-206), n iterations at a time
dpmm_status Sampler::step(int n, dpmm_model_info* mi)
{
    mi->n = N_;
    for (int q = 0; q < n && iter_ < cfg_.iterations; ++q) {
        IterState st = begin_iteration();
        DPMM_TRY(group_step(st.no_more_splits, st.final_));
        DPMM_TRY(end_iteration(st, mi));
    }
    return DPMM_OK;
}

// the loop head of run_model (dp_parallel_sampling.cpp:139-150)
Sampler::IterState Sampler::begin_iteration()
{
    IterState st;
    st.i = ++iter_;
    st.final_ = st.i >= cfg_.iterations - cfg_.argmax_sample_stop;
    st.no_more_splits = st.i >= cfg_.iterations - cfg_.split_stop || (double)clusters_.size() >= cfg_.max_clusters;
    st.t0 = std::chrono::steady_clock::now();
    return st;
}

// the loop tail: iteration time, histories, verbose line (dp_parallel_sampling.cpp:151-200)
dpmm_status Sampler::end_iteration(const IterState& st, dpmm_model_info* mi)
{
    mi->n = N_;
    const int i = st.i;
    {
        auto t1 = std::chrono::steady_clock::now();
        mi->iter_count.push_back(std::chrono::duration<double>(t1 - st.t0).count());
        mi->cluster_count_history.push_back((int32_t)clusters_.size());
        if (cfg_.verbose) {
            double lp = 0;
            DPMM_TRY(calculate_posterior(&lp));
            mi->likelihood_history.push_back(lp);
            if (!cfg_.gt.empty()) {   // scored on the device: only the contingency table comes back
                double v = 0;
                DPMM_TRY(dpmm_label_agreement(ctx_, (int)clusters_.size(), &v, nullptr));
                mi->nmi_history.push_back(v);
            }
            std::printf("Iteration: %d || Clusters count: %d || Log posterior: %f || NMI score: %f || Iter Time: %f\n", i,
                        (int)clusters_.size(), mi->likelihood_history.back(),
                        mi->nmi_history.empty() ? -1.0 : mi->nmi_history.back(), mi->iter_count.back());
        } else {
            mi->likelihood_history.push_back(1);
        }
    }
    return DPMM_OK;
}

dpmm_status Sampler::finish(dpmm_model_info* mi)
{
    mi->n = N_;
    mi->labels.resize(N_);
    DPMM_TRY(dpmm_get_labels(ctx_, mi->labels.data()));
    mi->weights = weights_;
    mi->screen = scr_;
    return DPMM_OK;
}

// ----------------------------------------------------------------- config helpers
static Hyper default_hyper(int prior, int D)   // niw.cpp:195-198 / multinomial_prior.cpp:98-101
{
    Hyper h;
    if (prior == DPMM_PRIOR_GAUSSIAN) {
        h.k = 1.0;
        h.v = 5;
        h.m.assign(D, 0.0);
        h.psi.assign((size_t)D * D, 0.0);
        for (int i = 0; i < D; ++i) h.psi[(size_t)i * D + i] = 1.0;
    } else {
        h.alpha.assign(D, 0.0);
    }
    return h;
}

static uint64_t resolve_seed(uint64_t s)   // global_params::init_random (global_params.cpp:97-106)
{
    if (s != 0) return s;
    std::srand((unsigned)std::time(nullptr));
    return (uint64_t)std::rand();
}

struct SamplerHandle {
    Config cfg;
    dpmm_ctx* ctx = nullptr;
    std::unique_ptr<Sampler> sampler;
    dpmm_model_info mi;
    ~SamplerHandle()
    {
        sampler.reset();
        if (ctx) dpmm_destroy(ctx);
    }
};

// dp_parallel_sampling_class(N, x, seed, prior) + global_params::init + init_model + init_first_clusters
dpmm_status make_sampler(const Config& cfg_in, int64_t N, int D, const void* points, bool f32,
                         std::unique_ptr<SamplerHandle>& out, const dpmm_shard* shard = nullptr)
{
    auto h = std::make_unique<SamplerHandle>();
    Config& cfg = h->cfg;
    cfg = cfg_in;
    cfg.seed = resolve_seed(cfg.seed);
    auto finish = [&](Hyper& hp) -> dpmm_status {
        if (cfg.prior == DPMM_PRIOR_GAUSSIAN) {
            if ((int)hp.m.size() != D || (int)hp.psi.size() != D * D)
                return fail(DPMM_ERR_INVALID_ARG, "NIW hyper-parameters do not match the data dimension");
            if (!la::cholesky(hp.psi.data(), D, hp.chol)) return fail(DPMM_ERR_NOT_PD, "prior psi is not positive definite");
            hp.logdet = la::logdet_from_chol(hp.chol, D);
        } else if ((int)hp.alpha.size() != D) {
            return fail(DPMM_ERR_INVALID_ARG, "multinomial alpha does not match the data dimension");
        }
        return DPMM_OK;
    };
    DPMM_TRY(finish(cfg.hyper));
    DPMM_TRY(finish(cfg.outlier_hyper));
    if (cfg.burnout < 1) return fail(DPMM_ERR_INVALID_ARG, "burnout must be >= 1");
    if (cfg.initial_clusters < 1) return fail(DPMM_ERR_INVALID_ARG, "initial_clusters must be >= 1");
    if (cfg.screen_mode < DPMM_SCREEN_OFF || cfg.screen_mode > DPMM_SCREEN_LOG)
        return fail(DPMM_ERR_INVALID_ARG, "unknown screen_mode");
    if (cfg.screen_top < 1 || cfg.screen_top > kScrMaxTop)
        return fail(DPMM_ERR_INVALID_ARG, "screen_top must be in [1, 256]");
    if (!(cfg.alpha > 0)) return fail(DPMM_ERR_INVALID_ARG, "alpha must be positive");
    dpmm_desc desc{};
    desc.n_points = N;
    desc.dim = D;
    desc.prior_type = cfg.prior;
    desc.k_max = cfg.k_max > 0 ? cfg.k_max : 256;
    desc.rng_kind = cfg.rng_kind;
    desc.seed = cfg.seed;
    desc.loglik_mode = cfg.loglik_mode;
    desc.device = cfg.device;
    if (desc.k_max < cfg.initial_clusters + 2) desc.k_max = cfg.initial_clusters + 2;
    DPMM_TRY(dpmm_create(&desc, &h->ctx));
    if (shard) DPMM_TRY(dpmm_set_shard(h->ctx, shard));
    if (f32) DPMM_TRY(dpmm_upload_points_f32(h->ctx, static_cast<const float*>(points)));
    else DPMM_TRY(dpmm_upload_points(h->ctx, static_cast<const double*>(points)));
    if (cfg.prior == DPMM_PRIOR_GAUSSIAN)
        DPMM_TRY(dpmm_set_prior_niw(h->ctx, cfg.hyper.k, cfg.hyper.m.data(), cfg.hyper.v, cfg.hyper.psi.data()));
    else
        DPMM_TRY(dpmm_set_prior_multinomial(h->ctx, cfg.hyper.alpha.data()));
    if (cfg.outlier_mod > 0) {   // the outlier prior on the device: its clusters' draws and ratios
        const host::Hyper& o = cfg.outlier_hyper;
        if (cfg.prior == DPMM_PRIOR_GAUSSIAN) DPMM_TRY(dpmm_set_outlier_prior_niw(h->ctx, o.k, o.m.data(), o.v, o.psi.data()));
        else DPMM_TRY(dpmm_set_outlier_prior_multinomial(h->ctx, o.alpha.data()));
    }
    if (h->ctx->d_prune_rh) DPMM_TRY(dpmm_set_label_pruning(h->ctx, cfg.label_prune_margin));
    if (cfg.verbose && !cfg.gt.empty()) {
        if ((int64_t)cfg.gt.size() != N) return fail(DPMM_ERR_INVALID_ARG, "ground truth needs one value per point");
        DPMM_TRY(dpmm_set_ground_truth(h->ctx, cfg.gt.data()));
    }
    if (cfg.screen_mode == DPMM_SCREEN_ON) {
        if ((int)cfg.screen_params.size() != kScrParams)
            return fail(DPMM_ERR_INVALID_ARG, "screen_mode DPMM_SCREEN_ON needs screen_params");
        DPMM_TRY(dpmm_screen_set_params(h->ctx, cfg.screen_params.data()));
    }
    h->sampler = std::make_unique<Sampler>(cfg, h->ctx, N, D);
    DPMM_TRY(h->sampler->init());
    out = std::move(h);
    return DPMM_OK;
}

dpmm_status run_sampler(const Config& cfg, int64_t N, int D, const void* points, bool f32, dpmm_model_info** out)
{
    std::unique_ptr<SamplerHandle> h;
    DPMM_TRY(make_sampler(cfg, N, D, points, f32, h));
    DPMM_TRY(h->sampler->step(h->cfg.iterations, &h->mi));
    DPMM_TRY(h->sampler->finish(&h->mi));
    *out = new dpmm_model_info(std::move(h->mi));
    return DPMM_OK;
}

static Hyper hyper_from_run(int prior, int D, double k, double v, const double* m, const double* psi, const double* alpha)
{
    Hyper h = default_hyper(prior, D);
    if (prior == DPMM_PRIOR_GAUSSIAN && m && psi) {
        h.k = k;
        h.v = v;
        h.m.assign(m, m + D);
        h.psi.assign(psi, psi + (size_t)D * D);
    } else if (prior == DPMM_PRIOR_MULTINOMIAL && alpha) {
        h.alpha.assign(alpha, alpha + D);
    }
    return h;
}

// niw::create_hyperparams / multinomial_prior::create_hyperparams (niw.cpp:155-193,
// multinomial_prior.cpp:80-96)
static Hyper hyper_from_json(int prior, int D, const io::Json& j)
{
    Hyper h = default_hyper(prior, D);
    if (prior == DPMM_PRIOR_GAUSSIAN) {
        h.k = j["k"].as_double(0.0);
        h.v = j["v"].as_double(0.0);
        const io::Json& m = j["m"];
        if (m.size() > 0) {
            h.m.resize(m.size());
            for (size_t i = 0; i < m.size(); ++i) h.m[i] = m[i].as_double(0.0);
        }
        const io::Json& psi = j["psi"];
        if (psi.size() > 0 && psi[0].size() > 0) {
            const size_t rows = psi.size(), cols = psi[0].size();
            h.psi.assign(rows * cols, 0.0);
            for (size_t r = 0; r < rows; ++r)
                for (size_t c = 0; c < cols; ++c) h.psi[c * rows + r] = psi[r][c].as_double(0.0);
        }
    } else {
        const io::Json& a = j["alpha"];
        if (a.size() > 0) {
            h.alpha.resize(a.size());
            for (size_t i = 0; i < a.size(); ++i) h.alpha[i] = a[i].as_double(0.0);
        }
    }
    return h;
}

}  // namespace host
}  // namespace dpmm

using namespace dpmm;

static void screen_from_run(const dpmm_run_desc* run, host::Config& cfg)
{
    cfg.screen_mode = run->screen_mode;
    cfg.screen_top = run->screen_top > 0 ? run->screen_top : 16;
    cfg.screen_sweep = run->screen_sweep_every > 0 ? run->screen_sweep_every : 10;
    cfg.screen_min_recall = run->screen_min_recall > 0 ? run->screen_min_recall : 0.5;
    cfg.screen_split_min = run->screen_split_min > 0 ? run->screen_split_min : 256;
    cfg.host_param_draws = run->host_param_draws != 0;
    cfg.label_prune_margin = run->label_prune_margin == 0 ? 30.0 : (double)run->label_prune_margin;
    if (run->screen_params) cfg.screen_params.assign(run->screen_params, run->screen_params + kScrParams);
}

static host::Config config_from_run(const dpmm_run_desc* run, int64_t n, int32_t d)
{
    host::Config cfg;
    cfg.prior = run->prior_type;
    cfg.iterations = run->iterations > 0 ? run->iterations : 100;
    cfg.initial_clusters = run->initial_clusters > 0 ? run->initial_clusters : 1;
    cfg.burnout = run->burnout > 0 ? run->burnout : 15;
    cfg.alpha = run->alpha;
    cfg.max_clusters = run->max_clusters > 0 ? run->max_clusters : 1e300;
    cfg.outlier_mod = run->outlier_weight;
    cfg.seed = run->seed;
    cfg.verbose = run->verbose != 0;
    cfg.loglik_mode = run->loglik_mode;
    cfg.rng_kind = run->rng_kind;
    cfg.k_max = run->k_max;
    cfg.device = run->device;
    cfg.hyper = host::hyper_from_run(cfg.prior, d, run->niw_k, run->niw_v, run->niw_m, run->niw_psi, run->mult_alpha);
    cfg.outlier_hyper = host::hyper_from_run(cfg.prior, d, run->out_niw_k, run->out_niw_v, run->out_niw_m,
                                             run->out_niw_psi, run->out_mult_alpha);
    if (run->gt) cfg.gt.assign(run->gt, run->gt + n);
    screen_from_run(run, cfg);
    return cfg;
}

extern "C" dpmm_status dpmm_dp_parallel(const dpmm_run_desc* run, int64_t n, int32_t d, const double* points,
                                        dpmm_model_info** out)
{
    if (!run || !points || !out || n <= 0 || d <= 0) return fail(DPMM_ERR_INVALID_ARG, "invalid argument");
    *out = nullptr;
    return host::run_sampler(config_from_run(run, n, d), n, d, points, false, out);
}

struct dpmm_sampler {
    std::unique_ptr<host::SamplerHandle> h;
};

extern "C" dpmm_status dpmm_sampler_create(const dpmm_run_desc* run, int64_t n, int32_t d, const void* points,
                                           int32_t points_f32, dpmm_sampler** out)
{
    if (!run || !points || !out || n <= 0 || d <= 0) return fail(DPMM_ERR_INVALID_ARG, "invalid argument");
    *out = nullptr;
    auto s = std::make_unique<dpmm_sampler>();
    DPMM_TRY(host::make_sampler(config_from_run(run, n, d), n, d, points, points_f32 != 0, s->h));
    *out = s.release();
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_sampler_create_sharded(const dpmm_run_desc* run, int64_t n, int32_t d, const void* points,
                                                   int32_t points_f32, const dpmm_shard* shard, dpmm_sampler** out)
{
    if (!run || !points || !out || n <= 0 || d <= 0 || !shard) return fail(DPMM_ERR_INVALID_ARG, "invalid argument");
    *out = nullptr;
    if (run->seed == 0 && shard->world > 1)
        return fail(DPMM_ERR_INVALID_ARG, "a sharded run needs an explicit seed (the same on every rank)");
    auto s = std::make_unique<dpmm_sampler>();
    DPMM_TRY(host::make_sampler(config_from_run(run, n, d), n, d, points, points_f32 != 0, s->h, shard));
    *out = s.release();
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_sampler_step(dpmm_sampler* s, int32_t n_iters)
{
    if (!s || n_iters < 0) return fail(DPMM_ERR_INVALID_ARG, "invalid argument");
    return s->h->sampler->step(n_iters, &s->h->mi);
}

extern "C" dpmm_status dpmm_sampler_num_clusters(const dpmm_sampler* s, int32_t* k)
{
    if (!s || !k) return fail(DPMM_ERR_INVALID_ARG, "invalid argument");
    *k = s->h->sampler->num_clusters();
    return DPMM_OK;
}

extern "C" void* dpmm_sampler_stream(const dpmm_sampler* s) { return s ? (void*)s->h->ctx->stream : nullptr; }

extern "C" dpmm_ctx* dpmm_sampler_context(const dpmm_sampler* s) { return s ? s->h->ctx : nullptr; }

extern "C" dpmm_status dpmm_sampler_model_info(dpmm_sampler* s, dpmm_model_info** out)
{
    if (!s || !out) return fail(DPMM_ERR_INVALID_ARG, "invalid argument");
    DPMM_TRY(s->h->sampler->finish(&s->h->mi));
    *out = new dpmm_model_info(s->h->mi);
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_sampler_destroy(dpmm_sampler* s)
{
    delete s;
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_dp_parallel_from_file(const char* npy_path, const char* params_path, int32_t prior_type,
                                                  const dpmm_run_desc* ov, dpmm_model_info** out)
{
    if (!npy_path || !params_path || !out) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    std::vector<double> pts;
    int64_t rows = 0, cols = 0;
    std::string err;
    if (!io::read_npy(npy_path, pts, rows, cols, err)) return fail(DPMM_ERR_IO, err);
    std::string text;
    if (!io::read_file(params_path, text)) return fail(DPMM_ERR_IO, std::string("cannot read ") + params_path);
    io::Json root;
    if (!io::parse_json(text, root, err)) return fail(DPMM_ERR_IO, "params JSON: " + err);
    const int D = (int)cols;
    host::Config cfg;   // global_params.h:37-78 defaults, then global_params.cpp:25-65 keys
    cfg.prior = prior_type;
    cfg.burnout = 20;
    cfg.outlier_mod = 0.05;
    cfg.alpha = root["alpha"].as_double(10.0);
    cfg.hyper = root["hyper_params"].is_null() ? host::default_hyper(prior_type, D)
                                               : host::hyper_from_json(prior_type, D, root["hyper_params"]);
    cfg.iterations = (int)root["iterations"].as_int(100);
    cfg.initial_clusters = (int)root["initial_clusters"].as_int(1);
    cfg.verbose = root["use_verbose"].as_bool(false);
    cfg.burnout = (int)root["burnout_period"].as_int(20);
    cfg.max_clusters = root["max_num_of_clusters"].as_double(1e300);
    cfg.outlier_mod = root["outlier_mod"].as_double(0.05);
    cfg.outlier_hyper = root["outlier_hyper_params"].is_null()
                            ? host::default_hyper(prior_type, D)
                            : host::hyper_from_json(prior_type, D, root["outlier_hyper_params"]);
    cfg.seed = (uint64_t)root["randomSeed"].as_double(0);
    const io::Json& gt = root["gt"];
    for (size_t i = 0; i < gt.size(); ++i) cfg.gt.push_back((int32_t)gt[i].as_int(0));
    // force_kernel (global_params.cpp:65): 1 -> SIMT FP32 contraction, 2 -> tensor cores
    int fk = (int)root["force_kernel"].as_int(0);
    cfg.loglik_mode = fk == 1 ? DPMM_LL_FP32 : fk == 2 ? DPMM_LL_TC_BF16X3 : DPMM_LL_AUTO;
    if (ov) {
        cfg.loglik_mode = ov->loglik_mode;
        cfg.rng_kind = ov->rng_kind;
        cfg.k_max = ov->k_max;
        cfg.device = ov->device;
        if (ov->seed) cfg.seed = ov->seed;
        screen_from_run(ov, cfg);
    }
    return host::run_sampler(cfg, rows, D, pts.data(), false, out);
}

extern "C" int64_t dpmm_model_info_n(const dpmm_model_info* mi) { return mi ? mi->n : 0; }
extern "C" const int32_t* dpmm_model_info_labels(const dpmm_model_info* mi) { return mi ? mi->labels.data() : nullptr; }
extern "C" int32_t dpmm_model_info_num_weights(const dpmm_model_info* mi) { return mi ? (int32_t)mi->weights.size() : 0; }
extern "C" const double* dpmm_model_info_weights(const dpmm_model_info* mi) { return mi ? mi->weights.data() : nullptr; }
extern "C" int32_t dpmm_model_info_iterations(const dpmm_model_info* mi) { return mi ? (int32_t)mi->iter_count.size() : 0; }
extern "C" const double* dpmm_model_info_iter_count(const dpmm_model_info* mi) { return mi ? mi->iter_count.data() : nullptr; }
extern "C" const double* dpmm_model_info_likelihood_history(const dpmm_model_info* mi)
{
    return mi ? mi->likelihood_history.data() : nullptr;
}
extern "C" const double* dpmm_model_info_nmi_history(const dpmm_model_info* mi)
{
    return (mi && !mi->nmi_history.empty()) ? mi->nmi_history.data() : nullptr;
}
extern "C" const int32_t* dpmm_model_info_cluster_count_history(const dpmm_model_info* mi)
{
    return mi ? mi->cluster_count_history.data() : nullptr;
}

extern "C" dpmm_status dpmm_model_info_write_json(const dpmm_model_info* mi, const char* path)
{
    if (!mi || !path) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    std::ofstream f(path);
    if (!f) return fail(DPMM_ERR_IO, std::string("cannot write ") + path);
    char buf[64];
    f << "{\"labels\": [";
    for (size_t i = 0; i < mi->labels.size(); ++i) f << (i ? ", " : "") << mi->labels[i];
    f << "], \"weights\": [";
    for (size_t i = 0; i < mi->weights.size(); ++i) {
        std::snprintf(buf, sizeof(buf), "%.17g", mi->weights[i]);
        f << (i ? ", " : "") << buf;
    }
    f << "], \"iter_count\": [";
    for (size_t i = 0; i < mi->iter_count.size(); ++i) {
        std::snprintf(buf, sizeof(buf), "%.9g", mi->iter_count[i]);
        f << (i ? ", " : "") << buf;
    }
    f << "]}\n";
    return f ? DPMM_OK : fail(DPMM_ERR_IO, "write failed");
}

extern "C" dpmm_status dpmm_model_info_screen_stats(const dpmm_model_info* mi, int64_t* out)
{
    if (!mi || !out) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    const host::ScreenRecord& r = mi->screen;
    const int64_t v[8] = {r.split_cand, r.split_exact, r.merge_cand, r.merge_exact,
                          r.sweeps,     r.sweep_accepts, r.sweep_hits, r.disabled_at};
    std::memcpy(out, v, sizeof(v));
    return DPMM_OK;
}
extern "C" int64_t dpmm_model_info_screen_log_rows(const dpmm_model_info* mi)
{
    return mi ? (int64_t)mi->screen.log_hr.size() : 0;
}
extern "C" const float* dpmm_model_info_screen_log_features(const dpmm_model_info* mi)
{
    return (mi && !mi->screen.log_features.empty()) ? mi->screen.log_features.data() : nullptr;
}
extern "C" const double* dpmm_model_info_screen_log_hr(const dpmm_model_info* mi)
{
    return (mi && !mi->screen.log_hr.empty()) ? mi->screen.log_hr.data() : nullptr;
}
extern "C" const int8_t* dpmm_model_info_screen_log_kind(const dpmm_model_info* mi)
{
    return (mi && !mi->screen.log_kind.empty()) ? mi->screen.log_kind.data() : nullptr;
}

extern "C" const int32_t* dpmm_model_info_screen_log_iter(const dpmm_model_info* mi)
{
    return (mi && !mi->screen.log_iter.empty()) ? mi->screen.log_iter.data() : nullptr;
}

extern "C" void dpmm_model_info_free(dpmm_model_info* mi) { delete mi; }

// ============================================================================== batches of samplers
// Many independent samplers (data sets of uneven N, D and K) advanced together, one iteration at a
// time: the host stages of all samplers run on a thread pool, and the label phase of every NIW data
// set of a padded dimension is ONE launch over a work list of (data set, block of points) items,
// replayed from a CUDA graph; the points per block are chosen per padded dimension by timing the
// candidates on the first iteration.  The reference can run one sampler per process only (its init
// calls cudaDeviceReset, cudaKernel.cu:615).
struct dpmm_batch {
    struct Group {
        int Dp = 0, kcap = 0, P = 0;
        std::vector<int> members;          // sampler indices
        std::vector<int> graph_members;    // the members the captured graph covers
        LabelJob* h_jobs = nullptr;        // pinned
        LabelJob* d_jobs = nullptr;
        int2* d_items = nullptr;
        int nitems = 0;
        cudaStream_t st = nullptr;
        cudaEvent_t done = nullptr;
        cudaGraphExec_t graph = nullptr;
        float tune_ms[3] = {0, 0, 0};
    };
    std::vector<std::unique_ptr<dpmm::host::SamplerHandle>> s;
    std::vector<Group> groups;
    std::vector<int> group_of;
    std::vector<cudaEvent_t> ready;
    int device = 0;
    int64_t batched_launches = 0, graph_launches = 0;
    ~dpmm_batch()
    {
        cudaSetDevice(device);
        for (Group& g : groups) {
            if (g.st) cudaStreamSynchronize(g.st);
            if (g.graph) cudaGraphExecDestroy(g.graph);
            if (g.h_jobs) cudaFreeHost(g.h_jobs);
            if (g.d_jobs) cudaFree(g.d_jobs);
            if (g.d_items) cudaFree(g.d_items);
            if (g.done) cudaEventDestroy(g.done);
            if (g.st) cudaStreamDestroy(g.st);
        }
        for (cudaEvent_t e : ready)
            if (e) cudaEventDestroy(e);
        s.clear();
    }
};

namespace dpmm {
namespace host {

static const int kBatchP[3] = {32, 64, 128};

// work list of a group for P points per block: one item per (job j, block) of the members in order
static dpmm_status batch_items(dpmm_batch& b, dpmm_batch::Group& g, const std::vector<int>& mem, int P)
{
    std::vector<int2> items;
    for (size_t j = 0; j < mem.size(); ++j) {
        const int64_t N = b.s[mem[j]]->sampler->context()->N;
        for (int64_t blk = 0; blk * P < N; ++blk) items.push_back(make_int2((int)j, (int)blk));
    }
    if (g.d_items) cudaFree(g.d_items);
    g.d_items = nullptr;
    DPMM_CUDA_TRY(cudaMalloc(&g.d_items, sizeof(int2) * std::max<size_t>(items.size(), 1)));
    DPMM_CUDA_TRY(cudaMemcpy(g.d_items, items.data(), sizeof(int2) * items.size(), cudaMemcpyHostToDevice));
    g.nitems = (int)items.size();
    return DPMM_OK;
}

// the label phase of one group; its members' parameters are ready (g.st waits on their events)
static dpmm_status batch_labels(dpmm_batch& b, dpmm_batch::Group& g, const std::vector<int>& mem,
                                const std::vector<Sampler::IterState>& st)
{
    for (size_t j = 0; j < mem.size(); ++j) {
        Sampler& sm = *b.s[mem[j]]->sampler;
        DPMM_TRY(make_label_job(sm.context(), sm.num_clusters(), st[mem[j]].final_ ? 1 : 0, &g.h_jobs[j]));
    }
    const size_t jb = sizeof(LabelJob) * mem.size();
    if (g.P == 0) {
        // first iteration: time every block size on the live jobs (each run draws the same labels:
        // a point's log-likelihoods and uniforms do not depend on the block size), keep the fastest
        cudaEvent_t e0, e1;
        DPMM_CUDA_TRY(cudaEventCreate(&e0));
        DPMM_CUDA_TRY(cudaEventCreate(&e1));
        DPMM_CUDA_TRY(cudaMemcpyAsync(g.d_jobs, g.h_jobs, jb, cudaMemcpyHostToDevice, g.st));
        int best = 0;
        for (int q = 0; q < 3; ++q) {
            DPMM_TRY(batch_items(b, g, mem, kBatchP[q]));
            DPMM_CUDA_TRY(cudaEventRecord(e0, g.st));
            DPMM_TRY(launch_labels_batched(g.Dp, kBatchP[q], g.d_jobs, g.d_items, g.nitems, g.kcap, g.st));
            DPMM_CUDA_TRY(cudaEventRecord(e1, g.st));
            DPMM_CUDA_TRY(cudaEventSynchronize(e1));
            DPMM_CUDA_TRY(cudaEventElapsedTime(&g.tune_ms[q], e0, e1));
            if (g.tune_ms[q] < g.tune_ms[best]) best = q;
            ++b.batched_launches;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        g.P = kBatchP[best];
        DPMM_TRY(batch_items(b, g, mem, g.P));
        return DPMM_OK;
    }
    if (!g.graph || g.graph_members != mem) {
        // (re)capture: jobs upload + the batched launch
        if (g.graph) {
            cudaGraphExecDestroy(g.graph);
            g.graph = nullptr;
        }
        DPMM_TRY(batch_items(b, g, mem, g.P));
        cudaGraph_t graph;
        DPMM_CUDA_TRY(cudaStreamBeginCapture(g.st, cudaStreamCaptureModeRelaxed));
        cudaMemcpyAsync(g.d_jobs, g.h_jobs, jb, cudaMemcpyHostToDevice, g.st);
        dpmm_status ls = launch_labels_batched(g.Dp, g.P, g.d_jobs, g.d_items, g.nitems, g.kcap, g.st);
        cudaError_t ce = cudaStreamEndCapture(g.st, &graph);
        DPMM_TRY(ls);
        DPMM_CUDA_TRY(ce);
        ce = cudaGraphInstantiate(&g.graph, graph, 0);
        cudaGraphDestroy(graph);
        DPMM_CUDA_TRY(ce);
        g.graph_members = mem;
    }
    DPMM_CUDA_TRY(cudaGraphLaunch(g.graph, g.st));
    ++b.graph_launches;
    ++b.batched_launches;
    return DPMM_OK;
}

static dpmm_status batch_iteration(dpmm_batch& b)
{
    const int n = (int)b.s.size();
    std::vector<Sampler::IterState> st(n);
    std::vector<uint8_t> act(n, 0);
    for (int i = 0; i < n; ++i) act[i] = b.s[i]->sampler->running();
    std::vector<dpmm_status> err(n, DPMM_OK);
    std::vector<std::string> msg(n);
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < n; ++i) {
        if (!act[i]) continue;
        Sampler& sm = *b.s[i]->sampler;
        st[i] = sm.begin_iteration();
        dpmm_status e = sm.stage_params();
        if (e == DPMM_OK && b.group_of[i] < 0)   // not batched: the context's own label phase
            e = dpmm_create_clusters_labels(sm.context(), sm.num_clusters(), st[i].final_ ? 1 : 0, nullptr, nullptr);
        if (e == DPMM_OK && b.group_of[i] >= 0) {
            cudaError_t ce = cudaEventRecord(b.ready[i], sm.context()->stream);
            if (ce != cudaSuccess) e = cuda_status(ce, "cudaEventRecord");
        }
        if (e != DPMM_OK) {
            err[i] = e;
            msg[i] = dpmm_last_error();
        }
    }
    for (int i = 0; i < n; ++i)
        if (err[i] != DPMM_OK) return fail(err[i], "data set " + std::to_string(i) + ": " + msg[i]);
    for (dpmm_batch::Group& g : b.groups) {
        std::vector<int> mem;
        for (int m : g.members)
            if (act[m]) mem.push_back(m);
        if (mem.empty()) continue;
        for (int m : mem) DPMM_CUDA_TRY(cudaStreamWaitEvent(g.st, b.ready[m], 0));
        DPMM_TRY(batch_labels(b, g, mem, st));
        DPMM_CUDA_TRY(cudaEventRecord(g.done, g.st));
        for (int m : mem) DPMM_CUDA_TRY(cudaStreamWaitEvent(b.s[m]->sampler->context()->stream, g.done, 0));
    }
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < n; ++i) {
        if (!act[i]) continue;
        Sampler& sm = *b.s[i]->sampler;
        dpmm_status e = sm.stage_rest(st[i].no_more_splits, st[i].final_);
        if (e == DPMM_OK) e = sm.end_iteration(st[i], &b.s[i]->mi);
        if (e != DPMM_OK) {
            err[i] = e;
            msg[i] = dpmm_last_error();
        }
    }
    for (int i = 0; i < n; ++i)
        if (err[i] != DPMM_OK) return fail(err[i], "data set " + std::to_string(i) + ": " + msg[i]);
    return DPMM_OK;
}

}  // namespace host
}  // namespace dpmm

extern "C" dpmm_status dpmm_batch_create(int32_t count, const dpmm_run_desc* runs, const int64_t* n, const int32_t* d,
                                         const double* const* points, dpmm_batch** out)
{
    if (count < 1 || !runs || !n || !d || !points || !out) return fail(DPMM_ERR_INVALID_ARG, "invalid argument");
    *out = nullptr;
    auto b = std::make_unique<dpmm_batch>();
    b->device = runs[0].device;
    for (int i = 0; i < count; ++i)
        if (runs[i].device != b->device) return fail(DPMM_ERR_INVALID_ARG, "all data sets of a batch share one device");
    b->s.resize(count);
    std::vector<dpmm_status> err(count, DPMM_OK);
    std::vector<std::string> msg(count);
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < count; ++i) {
        if (n[i] <= 0 || d[i] <= 0 || !points[i]) {
            err[i] = DPMM_ERR_INVALID_ARG;
            msg[i] = "invalid data set";
            continue;
        }
        host::Config cfg = config_from_run(&runs[i], n[i], d[i]);
        if (cfg.prior == DPMM_PRIOR_GAUSSIAN) cfg.loglik_mode = DPMM_LL_FP32;   // the batched SIMT label kernel
        if (cudaSetDevice(b->device) != cudaSuccess) {
            err[i] = DPMM_ERR_NO_DEVICE;
            continue;
        }
        dpmm_status e = host::make_sampler(cfg, n[i], d[i], points[i], false, b->s[i]);
        if (e != DPMM_OK) {
            err[i] = e;
            msg[i] = dpmm_last_error();
        }
    }
    for (int i = 0; i < count; ++i)
        if (err[i] != DPMM_OK) return fail(err[i], "data set " + std::to_string(i) + ": " + msg[i]);
    DPMM_CUDA_TRY(cudaSetDevice(b->device));
    b->group_of.assign(count, -1);
    b->ready.assign(count, nullptr);
    for (int i = 0; i < count; ++i) {
        dpmm_ctx* c = b->s[i]->sampler->context();
        if (c->prior != DPMM_PRIOR_GAUSSIAN) continue;
        int gi = -1;
        for (size_t q = 0; q < b->groups.size(); ++q)
            if (b->groups[q].Dp == c->Dp) gi = (int)q;
        if (gi < 0) {
            b->groups.emplace_back();
            gi = (int)b->groups.size() - 1;
            b->groups[gi].Dp = c->Dp;
        }
        b->groups[gi].members.push_back(i);
        b->groups[gi].kcap = std::max(b->groups[gi].kcap, c->k_max);
        b->group_of[i] = gi;
        DPMM_CUDA_TRY(cudaEventCreateWithFlags(&b->ready[i], cudaEventDisableTiming));
    }
    for (dpmm_batch::Group& g : b->groups) {
        DPMM_CUDA_TRY(cudaStreamCreateWithFlags(&g.st, cudaStreamNonBlocking));
        DPMM_CUDA_TRY(cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming));
        DPMM_CUDA_TRY(cudaMallocHost(&g.h_jobs, sizeof(LabelJob) * g.members.size()));
        DPMM_CUDA_TRY(cudaMalloc(&g.d_jobs, sizeof(LabelJob) * g.members.size()));
        if (gauss_label_smem_bytes(g.Dp, 128, g.kcap) > 220 * 1024)
            return fail(DPMM_ERR_INVALID_ARG, "k_max too large for the batched label kernel at this dimension");
    }
    *out = b.release();
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_batch_step(dpmm_batch* b, int32_t n_iters)
{
    if (!b || n_iters < 0) return fail(DPMM_ERR_INVALID_ARG, "invalid argument");
    DPMM_CUDA_TRY(cudaSetDevice(b->device));
    for (int q = 0; q < n_iters; ++q) DPMM_TRY(host::batch_iteration(*b));
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_batch_info(const dpmm_batch* b, int64_t* out)
{
    if (!b || !out) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    out[0] = (int64_t)b->s.size();
    out[1] = (int64_t)b->groups.size();
    out[2] = b->batched_launches;
    out[3] = b->graph_launches;
    const int dps[6] = {4, 8, 16, 32, 64, 128};
    for (int q = 0; q < 6; ++q) {
        out[4 + q] = 0;
        for (const auto& g : b->groups)
            if (g.Dp == dps[q]) out[4 + q] = g.P;
    }
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_batch_model_info(dpmm_batch* b, int32_t index, dpmm_model_info** out)
{
    if (!b || !out || index < 0 || index >= (int)b->s.size()) return fail(DPMM_ERR_INVALID_ARG, "invalid argument");
    DPMM_TRY(b->s[index]->sampler->finish(&b->s[index]->mi));
    *out = new dpmm_model_info(b->s[index]->mi);
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_batch_destroy(dpmm_batch* b)
{
    delete b;
    return DPMM_OK;
}

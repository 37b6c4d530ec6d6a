// ref_shim.cpp -- C entry points over the reference's OWN compiled host code.
//
// TEST INFRASTRUCTURE ONLY.  Linked (by oracle/Makefile) against object files compiled
// out-of-tree from the reference sources, so that tests can compare the C restatement
// (dpmm_oracle.c) and the CUDA path with the reference's real arithmetic:
//   niw::calc_posterior / log_marginal_likelihood        (priors/niw.cpp:23-49, :122-138)
//   multinomial_prior::calc_posterior / lml               (priors/multinomial_prior.cpp:12-22, :56-67)
//   r8_gamma_log                                          (distributions_util/pdflib.cpp)
//   utils::log_multivariate_gamma                         (utils.cpp:94-102)
//   local_clusters_actions::should_split_local            (local_clusters_actions.cpp:215-242)
//   shared_actions::should_merge                          (shared_actions.cpp:88-111)
// No GPU is touched: the global_params objects built here never create a cudaKernel.
#include <memory>
#include <random>
#include <vector>
#include "global_params.h"
#include "local_clusters_actions.h"
#include "shared_actions.h"
#include "utils.h"
#include "priors/niw.h"
#include "priors/niw_hyperparams.h"
#include "priors/niw_sufficient_statistics.h"
#include "priors/multinomial_prior.h"
#include "priors/multinomial_hyper.h"
#include "priors/multinomial_sufficient_statistics.h"
#include "distributions_util/pdflib.hpp"

namespace {

std::shared_ptr<niw_hyperparams> niw_hp(int d, double k, const double* m, double v, const double* psi)
{
    auto h = std::make_shared<niw_hyperparams>();
    h->k = k;
    h->v = v;
    h->m = Eigen::Map<const Eigen::VectorXd>(m, d);
    h->psi = Eigen::Map<const Eigen::MatrixXd>(psi, d, d);
    return h;
}

std::shared_ptr<sufficient_statistics> niw_ss(int d, int n, const double* sum, const double* S)
{
    return std::make_shared<niw_sufficient_statistics>(n, Eigen::Map<const Eigen::VectorXd>(sum, d),
                                                       Eigen::Map<const Eigen::MatrixXd>(S, d, d));
}

std::shared_ptr<sufficient_statistics> mult_ss(int d, int n, const double* sum)
{
    return std::make_shared<multinomial_sufficient_statistics>(n, Eigen::Map<const Eigen::VectorXd>(sum, d));
}

std::shared_ptr<global_params> host_params(prior_type pt, unsigned long long seed)
{
    auto gp = std::make_shared<global_params>();
    gp->init_prior(pt);
    gp->init_random(seed);
    return gp;
}

// cluster_parameters with prior, stats and the posterior the sampler would hold
std::shared_ptr<cluster_parameters> make_cp(prior& pr, const std::shared_ptr<hyperparams>& hp,
                                            const std::shared_ptr<sufficient_statistics>& ss)
{
    auto cp = std::make_shared<cluster_parameters>();
    cp->prior_hyperparams = hp->clone();
    cp->suff_statistics = ss;
    cp->posterior_hyperparams = pr.calc_posterior(hp, ss);
    return cp;
}

class scripted_shared_actions : public shared_actions {
public:
    scripted_shared_actions(std::shared_ptr<global_params>& gp, double u) : shared_actions(gp), u_(u) {}
protected:
    double get_uniform_real_distribution() override { return u_; }
private:
    double u_;
};

}  // namespace

extern "C" {

double ref_r8_gamma_log(double x) { return r8_gamma_log(x); }

double ref_log_multivariate_gamma(double x, int d) { return utils::log_multivariate_gamma(x, d); }

void ref_niw_posterior(int d, double k, const double* m, double v, const double* psi, int n,
                       const double* sum, const double* S, double* k_out, double* m_out,
                       double* v_out, double* psi_out)
{
    niw pr;
    auto post = std::dynamic_pointer_cast<niw_hyperparams>(pr.calc_posterior(niw_hp(d, k, m, v, psi), niw_ss(d, n, sum, S)));
    *k_out = post->k;
    *v_out = post->v;
    Eigen::Map<Eigen::VectorXd>(m_out, d) = post->m;
    Eigen::Map<Eigen::MatrixXd>(psi_out, d, d) = post->psi;
}

double ref_niw_lml(int d, double k0, const double* m0, double v0, const double* psi0, double kp,
                   const double* mp, double vp, const double* psip, int n)
{
    niw pr;
    std::vector<double> zeros((size_t)d * d, 0.0);
    return pr.log_marginal_likelihood(niw_hp(d, k0, m0, v0, psi0), niw_hp(d, kp, mp, vp, psip),
                                      niw_ss(d, n, zeros.data(), zeros.data()));
}

void ref_mult_posterior(int d, const double* alpha, int n, const double* sum, double* alpha_out)
{
    multinomial_prior pr;
    auto h = std::make_shared<multinomial_hyper>(Eigen::Map<const Eigen::VectorXd>(alpha, d));
    auto post = std::dynamic_pointer_cast<multinomial_hyper>(pr.calc_posterior(h, mult_ss(d, n, sum)));
    Eigen::Map<Eigen::VectorXd>(alpha_out, d) = post->alpha;
}

double ref_mult_lml(int d, const double* alpha0, const double* alphap)
{
    multinomial_prior pr;
    std::vector<double> zeros((size_t)d, 0.0);
    auto h0 = std::make_shared<multinomial_hyper>(Eigen::Map<const Eigen::VectorXd>(alpha0, d));
    auto hp = std::make_shared<multinomial_hyper>(Eigen::Map<const Eigen::VectorXd>(alphap, d));
    return pr.log_marginal_likelihood(h0, hp, mult_ss(d, 0, zeros.data()));
}

// Split test of one cluster. n[3], sum[3*d], S[3*d*d] hold cluster, l, r statistics (S may be
// NULL for the multinomial prior).  Returns log_HR assembled from the reference's building
// blocks exactly as local_clusters_actions.cpp:222-233 does; *decision is the reference's own
// should_split_local run with an mt19937 seeded by `seed`, and *u_used the uniform it drew.
double ref_split_log_hr(int prior_kind, int d, double k0, const double* m0, double v0,
                        const double* psi0, const double* alpha0, double alpha, const int* n,
                        const double* sum, const double* S, unsigned long long seed,
                        int final_, int* decision, double* u_used)
{
    prior_type pt = prior_kind == 0 ? prior_type::Gaussian : prior_type::Multinomial;
    auto gp = host_params(pt, seed);
    std::shared_ptr<hyperparams> hp;
    std::shared_ptr<sufficient_statistics> ss[3];
    for (int q = 0; q < 3; ++q)
        ss[q] = pt == prior_type::Gaussian ? niw_ss(d, n[q], sum + (size_t)q * d, S + (size_t)q * d * d)
                                           : mult_ss(d, n[q], sum + (size_t)q * d);
    if (pt == prior_type::Gaussian) hp = niw_hp(d, k0, m0, v0, psi0);
    else hp = std::make_shared<multinomial_hyper>(Eigen::Map<const Eigen::VectorXd>(alpha0, d));

    auto scp = std::make_shared<splittable_cluster_params>();
    scp->cluster_params = make_cp(*gp->pPrior, hp, ss[0]);
    scp->cluster_params_l = make_cp(*gp->pPrior, hp, ss[1]);
    scp->cluster_params_r = make_cp(*gp->pPrior, hp, ss[2]);

    prior& pr = *gp->pPrior;
    auto post = pr.calc_posterior(hp, ss[0]);
    auto lpost = pr.calc_posterior(hp, ss[1]);
    auto rpost = pr.calc_posterior(hp, ss[2]);
    double ll_l = pr.log_marginal_likelihood(hp, lpost, ss[1]);
    double ll_r = pr.log_marginal_likelihood(hp, rpost, ss[2]);
    double ll = pr.log_marginal_likelihood(hp, post, ss[0]);
    double log_hr = log(alpha) + r8_gamma_log(n[1]) + ll_l + r8_gamma_log(n[2]) + ll_r -
                    (r8_gamma_log(n[0]) + ll);

    std::mt19937 probe((unsigned long)seed);
    std::uniform_real_distribution<double> dist(0, 1);
    *u_used = dist(probe);

    local_clusters_actions lca(gp);
    int should_split = 0;
    lca.should_split_local(should_split, scp, alpha, final_ != 0);
    *decision = should_split;
    return log_hr;
}

// Merge test of clusters i (slot 0) and j (slot 1).  Returns log_HR assembled as
// shared_actions.cpp:90-99 does; *decision is the reference's own should_merge run with the
// scripted uniform u.
double ref_merge_log_hr(int prior_kind, int d, double k0, const double* m0, double v0,
                        const double* psi0, const double* alpha0, double alpha, const int* n,
                        const double* sum, const double* S, double u, int final_, int* decision)
{
    prior_type pt = prior_kind == 0 ? prior_type::Gaussian : prior_type::Multinomial;
    auto gp = host_params(pt, 1);
    std::shared_ptr<hyperparams> hp;
    std::shared_ptr<sufficient_statistics> ss[2];
    for (int q = 0; q < 2; ++q)
        ss[q] = pt == prior_type::Gaussian ? niw_ss(d, n[q], sum + (size_t)q * d, S + (size_t)q * d * d)
                                           : mult_ss(d, n[q], sum + (size_t)q * d);
    if (pt == prior_type::Gaussian) hp = niw_hp(d, k0, m0, v0, psi0);
    else hp = std::make_shared<multinomial_hyper>(Eigen::Map<const Eigen::VectorXd>(alpha0, d));
    prior& pr = *gp->pPrior;
    auto cpl = make_cp(pr, hp, ss[0]);
    auto cpr = make_cp(pr, hp, ss[1]);

    std::shared_ptr<cluster_parameters> cp = cpl->clone();
    pr.aggregate_suff_stats(cpl->suff_statistics, cpr->suff_statistics, cp->suff_statistics);
    cp->posterior_hyperparams = pr.calc_posterior(cp->prior_hyperparams, cp->suff_statistics);
    double ll_l = pr.log_marginal_likelihood(cpl->prior_hyperparams, cpl->posterior_hyperparams, cpl->suff_statistics);
    double ll_r = pr.log_marginal_likelihood(cpr->prior_hyperparams, cpr->posterior_hyperparams, cpr->suff_statistics);
    double ll = pr.log_marginal_likelihood(cp->prior_hyperparams, cp->posterior_hyperparams, cp->suff_statistics);
    int N = cp->suff_statistics->N, Nl = cpl->suff_statistics->N, Nr = cpr->suff_statistics->N;
    double log_hr = (-log(alpha) + r8_gamma_log(alpha) - 2 * r8_gamma_log(0.5 * alpha) + r8_gamma_log(N) -
                     r8_gamma_log(N + alpha) + r8_gamma_log(Nl + 0.5 * alpha) - r8_gamma_log(Nl) -
                     r8_gamma_log(Nr) + r8_gamma_log(Nr + 0.5 * alpha) + ll - ll_l - ll_r);

    // the reference's own decision; fresh copies so its aggregation does not alias ours
    auto cpl2 = make_cp(pr, hp, ss[0]->clone());
    auto cpr2 = make_cp(pr, hp, ss[1]->clone());
    scripted_shared_actions sa(gp, u);
    bool merge = false;
    sa.should_merge(merge, cpl2, cpr2, alpha, final_ != 0);
    *decision = merge ? 1 : 0;
    return log_hr;
}

}  // extern "C"

/*
 * dpmm_oracle.h -- CPU FP64 restatement of the per-iteration data-parallel path
 * of the sub-cluster DPMM sampler (BGU-CS-VIL/DPMMSubClusters_GPU).
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path is
 * compared against.  It is never linked into, loaded by, or called from the
 * product library (dpmmsubclusters_gpu_b200/libdpmm_b200.so); only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm use it.
 *
 * Conventions follow the reference exactly:
 *   - points are point-major (D x N column-major in Eigen terms == N x D row-major),
 *   - labels are 1-based int32, sub-labels are in {1, 2},
 *   - every per-point quantity is FP64.
 * Each function names the reference file:line it restates.
 */
#ifndef DPMM_ORACLE_H
#define DPMM_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* cudaKernel_gaussian.cu:82-113 + cudaKernel.cu:336-350 (dcolwise_dot_with_log_kernel).
 * r[n] = -(D*D*log(2*pi) + logdet_sigma)/2 - 0.5*(x-mu)^T inv_sigma (x-mu) + log(weight).
 * add_log_weight = 0 gives the sub-cluster form (cudaKernel_gaussian.cu:43-79, cudaKernel.cu:320-334). */
void or_gauss_loglik(int64_t n, int d, const double* x, const double* mu,
                     const double* inv_sigma, double logdet_sigma, double weight,
                     int add_log_weight, double* r);

/* cudaKernel_multinomial.cu:22-35 / :60-76: r[n] = sum_d x[n,d] * log_theta[d] (no weight term). */
void or_mult_loglik(int64_t n, int d, const double* x, const double* log_theta, double* r);

/* cudaKernel.cu:374-403: in-place row softmax of an N x K column-major matrix. */
void or_softmax_rows(int64_t n, int k, double* r);

/* cudaKernel.cu:27-124: Walker alias draw over k probabilities p[0..k-1] from two
 * uniforms; returns the 1-based category.  work must hold 2*(k+2) ints and (k+2) doubles.
 * margin (nullable) receives the smallest |y - threshold| over every comparison the
 * construction and the draw made: a perturbation of the probabilities smaller than that
 * cannot change the result. */
int or_alias_draw(int k, const double* p, double u1, double u2, double* margin,
                  double* ywork, int* iwork);

/* cudaKernel.cu:805-829 + :126-133 (or :405-424 when final): label phase from an
 * N x K column-major log-likelihood matrix r (softmax applied in place unless final).
 * u holds 2 uniforms per point (u[2n], u[2n+1]); margin (nullable) per point. */
void or_sample_labels(int64_t n, int k, double* r, const double* u, int final_,
                      int32_t* labels, double* margin);

/* cudaKernel.cu:352-372 + :135-142: sub-cluster draw for the points of one cluster.
 * r is m x 2 column-major (l then r log-likelihoods, no weights yet); lr_weights[2]. */
void or_sample_sub_from_loglik(int64_t m, double* r, const double* lr_weights, const double* u,
                               int32_t* sub_labels, double* margin);

/* cudaKernel.cu:1299-1398 with cudaKernel_gaussian.cu:43-79: full sub-label phase for
 * K clusters.  Per cluster c: mu_lr[(2c+s)*D], inv_sigma_lr[(2c+s)*D*D], logdet_lr[2c+s],
 * lr_weights[2c+s], s = 0 (l), 1 (r).  u has 2 uniforms per point (indexed by point). */
void or_gauss_sub_labels(int64_t n, int d, const double* x, const int32_t* labels, int k,
                         const double* mu_lr, const double* inv_sigma_lr, const double* logdet_lr,
                         const double* lr_weights, const double* u, int32_t* sub_labels,
                         double* margin, double* r_out /* nullable, n x 2 point-major */);

/* cudaKernel_multinomial.cu:37-58 form of the above. log_theta_lr[(2c+s)*D]. */
void or_mult_sub_labels(int64_t n, int d, const double* x, const int32_t* labels, int k,
                        const double* log_theta_lr, const double* lr_weights, const double* u,
                        int32_t* sub_labels, double* margin, double* r_out);

/* cudaKernel.cu:844-941 + cudaKernel_gaussian.cu:126-168: per cluster c in 0..k-1 the
 * statistics of the cluster (slot 3c), its l sub-cluster (3c+1) and r sub-cluster (3c+2):
 * count[3k], sum[3k*D], and (if S != NULL) the uncentred scatter S[3k*D*D] = sum x x^T. */
void or_suff_stats(int64_t n, int d, const double* x, const int32_t* labels,
                   const int32_t* sub_labels, int k, int64_t* count, double* sum, double* S);

/* Label maintenance, cudaKernel.cu:144-279.  bits[n] stands for curand() of point n. */
void or_sample_labels_init(int64_t n, const double* u, int initial_clusters, double outlier_mod,
                           int32_t* labels);                                   /* :158-170 */
void or_sample_sub_labels_init(int64_t n, const double* u, int32_t* sub_labels); /* :144-156 */
void or_split_cluster(int64_t n, int32_t* labels, int32_t* sub_labels, int index, int new_index,
                      const uint32_t* bits);                                   /* :202-221 */
void or_merge_clusters(int64_t n, int32_t* labels, int32_t* sub_labels, int index, int new_index); /* :223-246 */
void or_reset_bad_cluster(int64_t n, const int32_t* labels, int32_t* sub_labels, int index,
                          const uint32_t* bits);                               /* :248-263 */
void or_remove_empty_cluster(int64_t n, int32_t* labels, int limit);           /* :172-187 */
void or_sub_labels_count(int64_t n, const int32_t* sub_labels, int* l, int* r); /* :265-279 */

/* priors/niw.cpp:23-49 (calc_posterior). Outputs k', m'[D], v', psi'[D*D]. */
void or_niw_posterior(int d, double k, const double* m, double v, const double* psi,
                      int64_t count, const double* sum, const double* S,
                      double* k_out, double* m_out, double* v_out, double* psi_out);
/* distributions_util/logdet.h:4-26 (Cholesky branch); returns NaN if not positive definite. */
double or_logdet_chol(int d, const double* a);
/* utils.cpp:94-102 */
double or_log_multivariate_gamma(double x, int d);
/* priors/niw.cpp:122-138 */
double or_niw_lml(int d, double k0, double v0, const double* psi0, double kp, double vp,
                  const double* psip, int64_t count);
/* priors/multinomial_prior.cpp:12-22 and :56-67 */
void or_mult_posterior(int d, const double* alpha, const double* sum, int64_t count, double* alpha_out);
double or_mult_lml(int d, const double* alpha0, const double* alphap);
/* local_clusters_actions.cpp:230-233 */
double or_split_log_hr(double alpha, int64_t n, int64_t nl, int64_t nr, double lml, double lml_l,
                       double lml_r);
/* shared_actions.cpp:97-99 */
double or_merge_log_hr(double alpha, int64_t ni, int64_t nj, double lml_i, double lml_j,
                       double lml_ij);

#ifdef __cplusplus
}
#endif
#endif

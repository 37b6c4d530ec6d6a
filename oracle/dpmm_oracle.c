/*
 * dpmm_oracle.c -- FP64 CPU restatement of the reference's per-iteration path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, never part of the product.
 * Every routine cites the reference file:line it restates (paths relative to the
 * reference's DPMMSubClusters/ directory).  The restatement keeps the reference's
 * arithmetic order where it matters for parity (the D*D constant, the Walker alias
 * construction, strict/non-strict comparisons, first-max argmax).
 */
#include "dpmm_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define OR_PI 3.14159265358979323846

static double fmin2(double a, double b) { return a < b ? a : b; }

void or_gauss_loglik(int64_t n, int d, const double* x, const double* mu,
                     const double* inv_sigma, double logdet_sigma, double weight,
                     int add_log_weight, double* r)
{
    /* scalar = -((sigma.size() * log(2*pi) + logdetSigma) / 2), sigma.size() == D*D
     * (cudaKernel_gaussian.cu:75 and :108). */
    const double scalar = -(((double)d * (double)d * log(2 * OR_PI) + logdet_sigma) / 2);
    double* z = (double*)malloc(sizeof(double) * (size_t)d);
    for (int64_t p = 0; p < n; ++p) {
        const double* xp = x + (size_t)p * d;
        for (int j = 0; j < d; ++j) z[j] = xp[j] - mu[j];       /* divide_points_by_mu_all_kernel */
        double sum = 0;
        for (int i = 0; i < d; ++i) {                            /* c = invSigma * z (column-major) */
            double c = 0;
            for (int j = 0; j < d; ++j) c += inv_sigma[(size_t)j * d + i] * z[j];
            sum += z[i] * c;                                     /* dcolwise dot */
        }
        r[p] = add_log_weight ? scalar - sum / 2 + log(weight) : scalar - sum / 2;
    }
    free(z);
}

void or_mult_loglik(int64_t n, int d, const double* x, const double* log_theta, double* r)
{
    for (int64_t p = 0; p < n; ++p) {
        double sum = 0;
        for (int i = 0; i < d; ++i) sum += log_theta[i] * x[(size_t)p * d + i];
        r[p] = sum;
    }
}

void or_softmax_rows(int64_t n, int k, double* r)
{
    for (int64_t p = 0; p < n; ++p) {
        double mx = 0;
        int first = 1;
        for (int j = 0; j < k; ++j) {
            double v = r[(size_t)j * n + p];
            if (first || v > mx) { first = 0; mx = v; }
        }
        double sum = 0;
        for (int j = 0; j < k; ++j) {
            double e = exp(r[(size_t)j * n + p] - mx);
            r[(size_t)j * n + p] = e;
            sum += e;
        }
        for (int j = 0; j < k; ++j) r[(size_t)j * n + p] = r[(size_t)j * n + p] / sum;
    }
}

int or_alias_draw(int k, const double* prob, double u1, double u2, double* margin,
                  double* y, int* iwork)
{
    int* a = iwork;
    int* b = iwork + (k + 2);
    const int nn = k;
    double mg = INFINITY;
    int i, j, t;
    for (i = 0; i <= nn + 1; ++i) { a[i] = i; b[i] = i; }
    y[0] = 0.0;
    for (i = 1; i <= nn; ++i) y[i] = prob[i - 1] * nn;
    y[nn + 1] = 2.0;

    /* partition: small (y < 1) to the left, large to the right (cudaKernel.cu:56-79) */
    i = 0;
    j = nn + 1;
    for (;;) {
        do { i++; mg = fmin2(mg, fabs(y[b[i]] - 1.0)); } while (y[b[i]] < 1.0);
        do { j--; mg = fmin2(mg, fabs(y[b[j]] - 1.0)); } while (1.0 <= y[b[j]]);
        if (j <= i) break;
        t = b[i]; b[i] = b[j]; b[j] = t;
    }
    /* pairing (cudaKernel.cu:81-111) */
    i = j;
    j++;
    while (0 < i) {
        while (mg = fmin2(mg, fabs(y[b[j]] - 1.0)), y[b[j]] <= 1.0) j++;
        if (nn < j) break;
        y[b[j]] = y[b[j]] - (1.0 - y[b[i]]);
        a[b[i]] = b[j];
        mg = fmin2(mg, fabs(y[b[j]] - 1.0));
        if (y[b[j]] < 1.0) {
            t = b[i]; b[i] = b[j]; b[j] = t;
            j++;
        } else {
            i--;
        }
    }
    /* draw (cudaKernel.cu:113-123) */
    int col = (int)(u1 * (nn - 1 + 0.999999) + 1);
    int label = col;
    mg = fmin2(mg, fabs(y[col] - u2));
    if (y[col] < u2) label = a[col];
    if (margin) *margin = mg;
    return label;
}

void or_sample_labels(int64_t n, int k, double* r, const double* u, int final_,
                      int32_t* labels, double* margin)
{
    if (final_) {
        /* update_labels_by_max_index_kernel (cudaKernel.cu:405-424) on the raw log-likelihoods */
        for (int64_t p = 0; p < n; ++p) {
            double mx = 0;
            int first = 1, arg = 0;
            for (int j = 0; j < k; ++j) {
                double v = r[(size_t)j * n + p];
                if (first || mx < v) { first = 0; mx = v; arg = j; }
            }
            labels[p] = arg + 1;
            if (margin) {
                double gap = INFINITY;
                for (int j = 0; j < k; ++j)
                    if (j != arg) gap = fmin2(gap, fabs(mx - r[(size_t)j * n + p]));
                margin[p] = gap;
            }
        }
        return;
    }
    or_softmax_rows(n, k, r);
    double* y = (double*)malloc(sizeof(double) * (size_t)(k + 2));
    int* iw = (int*)malloc(sizeof(int) * 2 * (size_t)(k + 2));
    double* pr = (double*)malloc(sizeof(double) * (size_t)k);
    for (int64_t p = 0; p < n; ++p) {
        for (int j = 0; j < k; ++j) pr[j] = r[(size_t)j * n + p];
        double mg;
        labels[p] = or_alias_draw(k, pr, u[2 * p], u[2 * p + 1], &mg, y, iw);
        if (margin) margin[p] = mg;
    }
    free(y); free(iw); free(pr);
}

void or_sample_sub_from_loglik(int64_t m, double* r, const double* lr_weights, const double* u,
                               int32_t* sub_labels, double* margin)
{
    double y[4];
    int iw[8];
    for (int64_t p = 0; p < m; ++p) {
        double a = r[p] + log(lr_weights[0]);
        double b = r[p + m] + log(lr_weights[1]);
        double mx = fmax(a, b);
        a = exp(a - mx);
        b = exp(b - mx);
        double s = a + b;
        double pr[2] = {a / s, b / s};
        double mg;
        sub_labels[p] = or_alias_draw(2, pr, u[2 * p], u[2 * p + 1], &mg, y, iw);
        if (margin) margin[p] = mg;
    }
}

/* Shared driver for the sub-label phase: the reference compacts each cluster's points
 * (find_indices, cudaKernel.cu:189-200), computes the two sub-cluster log-likelihoods,
 * adds log lr_weights, normalises and draws with the point's own RNG state
 * (sample_log_cat_array_sub_cluster_all, cudaKernel.cu:135-142).  The draw is per point,
 * so iterating points in index order gives the same labels as the compacted order. */
static void sub_labels_common(int64_t n, int d, const double* x, const int32_t* labels, int k,
                              int gauss, const double* mu_lr, const double* inv_sigma_lr,
                              const double* logdet_lr, const double* log_theta_lr,
                              const double* lr_weights, const double* u, int32_t* sub_labels,
                              double* margin, double* r_out)
{
    for (int64_t p = 0; p < n; ++p) {
        int c = labels[p] - 1;
        if (c < 0 || c >= k) continue;
        double r2[2];
        for (int s = 0; s < 2; ++s) {
            if (gauss)
                or_gauss_loglik(1, d, x + (size_t)p * d, mu_lr + (size_t)(2 * c + s) * d,
                                inv_sigma_lr + (size_t)(2 * c + s) * d * d, logdet_lr[2 * c + s],
                                1.0, 0, &r2[s]);
            else
                or_mult_loglik(1, d, x + (size_t)p * d, log_theta_lr + (size_t)(2 * c + s) * d, &r2[s]);
        }
        if (r_out) { r_out[2 * p] = r2[0]; r_out[2 * p + 1] = r2[1]; }
        double mg;
        or_sample_sub_from_loglik(1, r2, lr_weights + 2 * c, u + 2 * p, sub_labels + p, &mg);
        if (margin) margin[p] = mg;
    }
}

void or_gauss_sub_labels(int64_t n, int d, const double* x, const int32_t* labels, int k,
                         const double* mu_lr, const double* inv_sigma_lr, const double* logdet_lr,
                         const double* lr_weights, const double* u, int32_t* sub_labels,
                         double* margin, double* r_out)
{
    sub_labels_common(n, d, x, labels, k, 1, mu_lr, inv_sigma_lr, logdet_lr, NULL, lr_weights, u,
                      sub_labels, margin, r_out);
}

void or_mult_sub_labels(int64_t n, int d, const double* x, const int32_t* labels, int k,
                        const double* log_theta_lr, const double* lr_weights, const double* u,
                        int32_t* sub_labels, double* margin, double* r_out)
{
    sub_labels_common(n, d, x, labels, k, 0, NULL, NULL, NULL, log_theta_lr, lr_weights, u,
                      sub_labels, margin, r_out);
}

void or_suff_stats(int64_t n, int d, const double* x, const int32_t* labels,
                   const int32_t* sub_labels, int k, int64_t* count, double* sum, double* S)
{
    memset(count, 0, sizeof(int64_t) * 3 * (size_t)k);
    memset(sum, 0, sizeof(double) * 3 * (size_t)k * d);
    if (S) memset(S, 0, sizeof(double) * 3 * (size_t)k * d * d);
    for (int64_t p = 0; p < n; ++p) {
        int c = labels[p] - 1;
        if (c < 0 || c >= k) continue;
        int s = sub_labels[p];
        /* create_suff_stats_dict_worker_all (cudaKernel.cu:281-318) only gathers points whose
         * sub-label is 1 or 2; the cluster set is their union. */
        if (s != 1 && s != 2) continue;
        const double* xp = x + (size_t)p * d;
        int slots[2] = {3 * c, 3 * c + s};
        for (int q = 0; q < 2; ++q) {
            int sl = slots[q];
            count[sl] += 1;
            for (int i = 0; i < d; ++i) sum[(size_t)sl * d + i] += xp[i];
            if (S)
                for (int j = 0; j < d; ++j)
                    for (int i = 0; i < d; ++i)
                        S[(size_t)sl * d * d + (size_t)j * d + i] += xp[i] * xp[j];
        }
    }
}

void or_sample_labels_init(int64_t n, const double* u, int initial_clusters, double outlier_mod,
                           int32_t* labels)
{
    for (int64_t p = 0; p < n; ++p)
        labels[p] = (int)(u[p] * (initial_clusters - 1 + 0.999999) + 1 + ((outlier_mod > 0) ? 1 : 0));
}

void or_sample_sub_labels_init(int64_t n, const double* u, int32_t* sub_labels)
{
    for (int64_t p = 0; p < n; ++p) sub_labels[p] = (int)(u[p] * (2 - 1 + 0.999999) + 1);
}

void or_split_cluster(int64_t n, int32_t* labels, int32_t* sub_labels, int index, int new_index,
                      const uint32_t* bits)
{
    for (int64_t p = 0; p < n; ++p) {
        if (labels[p] == index + 1) {
            if (sub_labels[p] == 2) labels[p] = new_index + 1;
            sub_labels[p] = (int)(bits[p] % 2 + 1);
        }
    }
}

void or_merge_clusters(int64_t n, int32_t* labels, int32_t* sub_labels, int index, int new_index)
{
    for (int64_t p = 0; p < n; ++p) {
        if (labels[p] == index + 1) sub_labels[p] = 1;
        if (labels[p] == new_index + 1) sub_labels[p] = 2;
        if (labels[p] == new_index + 1) labels[p] = index + 1;
    }
}

void or_reset_bad_cluster(int64_t n, const int32_t* labels, int32_t* sub_labels, int index,
                          const uint32_t* bits)
{
    for (int64_t p = 0; p < n; ++p)
        if (labels[p] == index + 1) sub_labels[p] = (int)(bits[p] % 2 + 1);
}

void or_remove_empty_cluster(int64_t n, int32_t* labels, int limit)
{
    for (int64_t p = 0; p < n; ++p)
        if (labels[p] > limit) labels[p] -= 1;
}

void or_sub_labels_count(int64_t n, const int32_t* sub_labels, int* l, int* r)
{
    int a = 0, b = 0;
    for (int64_t p = 0; p < n; ++p) {
        if (sub_labels[p] == 1) a++;
        else if (sub_labels[p] == 2) b++;
    }
    *l = a;
    *r = b;
}

void or_niw_posterior(int d, double k, const double* m, double v, const double* psi,
                      int64_t count, const double* sum, const double* S,
                      double* k_out, double* m_out, double* v_out, double* psi_out)
{
    if (count == 0) {          /* niw.cpp:27-30 returns a clone of the prior */
        *k_out = k;
        *v_out = v;
        memcpy(m_out, m, sizeof(double) * (size_t)d);
        memcpy(psi_out, psi, sizeof(double) * (size_t)d * d);
        return;
    }
    double kp = k + (double)count;
    double vp = v + (double)count;
    for (int i = 0; i < d; ++i) m_out[i] = (m[i] * k + sum[i]) / kp;
    /* psi' = (v psi + k m m^T - k' m' m'^T + S) / v', then symmetrised (niw.cpp:39-46) */
    double* t = (double*)malloc(sizeof(double) * (size_t)d * d);
    for (int j = 0; j < d; ++j)
        for (int i = 0; i < d; ++i) {
            size_t ij = (size_t)j * d + i;
            double tm = v * psi[ij] + k * m[i] * m[j];
            t[ij] = (tm - kp * m_out[i] * m_out[j] + S[ij]) / vp;
        }
    /* selfadjointView<Upper>: take the upper triangle, mirror it; then (A + A^T)/2 */
    for (int j = 0; j < d; ++j)
        for (int i = 0; i < d; ++i) {
            double up = (i <= j) ? t[(size_t)j * d + i] : t[(size_t)i * d + j];
            psi_out[(size_t)j * d + i] = up;
        }
    for (int j = 0; j < d; ++j)
        for (int i = 0; i < j; ++i) {
            size_t a = (size_t)j * d + i, b = (size_t)i * d + j;
            double s = (psi_out[a] + psi_out[b]) / 2;
            psi_out[a] = s;
            psi_out[b] = s;
        }
    free(t);
    *k_out = kp;
    *v_out = vp;
}

double or_logdet_chol(int d, const double* a)
{
    double* l = (double*)malloc(sizeof(double) * (size_t)d * d);
    memcpy(l, a, sizeof(double) * (size_t)d * d);
    double ld = 0;
    for (int j = 0; j < d; ++j) {
        double s = l[(size_t)j * d + j];
        for (int q = 0; q < j; ++q) s -= l[(size_t)q * d + j] * l[(size_t)q * d + j];
        if (!(s > 0)) { free(l); return NAN; }
        double djj = sqrt(s);
        l[(size_t)j * d + j] = djj;
        ld += log(djj);
        for (int i = j + 1; i < d; ++i) {
            double t = l[(size_t)j * d + i];
            for (int q = 0; q < j; ++q) t -= l[(size_t)q * d + i] * l[(size_t)q * d + j];
            l[(size_t)j * d + i] = t / djj;
        }
    }
    free(l);
    return 2 * ld;
}

double or_log_multivariate_gamma(double x, int d)
{
    double res = d * (d - 1) / 4.0 * log(OR_PI);
    for (long q = 1; q <= d; ++q) res += lgamma(x + (1 - q) / 2.0);
    return res;
}

double or_niw_lml(int d, double k0, double v0, const double* psi0, double kp, double vp,
                  const double* psip, int64_t count)
{
    double logpi = log(OR_PI);
    double ld0 = or_logdet_chol(d, psi0);
    double ldp = or_logdet_chol(d, psip);
    return -(double)count * d * 0.5 * logpi + or_log_multivariate_gamma(vp / 2.0, d) -
           or_log_multivariate_gamma(v0 / 2.0, d) + (v0 / 2.0) * (d * log(v0) + ld0) -
           (vp / 2.0) * (d * log(vp) + ldp) + (d / 2.0) * (log(k0 / kp));
}

void or_mult_posterior(int d, const double* alpha, const double* sum, int64_t count, double* alpha_out)
{
    for (int i = 0; i < d; ++i) alpha_out[i] = count == 0 ? alpha[i] : alpha[i] + sum[i];
}

double or_mult_lml(int d, const double* alpha0, const double* alphap)
{
    double s0 = 0, sp = 0;
    for (int i = 0; i < d; ++i) { s0 += alpha0[i]; sp += alphap[i]; }
    double val = lgamma(s0) - lgamma(sp);
    for (int i = 0; i < d; ++i) val += lgamma(alphap[i]) - lgamma(alpha0[i]);
    return val;
}

double or_split_log_hr(double alpha, int64_t n, int64_t nl, int64_t nr, double lml, double lml_l,
                       double lml_r)
{
    return log(alpha) + lgamma((double)nl) + lml_l + lgamma((double)nr) + lml_r -
           (lgamma((double)n) + lml);
}

double or_merge_log_hr(double alpha, int64_t ni, int64_t nj, double lml_i, double lml_j,
                       double lml_ij)
{
    double n = (double)(ni + nj);
    return -log(alpha) + lgamma(alpha) - 2 * lgamma(0.5 * alpha) + lgamma(n) - lgamma(n + alpha) +
           lgamma((double)ni + 0.5 * alpha) - lgamma((double)ni) - lgamma((double)nj) +
           lgamma((double)nj + 0.5 * alpha) + lml_ij - lml_i - lml_j;
}

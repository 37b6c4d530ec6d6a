// linalg.h -- small dense FP64 helpers for the host side (D <= a few hundred): Cholesky,
// triangular solves and inverses, log-determinants.  Column-major storage, as Eigen's default
// (the reference's MatrixXd), so matrices cross the C ABI unchanged.
#pragma once

#include <cmath>
#include <vector>

namespace dpmm {
namespace la {

inline double& at(std::vector<double>& a, int n, int i, int j) { return a[(size_t)j * n + i]; }
inline double at(const std::vector<double>& a, int n, int i, int j) { return a[(size_t)j * n + i]; }

// Lower Cholesky factor L (A = L L^T) of a symmetric matrix, reading A's lower triangle.
// Returns false if A is not positive definite.  Left-looking by columns: column j of L is A's
// column j minus L(j, q) times column q of L for q < j, each a contiguous AXPY (the terms are
// subtracted in the same order, q ascending, as in the dot-product form).
inline bool cholesky(const double* A, int n, std::vector<double>& L)
{
    L.assign((size_t)n * n, 0.0);
    for (int j = 0; j < n; ++j) {
        double* cj = &L[(size_t)j * n];
        for (int i = j; i < n; ++i) cj[i] = A[(size_t)j * n + i];
        for (int q = 0; q < j; ++q) {
            const double* cq = &L[(size_t)q * n];
            const double f = cq[j];
            for (int i = j; i < n; ++i) cj[i] -= f * cq[i];
        }
        const double s = cj[j];
        if (!(s > 0) || !std::isfinite(s)) return false;
        const double d = std::sqrt(s);
        cj[j] = d;
        for (int i = j + 1; i < n; ++i) cj[i] /= d;
    }
    return true;
}

inline double logdet_from_chol(const std::vector<double>& L, int n)
{
    double s = 0;
    for (int j = 0; j < n; ++j) s += std::log(L[(size_t)j * n + j]);
    return 2 * s;
}

// Inverse of a lower-triangular matrix (result lower-triangular).
inline void tri_lower_inverse(const std::vector<double>& L, int n, std::vector<double>& Li)
{
    Li.assign((size_t)n * n, 0.0);
    for (int j = 0; j < n; ++j) {
        Li[(size_t)j * n + j] = 1.0 / L[(size_t)j * n + j];
        for (int i = j + 1; i < n; ++i) {
            double s = 0;
            for (int q = j; q < i; ++q) s += L[(size_t)q * n + i] * Li[(size_t)j * n + q];
            Li[(size_t)j * n + i] = -s / L[(size_t)i * n + i];
        }
    }
}

// C = A * B (n x n lower-triangular A and B; C lower-triangular)
inline void tri_lower_mul(const std::vector<double>& A, const std::vector<double>& B, int n, std::vector<double>& C)
{
    C.assign((size_t)n * n, 0.0);
    for (int j = 0; j < n; ++j)
        for (int i = j; i < n; ++i) {
            double s = 0;
            for (int q = j; q <= i; ++q) s += A[(size_t)q * n + i] * B[(size_t)j * n + q];
            C[(size_t)j * n + i] = s;
        }
}

// Inverse of a symmetric positive-definite matrix through its Cholesky factor.
inline bool spd_inverse(const double* A, int n, std::vector<double>& Ainv)
{
    std::vector<double> L, Li;
    if (!cholesky(A, n, L)) return false;
    tri_lower_inverse(L, n, Li);
    Ainv.assign((size_t)n * n, 0.0);
    // A^-1 = Li^T Li
    for (int j = 0; j < n; ++j)
        for (int i = j; i < n; ++i) {
            double s = 0;
            for (int q = i; q < n; ++q) s += Li[(size_t)i * n + q] * Li[(size_t)j * n + q];
            Ainv[(size_t)j * n + i] = s;
            Ainv[(size_t)i * n + j] = s;
        }
    return true;
}

}  // namespace la
}  // namespace dpmm

"""The reference back-end's FP64 matrix helpers (csrc/dpmm_linalg.cu): cudaKernel::inverse_matrix
(cudaKernel.cu:1558-1598) and cudaKernel::multiplie_matrix_for_inverseWishart (cudaKernel.cu:980-1016),
which niw::sample_distribution (priors/niw.cpp:61-107) calls, against numpy FP64.

Criteria: A^-1 A = I within 1e-9 n (well-conditioned inputs, among them the NIW draw's nu psi' and
matrices that need row exchanges, which the reference's Gauss-Jordan without pivoting cannot invert);
a singular matrix reports DPMM_ERR_NUMERIC; (A B)(A B)^T within 1e-12 relative of numpy and exactly
symmetric."""
import numpy as np
import pytest

from dpmmsubclusters_gpu_b200 import CudaKernel, DpmmError, prior_type

pytestmark = pytest.mark.gpu

DPMM_ERR_NUMERIC = 6


@pytest.fixture(scope="module")
def ck():
    rng = np.random.default_rng(0)
    k = CudaKernel(prior_type.Gaussian, k_max=4).init(1000, rng.normal(size=(1000, 8)), 1, points_major=True)
    yield k
    k.release()


@pytest.mark.parametrize("n", [1, 2, 3, 7, 31, 64, 100, 257])
def test_inverse_matches_numpy(ck, n):
    rng = np.random.default_rng(n)
    G = rng.normal(size=(n, n))
    spd = G @ G.T / n + 0.5 * np.eye(n)                       # the NIW use: nu psi'
    general = rng.normal(size=(n, n)) + 3.0 * np.eye(n)
    for A in (spd, 70.0 * spd, general):
        B = ck.inverse_matrix(A)
        np.testing.assert_allclose(B @ A, np.eye(n), atol=1e-9 * n)
        np.testing.assert_allclose(B, np.linalg.inv(A), rtol=1e-8, atol=1e-10 * np.abs(B).max())


def test_inverse_needs_row_exchanges(ck):
    # zero diagonal: Gauss-Jordan without pivoting divides by zero here
    A = np.array([[0.0, 2.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 4.0]])
    np.testing.assert_allclose(ck.inverse_matrix(A), np.linalg.inv(A), atol=1e-15)
    P = np.eye(6)[[3, 0, 5, 1, 4, 2]] * np.arange(1, 7)
    np.testing.assert_allclose(ck.inverse_matrix(P) @ P, np.eye(6), atol=1e-14)


def test_singular_matrix_reported(ck):
    A = np.ones((5, 5))
    with pytest.raises(DpmmError) as e:
        ck.inverse_matrix(A)
    assert e.value.status == DPMM_ERR_NUMERIC
    A = np.diag([1.0, 2.0, 0.0, 3.0])
    with pytest.raises(DpmmError) as e:
        ck.inverse_matrix(A)
    assert e.value.status == DPMM_ERR_NUMERIC
    np.testing.assert_allclose(ck.inverse_matrix(np.diag([1.0, 2.0])), np.diag([1.0, 0.5]))   # still usable


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (8, 8, 8), (64, 64, 64), (5, 9, 3), (100, 40, 70)])
def test_wishart_product_matches_numpy(ck, m, n, k):
    rng = np.random.default_rng(m * 1000 + n * 10 + k)
    A = np.tril(rng.normal(size=(m, n)))
    B = rng.normal(size=(n, k))
    C = ck.multiplie_matrix_for_inverseWishart(A, B)
    T = A @ B
    ref = T @ T.T
    np.testing.assert_allclose(C, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    np.testing.assert_array_equal(C, C.T)

"""The bounds behind the pruned label phase (csrc/dpmm_kernels.cu k_prune_prep / k_prune_scan*),
restated in numpy and checked as lower bounds of the exact whitened distance |W_k^T (x - mu_k)| on
random clusters and points:
  chunk bound  M_hk - lam_k R  with M_hk = |W_k^T (mu_h - mu_k)| (deflated by 1e-5), lam_k^2 the
               Gershgorin bound of W_k W_k^T (inflated by 1e-5) and R >= |x - mu_h|;
  point bound  |v_hk^T x - beta_hk|  with v_hk = W_k u, u = W_k^T (mu_h - mu_k) / M_hk,
               beta_hk = v_hk^T mu_k.
A cluster left out by either bound has r_k(x) = c_k - |W_k^T (x - mu_k)|^2 / 2 below the bound's
c_k - bound^2 / 2, which the kernels compare against r_h(x) - margin."""
import numpy as np
import pytest


def prep(W, mu):
    K, D, _ = W.shape
    lam = np.empty(K)
    M = np.empty((K, K))
    V = np.zeros((K, K, D))
    beta = np.zeros((K, K))
    for k in range(K):
        G = W[k] @ W[k].T
        lam[k] = np.sqrt(np.abs(G).sum(1).max()) * (1 + 1e-5)
        for h in range(K):
            z = W[k].T @ (mu[h] - mu[k])
            nz = np.linalg.norm(z)
            M[h, k] = nz * (1 - 1e-5)
            if nz > 0:
                V[h, k] = W[k] @ (z / nz)
            beta[h, k] = V[h, k] @ mu[k]
    return lam, M, V, beta


@pytest.mark.parametrize("D,K,seed", [(4, 6, 0), (16, 8, 1), (64, 5, 2)])
def test_bounds_are_lower_bounds(D, K, seed):
    rng = np.random.default_rng(seed)
    mu = rng.normal(size=(K, D)) * 5
    W = np.stack([np.linalg.cholesky(np.linalg.inv(A @ A.T / D + 0.5 * np.eye(D)))
                  for A in rng.normal(size=(K, D, D))])
    lam, M, V, beta = prep(W, mu)
    for h in range(K):
        x = mu[h] + rng.normal(size=(2000, D)) * rng.uniform(0.2, 3.0)
        R = np.linalg.norm(x - mu[h], axis=1).max()
        for k in range(K):
            exact = np.linalg.norm((x - mu[k]) @ W[k], axis=1)
            chunk = M[h, k] - lam[k] * R
            assert np.all(exact >= chunk - 1e-9 * (1 + abs(chunk))), (h, k)
            if h != k:
                point = np.abs(x @ V[h, k] - beta[h, k])
                assert np.all(exact >= point * (1 - 1e-12) - 1e-9), (h, k)


def test_left_out_cluster_is_below_the_margin():
    # a cluster excluded by the point bound at margin m has r_k < r_h - m at that point
    rng = np.random.default_rng(7)
    D, K, margin = 8, 4, 30.0
    mu = rng.normal(size=(K, D)) * 8
    W = np.stack([np.eye(D) * rng.uniform(0.8, 1.5) for _ in range(K)])
    c = rng.normal(size=K)
    _, _, V, beta = prep(W, mu)
    x = mu[0] + rng.normal(size=(5000, D))
    r = np.stack([c[k] - 0.5 * np.sum(((x - mu[k]) @ W[k]) ** 2, 1) for k in range(K)], 1)
    for k in range(1, K):
        ub = c[k] - 0.5 * (x @ V[0, k] - beta[0, k]) ** 2
        out = ub < r[:, 0] - margin
        assert np.all(r[out, k] < r[out, 0] - margin)

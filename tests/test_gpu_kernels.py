"""GPU parity of every kernel of the path against the FP64 oracle and the reference's goldens,
called through the C ABI (dpmmsubclusters_gpu_b200.CudaKernel wraps include/dpmm_capi.h).

Tolerances (stated per check; tests/parity.py gives the criteria):
  * Gaussian log-likelihoods of the FP32 / tensor-core contraction, without the reference's
    -D^2 log(2 pi)/2 constant: |r - r64| <= 1e-4 |log N(x; mu, Sigma)| and
    |r - r64| <= 1e-4 max((x - mu)^T Sigma^-1 (x - mu) / 2, 1) (relative to the data term);
  * labels / sub-labels: bit-exact against the oracle's alias draw on FP64 log-likelihoods with the
    same uniforms, except points whose FP64 decision margin is below what the row's log-likelihood
    error can move (4 K (row error + 1e-6)); the count is recorded.  Also bit-exact against the
    oracle's draw on the GPU's own log-likelihoods except at margins below 1e-4 (the draw itself);
  * sufficient statistics: counts exact; sums and scatter within 1e-6 relative;
  * Hastings ratios: within 1e-6 * max(1, |value|) + 1e-6 * |lml| scale (FP64 both sides).
"""
import math

import numpy as np
import pytest

import parity as P
from conftest import eigen, inits, uniforms
from dpmmsubclusters_gpu_b200 import RNG_CURAND_XORWOW, RNG_PHILOX, CudaKernel, LL_FP32, prior_type
from oracle import oracle as O

pytestmark = pytest.mark.gpu

LOG2PI = math.log(2 * math.pi)


def _gauss_mixture(rng, N, D, K, spread=4.0):
    mus = rng.normal(size=(K, D)) * spread
    covs = []
    for _ in range(K):
        A = rng.normal(size=(D, D))
        covs.append(A @ A.T / D + 0.5 * np.eye(D))
    z = rng.integers(0, K, size=N)
    x = np.empty((N, D))
    for k in range(K):
        idx = np.where(z == k)[0]
        x[idx] = rng.multivariate_normal(mus[k], covs[k], size=idx.size)
    return x, z, mus, np.array(covs)


def _params(rng, mus, covs, jitter=0.3):
    K, D = mus.shape
    mu = mus + jitter * rng.normal(size=mus.shape)
    inv = np.array([np.linalg.inv(c) for c in covs])
    logdet = np.array([np.linalg.slogdet(c)[1] for c in covs])
    w = rng.dirichlet(np.ones(K) * 2)
    return mu, inv, logdet, w


def _mismatch_ok(lab_gpu, lab_or, margin, tol=1e-4, frac=1e-3):
    bad = lab_gpu != lab_or
    assert np.all(margin[bad] < tol), (bad.sum(), margin[bad][:10])
    assert bad.mean() <= frac, bad.mean()
    return int(bad.sum())


# ------------------------------------------------------------------ goldens
@pytest.mark.parametrize("name,weight", [("log_likelihood", 0.5), ("log_likelihood_ignore_weight", 1.0)])
def test_loglik_goldens_seam_and_kernel(goldens, name, weight):
    # test/cudaKernel_gaussian_test.cpp:748-829 through the FP64 seam and the product kernel
    t = goldens["cudaKernel_gaussian_test::" + name]
    I = inits(t)
    x = eigen(I["x"][0], 2, 10)                        # D x N
    mu, inv = I["mu"][0], eigen(I["invSigma"][0], 2, 2)
    ld = t["scalars"]["logdetSigma"]
    exp = np.array([e["value"] for e in t["expect"] if e["kind"] == "near"])
    ck = CudaKernel(prior_type.Gaussian).init(10, x, 12345)
    r = ck.log_likelihood_labels(weight, mu, inv, ld)
    np.testing.assert_allclose(r, exp, atol=1e-4)
    ck.set_gaussian_params(mu[None], inv[None], [ld], [weight])
    r2 = ck.create_clusters_labels(1, uniforms=uniforms(20, 1), return_loglik=True)[:, 0]
    np.testing.assert_allclose(r2 - 4 * LOG2PI / 2, exp, atol=1e-4)
    assert np.all(ck.get_labels() == 1)


def test_multinomial_loglik_golden(goldens):
    t = goldens["cudaKernel_multinomial_test::log_likelihood_labels"]
    x = eigen(inits(t)["x"][0], 2, 10)
    lt = np.array(t["alpha_push"])
    exp = np.array([e["value"] for e in t["expect"] if e["kind"] == "near"])
    ck = CudaKernel(prior_type.Multinomial).init(10, x)
    np.testing.assert_allclose(ck.log_likelihood_labels(1.0, None, log_theta=lt), exp, atol=1e-4)
    ck.set_multinomial_params(lt[None])
    r = ck.create_clusters_labels(1, uniforms=uniforms(20, 2), return_loglik=True)[:, 0]
    np.testing.assert_allclose(r, exp, atol=1e-4)


@pytest.mark.parametrize("a,b,one,two", [(0.4, 0.6, 45260, 54740), (0.6, 0.4, 55257, 44743)])
def test_alias_golden_counts_curand(a, b, one, two):
    # test/cudaKernel_gaussian_test.cpp:18-123: softmax + alias with the reference's XORWOW stream,
    # seed 0; FP64 seam and the fused FP32 label kernel both reproduce the counts
    n = 100000
    pts = np.zeros((2, n))
    ck = CudaKernel(prior_type.Gaussian, rng_kind=RNG_CURAND_XORWOW).init(n, pts, 0)
    ck.sample_log_cat_array(np.tile([a, b], (n, 1)))
    lab = ck.get_labels()
    assert (lab == 1).sum() == one and (lab == 2).sum() == two
    ck2 = CudaKernel(prior_type.Gaussian, rng_kind=RNG_CURAND_XORWOW).init(n, pts, 0)
    # zero precision factors: r_k = -logdet/2 + log w_k = a, b
    ck2.set_gaussian_params(np.zeros((2, 2)), np.zeros((2, 2, 2)), [0.0, 0.0], [math.exp(a), math.exp(b)],
                            factors=True)
    ck2.create_clusters_labels(2)
    lab2 = ck2.get_labels()
    assert (lab2 == 1).sum() == one and (lab2 == 2).sum() == two


def test_alias_golden_counts_sub_cluster_curand():
    # test/cudaKernel_gaussian_test.cpp:209-383
    n = 100000
    pts = np.zeros((2, n))
    ck = CudaKernel(prior_type.Gaussian, rng_kind=RNG_CURAND_XORWOW).init(n, pts, 0)
    ck.sample_log_cat_array_sub_cluster(np.tile([0.4, 0.6], (n, 1)), np.arange(n), [0.5, 0.5])
    s = ck.get_sub_labels()
    assert (s == 1).sum() == 45260 and (s == 2).sum() == 54740
    ck = CudaKernel(prior_type.Gaussian, rng_kind=RNG_CURAND_XORWOW).init(n, pts, 0)
    ck.sample_log_cat_array_sub_cluster(np.tile([0.1, 0.9], (n, 1)), np.arange(n), [0.5, 0.5])
    few = np.arange(0, n, 3)
    ck.sample_log_cat_array_sub_cluster(np.tile([0.1, 0.9], (few.size, 1)), few, [0.5, 0.5])
    s = ck.get_sub_labels()
    assert (s[few] == 1).sum() == 10279 and (s[few] == 2).sum() == 23055
    assert (s == 1).sum() == 31207 and (s == 2).sum() == 68793


# ------------------------------------------------------------------ label phase parity
@pytest.mark.parametrize("D,K,N", [(2, 1, 5000), (2, 3, 20000), (8, 9, 20000), (16, 20, 12000), (32, 20, 8000),
                                   (64, 37, 6000), (64, 100, 3000)])
def test_gaussian_labels_parity(D, K, N):
    rng = np.random.default_rng(D * 100 + K)
    x, z, mus, covs = _gauss_mixture(rng, N, D, K)
    mu, inv, logdet, w = _params(rng, mus, covs)
    ck = CudaKernel(prior_type.Gaussian, loglik_mode=LL_FP32).init(N, x, 7, points_major=True)
    ck.set_gaussian_params(mu, inv, logdet, w)
    u = uniforms(2 * N, D + K)
    r = ck.create_clusters_labels(K, uniforms=u, return_loglik=True).astype(np.float64)
    r64 = np.stack([O.gauss_loglik(x, mu[k], inv[k], logdet[k], w[k]) for k in range(K)], 1)
    row_err = P.gauss_ll(r, r64, D, logdet, np.log(w), "fp32", f"labels_fp32_D{D}_K{K}")
    lab = ck.get_labels()
    u2 = u.reshape(N, 2).astype(np.float64)
    lab_o, mg = O.sample_labels(r, u2)
    _mismatch_ok(lab, lab_o, mg)
    # against the FP64 log-likelihoods: differences only where the margin is inside the row's error
    P.labels_vs_fp64(lab, r64, u2, row_err, f"labels_fp32_D{D}_K{K}_vs_fp64")


@pytest.mark.parametrize("D,K", [(2, 4), (64, 25)])
def test_gaussian_labels_final_argmax(D, K):
    rng = np.random.default_rng(5 + D)
    N = 6000
    x, z, mus, covs = _gauss_mixture(rng, N, D, K)
    mu, inv, logdet, w = _params(rng, mus, covs)
    ck = CudaKernel(prior_type.Gaussian, loglik_mode=LL_FP32).init(N, x, 1, points_major=True)
    ck.set_gaussian_params(mu, inv, logdet, w)
    r = ck.create_clusters_labels(K, bFinal=True, return_loglik=True).astype(np.float64)
    lab = ck.get_labels()
    lab_o, gap = O.sample_labels(r, np.zeros((N, 2)), final=True)
    assert np.all((lab == lab_o) | (gap < 1e-5))
    r64 = np.stack([O.gauss_loglik(x, mu[k], inv[k], logdet[k], w[k]) for k in range(K)], 1)
    row_err = P.gauss_ll(r, r64, D, logdet, np.log(w), "fp32", f"argmax_fp32_D{D}_K{K}")
    P.labels_vs_fp64(lab, r64, np.zeros((N, 2)), row_err, f"argmax_fp32_D{D}_K{K}_vs_fp64", final=True)


@pytest.mark.parametrize("D,K,N", [(10, 3, 5000), (100, 12, 5000), (1000, 50, 2000)])
def test_multinomial_labels_parity(D, K, N):
    rng = np.random.default_rng(D + K)
    theta = rng.dirichlet(np.ones(D) * 0.3, size=K)
    z = rng.integers(0, K, size=N)
    x = np.stack([rng.multinomial(rng.poisson(60) + 1, theta[k]) for k in z]).astype(np.float64)
    lt = np.log(rng.dirichlet(np.ones(D), size=K) * 0.5 + theta * 0.5)
    ck = CudaKernel(prior_type.Multinomial).init(N, x, 3, points_major=True)
    ck.set_multinomial_params(lt)
    u = uniforms(2 * N, D)
    r = ck.create_clusters_labels(K, uniforms=u, return_loglik=True).astype(np.float64)
    r64 = np.stack([O.mult_loglik(x, lt[k]) for k in range(K)], 1)
    assert (np.abs(r - r64) / np.maximum(np.abs(r64), 32)).max() <= 2e-5
    lab_o, mg = O.sample_labels(r, u.reshape(N, 2).astype(np.float64))
    _mismatch_ok(ck.get_labels(), lab_o, mg)


# ------------------------------------------------------------------ sub-labels + statistics
def _gauss_sub_setup(rng, N, D, K):
    x, z, mus, covs = _gauss_mixture(rng, N, D, K)
    mu, inv, logdet, w = _params(rng, mus, covs)
    mu_lr = mu[:, None, :] + 0.7 * rng.normal(size=(K, 2, D))
    inv_lr = np.repeat(inv[:, None], 2, axis=1) * rng.uniform(0.8, 1.2, size=(K, 2, 1, 1))
    ld_lr = np.repeat(logdet[:, None], 2, axis=1) - D * np.log(rng.uniform(0.8, 1.2, size=(K, 2)) * 0 + 1)
    ld_lr = np.array([[-np.linalg.slogdet(inv_lr[k, s])[1] for s in range(2)] for k in range(K)])
    lrw = rng.dirichlet([2, 2], size=K)
    return x, z, mu, inv, logdet, w, mu_lr, inv_lr, ld_lr, lrw


@pytest.mark.parametrize("D,K,N", [(2, 2, 20000), (8, 5, 15000), (32, 7, 8000), (64, 12, 6000)])
def test_gaussian_sub_labels_and_stats_parity(D, K, N):
    rng = np.random.default_rng(31 * D + K)
    x, z, mu, inv, logdet, w, mu_lr, inv_lr, ld_lr, lrw = _gauss_sub_setup(rng, N, D, K)
    ck = CudaKernel(prior_type.Gaussian, loglik_mode=LL_FP32).init(N, x, 11, points_major=True)
    ck.set_gaussian_params(mu, inv, logdet, w, mu_lr, inv_lr, ld_lr, lrw)
    labels = (z + 1).astype(np.int32)
    ck.set_labels(labels)
    u = uniforms(2 * N, 77)
    r = ck.create_subclusters_labels(K, uniforms=u, return_loglik=True).astype(np.float64)
    sub = ck.get_sub_labels()
    # log-likelihoods vs FP64
    _, _, r64 = O.gauss_sub_labels(x, labels, mu_lr, inv_lr, ld_lr, lrw, u.astype(np.float64))
    ld_pt = ld_lr[labels - 1]
    row_err = P.gauss_ll(r, r64, D, ld_pt, 0.0, "fp32", f"sub_fp32_D{D}_K{K}")
    # draws vs the oracle on the GPU's own log-likelihoods
    u2 = u.reshape(N, 2).astype(np.float64)
    P.sub_labels_vs_fp64(sub, r64, labels, lrw, u2, row_err, f"sub_fp32_D{D}_K{K}_vs_fp64")
    sub_o = np.empty(N, np.int32)
    mg = np.empty(N)
    for k in range(K):
        idx = np.where(labels == k + 1)[0]
        s, m = O.sample_sub_from_loglik(r[idx], lrw[k], u2[idx])
        sub_o[idx], mg[idx] = s, m
    _mismatch_ok(sub, sub_o, mg)
    # statistics of the drawn sub-labels vs the oracle
    cnt, sm, S = ck.create_sufficient_statistics(np.arange(K))
    cnt_o, sm_o, S_o = O.suff_stats(x, labels, sub, K)
    np.testing.assert_array_equal(cnt, cnt_o)
    scale = np.abs(sm_o).max() + 1
    np.testing.assert_allclose(sm, sm_o, atol=1e-6 * scale * 10, rtol=1e-6)
    np.testing.assert_allclose(S, S_o, atol=1e-6 * (np.abs(S_o).max() + 1), rtol=1e-6)


@pytest.mark.parametrize("D,K,N", [(32, 5, 20000), (48, 7, 15000), (64, 6, 25000)])
def test_gaussian_sub_labels_tensor_core_parity(D, K, N):
    """Sub-labels on the tensor cores (split-BF16 contraction against each cluster's two
    sub-cluster factors, several 128-point tiles per chunk and several chunks per cluster):
    r against FP64 (parity.gauss_ll), draws exact against the oracle's draw on FP64 r up to the
    margin rule and on the GPU's own r except at margins below 1e-4, statistics of the drawn
    sub-labels exact / within 1e-6."""
    from dpmmsubclusters_gpu_b200 import LL_TC_BF16X3
    rng = np.random.default_rng(57 * D + K)
    x, z, mu, inv, logdet, w, mu_lr, inv_lr, ld_lr, lrw = _gauss_sub_setup(rng, N, D, K)
    x = x + 2.0
    mu = mu + 2.0
    mu_lr = mu_lr + 2.0
    ck = CudaKernel(prior_type.Gaussian, loglik_mode=LL_TC_BF16X3, k_max=64).init(N, x, 11, points_major=True)
    ck.set_gaussian_params(mu, inv, logdet, w, mu_lr, inv_lr, ld_lr, lrw)
    labels = (z + 1).astype(np.int32)
    ck.set_labels(labels)
    u = uniforms(2 * N, 91)
    r = ck.create_subclusters_labels(K, uniforms=u, return_loglik=True).astype(np.float64)
    sub = ck.get_sub_labels()
    _, _, r64 = O.gauss_sub_labels(x, labels, mu_lr, inv_lr, ld_lr, lrw, u.astype(np.float64))
    row_err = P.gauss_ll(r, r64, D, ld_lr[labels - 1], 0.0, "tc", f"sub_tc_D{D}_K{K}")
    u2 = u.reshape(N, 2).astype(np.float64)
    P.sub_labels_vs_fp64(sub, r64, labels, lrw, u2, row_err, f"sub_tc_D{D}_K{K}_vs_fp64")
    sub_o = np.empty(N, np.int32)
    mg = np.empty(N)
    for k in range(K):
        idx = np.where(labels == k + 1)[0]
        s, m = O.sample_sub_from_loglik(r[idx], lrw[k], u2[idx])
        sub_o[idx], mg[idx] = s, m
    _mismatch_ok(sub, sub_o, mg)
    cnt, sm, S = ck.create_sufficient_statistics(np.arange(K))
    cnt_o, sm_o, S_o = O.suff_stats(x, labels, sub, K)
    np.testing.assert_array_equal(cnt, cnt_o)
    np.testing.assert_allclose(sm, sm_o, atol=1e-6 * (np.abs(sm_o).max() + 1) * 10, rtol=1e-6)
    np.testing.assert_allclose(S, S_o, atol=1e-6 * (np.abs(S_o).max() + 1), rtol=1e-6)


@pytest.mark.parametrize("D,K,N", [(20, 3, 8000), (1000, 6, 3000)])
def test_multinomial_sub_labels_and_stats_parity(D, K, N):
    rng = np.random.default_rng(D)
    theta = rng.dirichlet(np.ones(D) * 0.3, size=K)
    z = rng.integers(0, K, size=N)
    x = np.stack([rng.multinomial(rng.poisson(80) + 1, theta[k]) for k in z]).astype(np.float64)
    lt = np.log(theta * 0.9 + 0.1 / D)
    lt_lr = np.log(rng.dirichlet(np.ones(D), size=(K, 2)) * 0.5 + theta[:, None] * 0.5)
    lrw = rng.dirichlet([3, 3], size=K)
    ck = CudaKernel(prior_type.Multinomial).init(N, x, 5, points_major=True)
    ck.set_multinomial_params(lt, None, lt_lr, lrw)
    labels = (z + 1).astype(np.int32)
    ck.set_labels(labels)
    u = uniforms(2 * N, 8)
    r = ck.create_subclusters_labels(K, uniforms=u, return_loglik=True).astype(np.float64)
    sub = ck.get_sub_labels()
    _, _, r64 = O.mult_sub_labels(x, labels, lt_lr, lrw, u.astype(np.float64))
    assert (np.abs(r - r64) / np.maximum(np.abs(r64), 32)).max() <= 2e-5
    u2 = u.reshape(N, 2).astype(np.float64)
    sub_o = np.empty(N, np.int32)
    mg = np.empty(N)
    for k in range(K):
        idx = np.where(labels == k + 1)[0]
        sub_o[idx], mg[idx] = O.sample_sub_from_loglik(r[idx], lrw[k], u2[idx])
    _mismatch_ok(sub, sub_o, mg)
    cnt, sm, S = ck.create_sufficient_statistics(np.arange(K))
    cnt_o, sm_o, _ = O.suff_stats(x, labels, sub, K, with_S=False)
    np.testing.assert_array_equal(cnt, cnt_o)
    np.testing.assert_array_equal(sm, sm_o)      # integer counts: exact


def test_stats_injected_labels_golden(goldens):
    # test/local_clusters_actions_test.cpp:281-315 and :15-172 statistics through the device
    t = goldens["local_clusters_actions_test::update_suff_stats_posterior"]
    I = inits(t)
    x = eigen(I["points"][0], 2, 10)
    ck = CudaKernel(prior_type.Gaussian).init(10, x)
    ck.set_labels(t["int_vectors"]["labels"])
    ck.set_sub_labels(t["int_vectors"]["sub_labels"])
    cnt, sm, S = ck.create_sufficient_statistics([0])
    cnt_o, sm_o, S_o = O.suff_stats(x.T, t["int_vectors"]["labels"], t["int_vectors"]["sub_labels"], 1)
    np.testing.assert_array_equal(cnt, cnt_o)
    np.testing.assert_allclose(sm, sm_o, atol=1e-5)
    np.testing.assert_allclose(S, S_o, atol=1e-4)
    assert abs(sm[0, 0, 0] - (-20.156998)) < 1e-4 and abs(S[0, 0, 0, 0] - 624.1152) < 1e-3


# ------------------------------------------------------------------ label maintenance
def test_relabel_parity():
    rng = np.random.default_rng(4)
    N, K = 50000, 9
    x = rng.normal(size=(N, 3))
    labels = rng.integers(1, K + 1, size=N).astype(np.int32)
    sub = rng.integers(1, 3, size=N).astype(np.int32)
    bits = rng.integers(0, 2 ** 32, size=N, dtype=np.uint64).astype(np.uint32)
    ck = CudaKernel(prior_type.Gaussian, k_max=32).init(N, x, 1, points_major=True)
    ck.set_labels(labels)
    ck.set_sub_labels(sub)
    # reset clusters 2 and 5, then split 1 -> 9 and 4 -> 10, merge (0, 3) and (6, 8), remove empties
    ck.reset_bad_clusters_worker([2, 5], bits)
    s_o = O.reset_bad_cluster(labels, sub, 2, bits)
    s_o = O.reset_bad_cluster(labels, s_o, 5, bits)
    np.testing.assert_array_equal(ck.get_sub_labels(), s_o)
    bits2 = bits[::-1].copy()
    ck.split_cluster_local_worker([1, 4], [9, 10], bits2)
    l_o, s_o = O.split_cluster(labels, s_o, 1, 9, bits2)
    l_o, s_o = O.split_cluster(l_o, s_o, 4, 10, bits2)
    np.testing.assert_array_equal(ck.get_labels(), l_o)
    np.testing.assert_array_equal(ck.get_sub_labels(), s_o)
    ck.merge_clusters_worker([0, 6], [3, 8])
    l_o, s_o = O.merge_clusters(l_o, s_o, 0, 3)
    l_o, s_o = O.merge_clusters(l_o, s_o, 6, 8)
    np.testing.assert_array_equal(ck.get_labels(), l_o)
    np.testing.assert_array_equal(ck.get_sub_labels(), s_o)
    limits = [4, 7]       # sequential remove_empty_clusters_worker calls
    ck.remove_empty_clusters_worker(limits)
    for lim in limits:
        l_o = O.remove_empty_cluster(l_o, lim)
    np.testing.assert_array_equal(ck.get_labels(), l_o)
    assert ck.get_sub_labels_count() == ((s_o == 1).sum(), (s_o == 2).sum())


def test_initial_labels_parity():
    N = 30000
    ck = CudaKernel(prior_type.Gaussian).init(N, np.zeros((2, N)))
    u = uniforms(N, 3)
    ck.sample_labels(5, 0.05, u)
    np.testing.assert_array_equal(ck.get_labels(), O.sample_labels_init(u.astype(np.float64), 5, 0.05))
    ck.sample_sub_labels(u)
    np.testing.assert_array_equal(ck.get_sub_labels(), O.sample_sub_labels_init(u.astype(np.float64)))


def test_philox_reproducible_and_uniform():
    N = 200000
    lab = []
    for _ in range(2):
        ck = CudaKernel(prior_type.Gaussian, rng_kind=RNG_PHILOX).init(N, np.zeros((2, N)), 99)
        ck.sample_labels(4, 0.0)
        lab.append(ck.get_labels())
    np.testing.assert_array_equal(lab[0], lab[1])
    freq = np.bincount(lab[0], minlength=5)[1:] / N
    assert np.abs(freq - 0.25).max() < 0.01


# ------------------------------------------------------------------ Hastings (one launch each)
@pytest.mark.parametrize("D,K", [(2, 6), (16, 9), (64, 5)])
def test_hastings_parity_niw(D, K):
    rng = np.random.default_rng(D * K)
    N = 4000 * K
    x, z, mus, covs = _gauss_mixture(rng, N, D, K, spread=3.0)
    x += 10.0     # away from the origin: exercises the shifted accumulation
    labels = (z + 1).astype(np.int32)
    sub = rng.integers(1, 3, size=N).astype(np.int32)
    ck = CudaKernel(prior_type.Gaussian, k_max=16).init(N, x, 1, points_major=True)
    ck.set_labels(labels)
    ck.set_sub_labels(sub)
    m0, psi0, k0, v0, alpha = np.zeros(D), np.eye(D), 1.0, D + 3.0, 10.0
    from dpmmsubclusters_gpu_b200 import niw_hyperparams
    ck.set_prior(niw_hyperparams(k0, m0, v0, psi0))
    ck.create_sufficient_statistics(np.arange(K))
    lml_g, hr_g = ck.split_hastings(K, alpha)
    mhr_g = ck.merge_hastings(K, alpha)
    cnt, sm, S = O.suff_stats(x, labels, sub, K)
    lml = np.empty((K, 3))
    for k in range(K):
        for s in range(3):
            kk, m, v, psi = O.niw_posterior(k0, m0, v0, psi0, cnt[k, s], sm[k, s], S[k, s])
            lml[k, s] = O.niw_lml(k0, v0, psi0, kk, v, psi, cnt[k, s])
    scale = np.abs(lml).max()
    assert np.abs(lml_g - lml).max() <= 1e-6 * scale, np.abs(lml_g - lml).max()
    hr = np.array([O.split_log_hr(alpha, *cnt[k], *lml[k]) for k in range(K)])
    assert np.abs(hr_g - hr).max() <= 1e-6 * scale
    for i in range(K):
        for j in range(i + 1, K):
            n2 = cnt[i, 0] + cnt[j, 0]
            kk, m, v, psi = O.niw_posterior(k0, m0, v0, psi0, n2, sm[i, 0] + sm[j, 0], S[i, 0] + S[j, 0])
            lij = O.niw_lml(k0, v0, psi0, kk, v, psi, n2)
            ref = O.merge_log_hr(alpha, cnt[i, 0], cnt[j, 0], lml[i, 0], lml[j, 0], lij)
            assert abs(mhr_g[i, j] - ref) <= 1e-6 * scale, (i, j, mhr_g[i, j], ref)
        assert np.all(np.isnan(mhr_g[i, : i + 1]))


def test_hastings_parity_multinomial():
    rng = np.random.default_rng(12)
    D, K, N = 50, 6, 6000
    theta = rng.dirichlet(np.ones(D) * 0.5, size=K)
    z = rng.integers(0, K, size=N)
    x = np.stack([rng.multinomial(40, theta[k]) for k in z]).astype(np.float64)
    labels = (z + 1).astype(np.int32)
    sub = rng.integers(1, 3, size=N).astype(np.int32)
    ck = CudaKernel(prior_type.Multinomial).init(N, x, 2, points_major=True)
    ck.set_labels(labels)
    ck.set_sub_labels(sub)
    from dpmmsubclusters_gpu_b200 import multinomial_hyper
    a0 = np.ones(D)
    ck.set_prior(multinomial_hyper(a0))
    ck.create_sufficient_statistics(np.arange(K))
    lml_g, hr_g = ck.split_hastings(K, 5.0)
    mhr_g = ck.merge_hastings(K, 5.0)
    cnt, sm, _ = O.suff_stats(x, labels, sub, K, with_S=False)
    lml = np.array([[O.mult_lml(a0, O.mult_posterior(a0, sm[k, s], cnt[k, s])) for s in range(3)] for k in range(K)])
    np.testing.assert_allclose(lml_g, lml, rtol=1e-10, atol=1e-6)
    for i in range(K):
        for j in range(i + 1, K):
            lij = O.mult_lml(a0, O.mult_posterior(a0, sm[i, 0] + sm[j, 0], 1))
            ref = O.merge_log_hr(5.0, cnt[i, 0], cnt[j, 0], lml[i, 0], lml[j, 0], lij)
            assert abs(mhr_g[i, j] - ref) <= 1e-8 * max(1, abs(ref))


# ------------------------------------------------------------------ tensor-core label phase
@pytest.mark.parametrize("D,K,N", [(64, 1, 300), (64, 2, 128), (64, 3, 5000), (64, 37, 6001), (64, 100, 3000),
                                   (64, 150, 1500), (48, 7, 2000), (32, 20, 4000)])
def test_gaussian_labels_tensor_core_parity(D, K, N):
    """split-BF16 tcgen05 contraction: r against FP64 (parity.gauss_ll: 1e-4 of the log density and
    the stated absolute bound), labels exact against the oracle's draw on FP64 r up to the margin
    rule and against its draw on the GPU's own r except at margins below 1e-4; argmax likewise."""
    from dpmmsubclusters_gpu_b200 import LL_TC_BF16X3
    rng = np.random.default_rng(1000 + D * 7 + K)
    x, z, mus, covs = _gauss_mixture(rng, N, D, K)
    x += 3.0
    mu, inv, logdet, w = _params(rng, mus + 3.0, covs)
    ck = CudaKernel(prior_type.Gaussian, loglik_mode=LL_TC_BF16X3, k_max=160).init(N, x, 7, points_major=True)
    ck.set_gaussian_params(mu, inv, logdet, w)
    u = uniforms(2 * N, D + K + 1)
    r = ck.create_clusters_labels(K, uniforms=u, return_loglik=True).astype(np.float64)
    r64 = np.stack([O.gauss_loglik(x, mu[k], inv[k], logdet[k], w[k]) for k in range(K)], 1)
    row_err = P.gauss_ll(r, r64, D, logdet, np.log(w), "tc", f"labels_tc_D{D}_K{K}")
    lab = ck.get_labels()
    u2 = u.reshape(N, 2).astype(np.float64)
    lab_o, mg = O.sample_labels(r, u2)
    _mismatch_ok(lab, lab_o, mg)
    P.labels_vs_fp64(lab, r64, u2, row_err, f"labels_tc_D{D}_K{K}_vs_fp64")
    # argmax (final iterations)
    rr = ck.create_clusters_labels(K, bFinal=True, return_loglik=True).astype(np.float64)
    lab_f = ck.get_labels()
    lab_of, gap = O.sample_labels(rr, np.zeros((N, 2)), final=True)
    assert np.all((lab_f == lab_of) | (gap < 1e-5))
    P.labels_vs_fp64(lab_f, r64, np.zeros((N, 2)), row_err, f"argmax_tc_D{D}_K{K}_vs_fp64", final=True)


@pytest.mark.parametrize("K", [1, 2, 5, 33, 64, 130, 200])
def test_tensor_core_alias_diffuse(K):
    """The warp-cooperative alias construction of the tensor-core kernel on diffuse distributions
    (every cluster within a few nats): labels exact against the oracle's sequential construction
    on the GPU's own r, except at decision margins below 1e-4."""
    from dpmmsubclusters_gpu_b200 import LL_TC_BF16X3
    rng = np.random.default_rng(500 + K)
    N, D = 4096, 64
    x = rng.normal(size=(N, D))
    mu = rng.normal(size=(K, D)) * 0.3
    inv = np.repeat((np.eye(D) * 0.05)[None], K, 0)
    logdet = np.full(K, -D * np.log(0.05))
    w = rng.dirichlet(np.ones(K) * 5)
    ck = CudaKernel(prior_type.Gaussian, loglik_mode=LL_TC_BF16X3, k_max=256).init(N, x, 7, points_major=True)
    ck.set_gaussian_params(mu, inv, logdet, w)
    u = uniforms(2 * N, K + 3)
    r = ck.create_clusters_labels(K, uniforms=u, return_loglik=True).astype(np.float64)
    lab = ck.get_labels()
    lab_o, mg = O.sample_labels(r, u.reshape(N, 2).astype(np.float64))
    # every cluster plausible: a point's construction makes O(K) comparisons near y = 1, so the
    # share of points with some margin below 1e-4 grows with K; the margin bound is the check
    _mismatch_ok(lab, lab_o, mg, frac=5e-3)
    assert len(np.unique(lab)) >= min(K, 5)
    # the same uniforms through the curand-compatible stream: TC and FP32 forms agree
    out = []
    for mode in (LL_FP32, LL_TC_BF16X3):
        c2 = CudaKernel(prior_type.Gaussian, loglik_mode=mode, k_max=256,
                        rng_kind=RNG_CURAND_XORWOW).init(N, x, 99, points_major=True)
        c2.set_gaussian_params(mu, inv, logdet, w)
        rr = c2.create_clusters_labels(K, return_loglik=True).astype(np.float64)
        out.append((rr, c2.get_labels()))
    assert np.mean(out[0][1] != out[1][1]) < 5e-3


@pytest.mark.parametrize("K", [25, 130, 200])
def test_tensor_core_persistent_many_tiles(K):
    """About four tiles per CTA, so the persistent loop, the A / B / bias rings and the TMEM r
    buffer all wrap (K = 25: three accumulators; 130: two; 200: one A slot).  r against the FP64
    oracle on every 7th point (parity.gauss_ll), labels against the oracle's draw on FP64 r there up
    to the margin rule and against its draw on the GPU's own r everywhere except at margins below
    1e-4, argmax labels against the oracle's argmax; the FP32 form agrees with the tensor-core form."""
    from dpmmsubclusters_gpu_b200 import LL_TC_BF16X3
    rng = np.random.default_rng(900 + K)
    N, D = 148 * 128 * 4 + 77, 64
    x = rng.normal(size=(N, D)) * 2.0
    mu = rng.normal(size=(K, D)) * 0.5
    A = rng.normal(size=(K, D, D)) / np.sqrt(D)
    inv = np.einsum("kij,klj->kil", A, A) * 0.05 + np.eye(D)[None] * 0.05
    logdet = -np.array([np.linalg.slogdet(m)[1] for m in inv])
    w = rng.dirichlet(np.ones(K) * 3)
    u = uniforms(2 * N, 40 + K)
    out = {}
    for mode in (LL_FP32, LL_TC_BF16X3):
        ck = CudaKernel(prior_type.Gaussian, loglik_mode=mode, k_max=256).init(N, x, 3, points_major=True)
        ck.set_gaussian_params(mu, inv, logdet, w)
        r = ck.create_clusters_labels(K, uniforms=u, return_loglik=True).astype(np.float64)
        lab = ck.get_labels()
        rf = ck.create_clusters_labels(K, bFinal=True, return_loglik=True).astype(np.float64)
        out[mode] = (r, lab, rf, ck.get_labels())
        ck.release()
    r_tc, lab_tc, rf_tc, labf_tc = out[LL_TC_BF16X3]
    sel = np.arange(0, N, 7)
    r64 = np.stack([O.gauss_loglik(x[sel], mu[k], inv[k], logdet[k], w[k]) for k in range(K)], 1)
    u2 = u.reshape(N, 2).astype(np.float64)
    for mode, path in ((LL_TC_BF16X3, "tc"), (LL_FP32, "fp32")):
        row_err = P.gauss_ll(out[mode][0][sel], r64, D, logdet, np.log(w), path, f"persistent_{path}_K{K}")
        P.labels_vs_fp64(out[mode][1][sel], r64, u2[sel], row_err, f"persistent_{path}_K{K}_vs_fp64")
    lab_o, mg = O.sample_labels(r_tc, u2)
    _mismatch_ok(lab_tc, lab_o, mg, frac=5e-3)
    lab_of, gap = O.sample_labels(rf_tc, np.zeros((N, 2)), final=True)
    assert np.all((labf_tc == lab_of) | (gap < 1e-5))


def test_tensor_core_matches_fp32_form():
    from dpmmsubclusters_gpu_b200 import LL_TC_BF16X3
    rng = np.random.default_rng(77)
    N, D, K = 20000, 64, 25
    x, z, mus, covs = _gauss_mixture(rng, N, D, K)
    mu, inv, logdet, w = _params(rng, mus, covs)
    u = uniforms(2 * N, 5)
    out = []
    for mode in (LL_FP32, LL_TC_BF16X3):
        ck = CudaKernel(prior_type.Gaussian, loglik_mode=mode).init(N, x, 7, points_major=True)
        ck.set_gaussian_params(mu, inv, logdet, w)
        r = ck.create_clusters_labels(K, uniforms=u, return_loglik=True)
        out.append((r, ck.get_labels()))
    assert np.abs(out[0][0] - out[1][0]).max() < 0.05
    assert np.mean(out[0][1] != out[1][1]) < 1e-3

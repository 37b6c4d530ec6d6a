"""GPU checks of the device parameter draws and the device statistics bookkeeping
(csrc/dpmm_params.cu), through the C ABI.

The draws are random, so they are checked against the distribution the reference samples
(niw::sample_distribution, niw.cpp:82-107: Sigma ~ IW(nu', nu' psi'), mu ~ N(m', Sigma / kappa'))
with the posterior (niw.cpp:23-49) restated in numpy from the same statistics:
  * E[W W^T] = psi'^-1 (the precision's mean): Frobenius error <= 6 sqrt(2 / (M nu')) + 2e-4 relative
  * E[mu] = m': every coordinate within 6 standard errors
  * E[log det Lambda] = sum_i digamma((nu' - i + 1) / 2) + D log 2 - log det(nu' psi'): within 6 standard
    errors (trigamma variance) + 1e-4
  * each slot's log marginal likelihood against the FP64 formula of niw.cpp:122-138: 1e-9 relative
  * b = W^T (mu - shift) as packed: FP32 rounding (1e-4 relative to the terms' scale)
  * the merge / compaction bookkeeping: exact
"""
import math

import numpy as np
import pytest
from scipy.special import digamma, gammaln, polygamma

from dpmmsubclusters_gpu_b200 import CudaKernel, niw_hyperparams, prior_type
from dpmmsubclusters_gpu_b200.api import dp_parallel_sampling_class

pytestmark = pytest.mark.gpu


def _setup(seed, N=24000, D=6, K=3, empty_r=False):
    rng = np.random.default_rng(seed)
    mus = rng.normal(size=(K, D)) * 4.0
    z = rng.integers(0, K, size=N)
    x = np.empty((N, D))
    for c in range(K):
        A = rng.normal(size=(D, D))
        idx = np.flatnonzero(z == c)
        x[idx] = rng.multivariate_normal(mus[c], A @ A.T / D + 0.5 * np.eye(D), size=idx.size)
    sub = rng.integers(1, 3, size=N).astype(np.int32)
    if empty_r:
        sub[z == 0] = 1
    kern = CudaKernel(prior_type.Gaussian, k_max=16).init(N, x.T, seed=seed)
    kern.set_labels((z + 1).astype(np.int32))
    kern.set_sub_labels(sub)
    kern.set_prior(niw_hyperparams(1.0, np.zeros(D), D + 3.0, np.eye(D)))
    cnt, sm, S = kern.create_sufficient_statistics(np.arange(K))
    return kern, x, cnt.reshape(-1), sm.reshape(-1, D), S.reshape(-1, D, D)


def _posterior(n, s, S, D, k0=1.0, v0=None, m0=None, psi0=None):
    v0 = D + 3.0 if v0 is None else v0
    m0 = np.zeros(D) if m0 is None else m0
    psi0 = np.eye(D) if psi0 is None else psi0
    kp, vp = k0 + n, v0 + n
    mp = (k0 * m0 + s) / kp
    U = np.triu(v0 * psi0 + k0 * np.outer(m0, m0) - kp * np.outer(mp, mp) + S)
    psi = (U + np.triu(U, 1).T) / vp
    return kp, vp, mp, psi


def _lml(n, D, psi, kp, vp, k0=1.0, v0=None):
    v0 = D + 3.0 if v0 is None else v0
    d = np.arange(1, D + 1)
    g = np.sum(gammaln(vp / 2 + (1 - d) / 2) - gammaln(v0 / 2 + (1 - d) / 2))
    ld = np.linalg.slogdet(psi)[1]
    return (-n * D * 0.5 * math.log(math.pi) + g + (v0 / 2) * (D * math.log(v0)) - (vp / 2) * (D * math.log(vp) + ld)
            + (D / 2) * math.log(k0 / kp))


@pytest.mark.parametrize("empty_r", [False, True])
def test_draw_moments_match_the_posterior(empty_r):
    D, K, M = 6, 3, 500
    kern, x, cnt, sm, S = _setup(3, D=D, K=K, empty_r=empty_r)
    shift = x.mean(0)
    w = np.array([0.5, 0.3, 0.2])
    lrw = np.full(2 * K, 0.5)
    accL = np.zeros((3 * K, D, D))
    accmu = np.zeros((3 * K, D))
    accld = np.zeros(3 * K)
    for d in range(M):
        lml = kern.sample_gaussian_params(K, 1234, d, w, lrw).reshape(-1)
        W, b, c, mu = kern.gaussian_params(K)
        W = W.astype(np.float64)
        accL += W @ np.swapaxes(W, 1, 2)
        accmu += mu
        ldl = 2 * c.astype(np.float64)                       # log det Lambda (+ 2 log w on cluster slots)
        ldl[0::3] -= 2 * np.log(w)
        accld += ldl
        if d == 0:
            # b = W^T (mu - shift) as packed
            bb = np.einsum("sij,si->sj", W, mu.astype(np.float64))
            scale = np.einsum("sij,si->sj", np.abs(W), np.abs(mu.astype(np.float64))) + 1e-6
            assert np.all(np.abs(b - bb) <= 1e-4 * scale)
            for q in range(3 * K):
                if cnt[q] == 0:
                    assert lml[q] == 0.0
                    continue
                kp, vp, mp, psi = _posterior(cnt[q], sm[q], S[q], D)
                ref = _lml(cnt[q], D, psi, kp, vp)
                assert abs(lml[q] - ref) <= 1e-9 * abs(ref) + 1e-9, (q, lml[q], ref)
    for q in range(3 * K):
        kp, vp, mp, psi = _posterior(cnt[q], sm[q], S[q], D)
        lam = np.linalg.inv(psi)
        err = np.linalg.norm(accL[q] / M - lam) / np.linalg.norm(lam)
        assert err <= 6 * math.sqrt(2.0 / (M * vp)) + 2e-4, (q, err)
        se = np.sqrt(np.diag(psi) * vp / max(vp - D - 1, 1.0) / kp / M)
        assert np.all(np.abs(accmu[q] / M + shift - mp) <= 6 * se + 1e-5), (q, accmu[q] / M + shift - mp, se)
        i = np.arange(1, D + 1)
        eld = np.sum(digamma((vp - i + 1) / 2)) + D * math.log(2) - np.linalg.slogdet(vp * psi)[1]
        sd = math.sqrt(np.sum(polygamma(1, (vp - i + 1) / 2)) / M)
        assert abs(accld[q] / M - eld) <= 6 * sd + 1e-4, (q, accld[q] / M, eld, sd)


def test_draw_is_a_function_of_seed_and_draw():
    kern, x, *_ = _setup(5)
    w, lrw = np.full(3, 1 / 3), np.full(6, 0.5)
    kern.sample_gaussian_params(3, 7, 11, w, lrw)
    a = kern.gaussian_params(3)
    kern.sample_gaussian_params(3, 7, 12, w, lrw)
    b = kern.gaussian_params(3)
    kern.sample_gaussian_params(3, 7, 11, w, lrw)
    c = kern.gaussian_params(3)
    for u, v in zip(a, c):
        np.testing.assert_array_equal(u, v)
    assert not np.array_equal(a[0], b[0])


def test_merge_and_compact_statistics_follow_the_host_bookkeeping():
    D, K = 5, 5
    kern, x, cnt, sm, S = _setup(9, D=D, K=K)
    c3 = lambda arr: arr.reshape(K, 3, *arr.shape[1:])
    cnt, sm, S = c3(cnt.astype(np.float64)), c3(sm), c3(S)
    kern.merge_statistics([0, 1], [3, 4])
    n2, s2, S2 = kern.create_sufficient_statistics(np.arange(K))
    for i, j in ((0, 3), (1, 4)):
        for slot, (en, es, eS) in enumerate(((cnt[i, 0] + cnt[j, 0], sm[i, 0] + sm[j, 0], S[i, 0] + S[j, 0]),
                                             (cnt[i, 0] + cnt[j, 0], sm[i, 0] + sm[j, 0], S[i, 0] + S[j, 0]),
                                             (cnt[j, 0], sm[j, 0], S[j, 0]))):
            assert n2[i, slot] == en
            np.testing.assert_array_equal(s2[i, slot], es)
            np.testing.assert_array_equal(S2[i, slot], eS)
    kern.compact_statistics([0, 1, 2])
    n3, s3, S3 = kern.create_sufficient_statistics(np.arange(3))
    np.testing.assert_array_equal(n3, n2[:3])
    np.testing.assert_array_equal(s3, s2[:3])
    np.testing.assert_array_equal(S3, S2[:3])
    np.testing.assert_array_equal(kern.statistics_counts(np.arange(3)), n2[:3])


def _mixture(seed, N, D, K, spread):
    rng = np.random.default_rng(seed)
    mus = rng.normal(size=(K, D)) * spread
    z = rng.integers(0, K, size=N)
    x = np.empty((N, D))
    for c in range(K):
        A = rng.normal(size=(D, D))
        idx = np.flatnonzero(z == c)
        x[idx] = rng.multivariate_normal(mus[c], A @ A.T / D + 0.5 * np.eye(D), size=idx.size)
    return x, z


def test_sampler_with_device_draws_matches_host_draws_statistically():
    from sklearn.metrics import normalized_mutual_info_score as nmi
    x, z = _mixture(71, 60000, 8, 6, 5.0)
    res = {}
    for host in (True, False):
        s = dp_parallel_sampling_class(x.shape[0], x.T, 11, prior_type.Gaussian, host_param_draws=host)
        mi = s.dp_parallel(niw_hyperparams(1.0, np.zeros(8), 11.0, np.eye(8)), 10.0, iters=60, init_clusters=3,
                           verbose=True, burnout=5)
        res[host] = (nmi(z, mi.labels), mi.cluster_count_history[-1], mi.likelihood_history[-1])
    (nh, kh, lh), (nd, kd, ld) = res[True], res[False]
    assert nh > 0.9 and nd > 0.9 and abs(nh - nd) <= 0.05, res
    assert abs(kh - kd) <= 2, res
    assert abs(lh - ld) <= 1e-2 * abs(lh), res


def test_dirichlet_draws_match_the_posterior():
    """multinomial_prior::sample_distribution on the device (dpmm_sample_multinomial_params): over M draws,
    E[theta] = alpha' / sum alpha' within 6 standard errors (Dirichlet variance), every draw on the simplex,
    and each slot's log marginal likelihood equal to multinomial_prior.cpp:56-67 in FP64 (1e-9 relative)."""
    from dpmmsubclusters_gpu_b200 import multinomial_hyper
    rng = np.random.default_rng(8)
    N, D, K, M = 3000, 12, 2, 400
    theta = rng.dirichlet(np.ones(D) * 0.5, size=K)
    z = rng.integers(0, K, size=N)
    x = np.stack([rng.multinomial(5, theta[k]) for k in z]).astype(np.float64)
    sub = rng.integers(1, 3, size=N).astype(np.int32)
    a0 = np.full(D, 0.7)
    kern = CudaKernel(prior_type.Multinomial, k_max=8).init(N, x.T, seed=1)
    kern.set_labels((z + 1).astype(np.int32))
    kern.set_sub_labels(sub)
    kern.set_prior(multinomial_hyper(a0))
    cnt, sm, _ = kern.create_sufficient_statistics(np.arange(K))
    ap = a0[None, None, :] + sm                      # (K, 3, D) posterior
    draws = np.empty((M, K, 3, D))
    for d in range(M):
        lml = kern.sample_multinomial_params(K, 77, d, np.full((K, 2), 0.5))
        draws[d] = np.exp(kern.get_multinomial_params(K).astype(np.float64))
    np.testing.assert_allclose(draws.sum(-1), 1.0, atol=1e-5)
    A = ap.sum(-1, keepdims=True)
    mean, var = ap / A, ap * (A - ap) / (A ** 2 * (A + 1))
    se = np.sqrt(var / M)
    assert np.all(np.abs(draws.mean(0) - mean) <= 6 * se + 1e-6), np.abs(draws.mean(0) - mean).max()
    lml_ref = gammaln(a0.sum()) - gammaln(A[..., 0]) + np.sum(gammaln(ap) - gammaln(a0), -1)
    np.testing.assert_allclose(lml, np.where(cnt > 0, lml_ref, 0.0), rtol=1e-9, atol=1e-9)
    # the draws differ from draw to draw and repeat for the same (seed, draw)
    kern.sample_multinomial_params(K, 77, 5, np.full((K, 2), 0.5))
    again = np.exp(kern.get_multinomial_params(K).astype(np.float64))
    np.testing.assert_array_equal(again, draws[5])
    assert not np.allclose(draws[5], draws[6])


def test_multinomial_run_with_device_draws_finds_the_components():
    """A whole multinomial run with the Dirichlet draws on the device (the default) against the same run
    with host draws: both recover the generating components (NMI), with similar cluster counts."""
    from dpmmsubclusters_gpu_b200 import multinomial_hyper
    rng = np.random.default_rng(12)
    N, D, K = 20000, 40, 4
    theta = rng.dirichlet(np.ones(D) * 0.2, size=K)
    z = rng.integers(0, K, size=N)
    x = np.stack([rng.multinomial(60, theta[k]) for k in z]).astype(np.float64)
    out = {}
    for host in (False, True):
        s = dp_parallel_sampling_class(N, x.T, 3, prior_type.Multinomial, host_param_draws=host)
        mi = s.dp_parallel(multinomial_hyper(np.ones(D)), 10.0, iters=60, init_clusters=1, verbose=False)
        from sklearn.metrics import normalized_mutual_info_score
        out[host] = (normalized_mutual_info_score(z, mi.labels), len(np.unique(mi.labels)))
    assert out[False][0] > 0.95 and out[True][0] > 0.95, out
    assert abs(out[False][1] - out[True][1]) <= 2, out

"""Device parameter draws in runs with an outlier cluster (outlier_mod > 0; the reference's default in
its params JSON, global_params.h:54): the outlier cluster's own prior on the device
(dpmm_set_outlier_prior_niw / dpmm_set_cluster_priors) and cluster 1 not redrawn
(local_clusters_actions.cpp:348-351), against the FP64 oracle.

The sampler keeps host draws for such runs: their course is dominated by the never-redrawn cluster 1,
and whole runs were not shown to match between the two kinds of draw.  The device path is for callers
of the C ABI; the device split / merge ratios use each cluster's own prior in either case.

Criteria: per-slot log marginal likelihoods within 1e-6 relative of the FP64 oracle under the prior
the slot's cluster carries (the Hastings tests' bound; the two priors differ by far more); cluster 1's
label parameters unchanged by a draw except its weight term; a whole run gathers the scattered points
in one cluster of the outlier prior."""
import ctypes

import numpy as np
import pytest

from dpmmsubclusters_gpu_b200 import (CudaKernel, dp_parallel_sampling_class, niw_hyperparams, multinomial_hyper,
                                      prior_type)
from dpmmsubclusters_gpu_b200.capi import check, lib
from oracle import oracle as O

pytestmark = pytest.mark.gpu

_PD = ctypes.POINTER(ctypes.c_double)
_PF = ctypes.POINTER(ctypes.c_float)


def _d(a):
    return np.ascontiguousarray(a, np.float64).ctypes.data_as(_PD)


def _mixture(seed, N, D, K, spread=4.0):
    rng = np.random.default_rng(seed)
    mus = rng.normal(size=(K, D)) * spread
    z = rng.integers(0, K, size=N)
    x = mus[z] + rng.normal(size=(N, D))
    return rng, x, z


def _oracle_lml(cnt, sm, S, prior):
    k0, m0, v0, psi0 = prior
    kk, m, v, psi = O.niw_posterior(k0, m0, v0, psi0, cnt, sm, S)
    return O.niw_lml(k0, v0, psi0, kk, v, psi, cnt)


def _setup(D, K, N, seed):
    rng, x, z = _mixture(seed, N, D, K)
    labels = (z + 1).astype(np.int32)
    sub = rng.integers(1, 3, size=N).astype(np.int32)
    ck = CudaKernel(prior_type.Gaussian, k_max=16).init(N, x, 1, points_major=True)
    ck.set_labels(labels)
    ck.set_sub_labels(sub)
    reg = (1.0, np.zeros(D), D + 3.0, np.eye(D))
    out = (0.3, np.full(D, 2.0), D + 6.0, 3.0 * np.eye(D))
    ck.set_prior(niw_hyperparams(*reg))
    check(lib().dpmm_set_outlier_prior_niw(ck.ctx, out[0], _d(out[1]), out[2], _d(out[3])))
    sel = np.array([1, 0, 1, 0, 0][:K], np.uint8)
    check(lib().dpmm_set_cluster_priors(ck.ctx, K, sel.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))
    return x, labels, sub, ck, reg, out, sel


def test_marginal_likelihoods_use_each_clusters_prior():
    D, K, N = 8, 5, 20000
    x, labels, sub, ck, reg, out, sel = _setup(D, K, N, 3)
    ck.create_sufficient_statistics(np.arange(K))
    lml_g, _ = ck.split_hastings(K, 10.0)
    cnt, sm, S = O.suff_stats(x, labels, sub, K)
    lml = np.array([[_oracle_lml(cnt[k, s], sm[k, s], S[k, s], out if sel[k] else reg) for s in range(3)]
                    for k in range(K)])
    assert np.abs(lml_g - lml).max() <= 1e-6 * np.abs(lml).max(), np.abs(lml_g - lml).max()
    ck.release()


def test_device_draw_keeps_cluster_1_and_uses_the_outlier_prior():
    D, K, N = 8, 5, 20000
    x, labels, sub, ck, reg, out, sel = _setup(D, K, N, 4)
    rng = np.random.default_rng(0)
    mu = rng.normal(size=(K, D))
    inv = np.repeat(np.eye(D)[None], K, 0) * rng.uniform(0.5, 2.0, size=(K, 1, 1))
    logdet = -np.array([np.linalg.slogdet(a)[1] for a in inv])
    w = np.full(K, 1.0 / K)
    mu_lr = np.repeat(mu[:, None], 2, 1)
    inv_lr = np.repeat(inv[:, None], 2, 1)
    ld_lr = np.repeat(logdet[:, None], 2, 1)
    ck.set_gaussian_params(mu, inv, logdet, w, mu_lr, inv_lr, ld_lr, np.full((K, 2), 0.5))
    ck.create_sufficient_statistics(np.arange(K))
    Dp = 8

    def params():
        wt = np.empty((3 * K, Dp, Dp), np.float32)
        b = np.empty((3 * K, Dp), np.float32)
        c = np.empty(3 * K, np.float32)
        m = np.empty((3 * K, Dp), np.float32)
        check(lib().dpmm_get_gaussian_params(ck.ctx, K, wt.ctypes.data_as(_PF), b.ctypes.data_as(_PF),
                                              c.ctypes.data_as(_PF), m.ctypes.data_as(_PF)))
        return wt, b, c, m

    before = params()
    w2 = np.array([0.05, 0.4, 0.25, 0.2, 0.1])
    lrw = np.full(2 * K, 0.5)
    lml = np.empty(3 * K)
    check(lib().dpmm_sample_gaussian_params(ck.ctx, K, 7, 1, _d(w2), _d(lrw), lml.ctypes.data_as(_PD)))
    after = params()
    # cluster 1 (slots 3..5): parameters kept, the cluster slot's weight term refreshed
    for a, b_ in zip(before[:2] + before[3:], after[:2] + after[3:]):
        np.testing.assert_array_equal(a[3:6], b_[3:6])
    np.testing.assert_allclose(after[2][3], -logdet[1] / 2 + np.log(w2[1]), rtol=1e-6)
    np.testing.assert_array_equal(after[2][4:6], before[2][4:6])
    # the others redrawn, with each cluster's prior in their marginal likelihoods
    assert not np.array_equal(before[0][0:3], after[0][0:3])
    assert not np.array_equal(before[0][6:], after[0][6:])
    cnt, sm, S = O.suff_stats(x, labels, sub, K)
    ref = np.array([_oracle_lml(cnt[k, s], sm[k, s], S[k, s], out if sel[k] else reg) for k in range(K) for s in range(3)])
    assert np.abs(lml - ref).max() <= 1e-6 * np.abs(ref).max(), np.abs(lml - ref).max()
    ck.release()


def _nmi(a, b):
    from sklearn.metrics import normalized_mutual_info_score
    return normalized_mutual_info_score(a, b)


def test_outlier_run_uses_each_clusters_prior_in_its_ratios():
    # whole runs with an outlier cluster (host draws; the device split / merge ratios with each
    # cluster's own prior): the outlier cluster keeps the scattered points
    rng = np.random.default_rng(21)
    N, D, K = 30000, 4, 5
    mus = rng.normal(size=(K, D)) * 8
    z = rng.integers(0, K, size=N)
    x = mus[z] + rng.normal(size=(N, D))
    n_out = 300
    x[:n_out] = rng.uniform(-60, 60, size=(n_out, D))   # scattered outliers
    hyper = niw_hyperparams(1.0, np.zeros(D), D + 3.0, np.eye(D))
    spc = dp_parallel_sampling_class(N, x.T, 3, prior_type.Gaussian)
    mi = spc.dp_parallel(hyper, 10.0, iters=60, verbose=False, burnout=15, outlier_weight=0.05,
                         outlier_params=niw_hyperparams(1.0, np.zeros(D), D + 3.0, 100.0 * np.eye(D)))
    lab = np.asarray(mi.labels)
    assert lab.size == N and mi.iter_count.size == 60
    # the scattered points end in one cluster of their own (the outlier cluster or one split from it,
    # both under the broad outlier prior) that takes almost none of the mixture's points
    vals, cnts = np.unique(lab[:n_out], return_counts=True)
    mode = vals[np.argmax(cnts)]
    assert cnts.max() / n_out > 0.9, (vals, cnts)
    assert np.mean(lab[n_out:] == mode) < 0.01

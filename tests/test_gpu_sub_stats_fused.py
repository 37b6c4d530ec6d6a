"""The fused sub-label + statistics pass (csrc/dpmm_tc.cu k_sub_stats_tc, dpmm_set_fused_sub_stats(ctx, 1):
each point gathered once for the sub-label contraction, the draw and the split-TF32 statistics) against
the two kernels it can replace (k_sub_labels_tc, then k_slot_stats_tc: the default) and the FP64 oracle.

Criteria:
  * sub-cluster log-likelihoods and sub-labels: bit-exact against the two-kernel path (the same
    split-BF16 operands and the same 12 products per 128-point tile), and r within the parity bounds
    of the FP64 oracle (tests/parity.py);
  * statistics of the drawn sub-labels: counts exact; sums and scatter within 1e-6 relative of the
    FP64 oracle (the two paths accumulate the same products in tiles of 16 and 32 points, so they agree
    to FP32 rounding, not bit for bit);
  * chunk tails: clusters of 1 .. 5000 points (partial 16-point statistics tiles, partial 128-point
    super-tiles, partial 256-point accumulation groups, several chunks per cluster).
"""
import numpy as np
import pytest

import parity as P
from conftest import uniforms
from dpmmsubclusters_gpu_b200 import LL_TC_BF16X3, CudaKernel, DpmmError, prior_type
from dpmmsubclusters_gpu_b200.capi import check, lib
from oracle import oracle as O

pytestmark = pytest.mark.gpu

DPMM_ERR_TIMEOUT = 5
SIZES = [1, 15, 16, 17, 127, 128, 129, 255, 256, 257, 1023, 1024, 1025, 4999]


def _setup(seed, D, sizes, offset):
    rng = np.random.default_rng(seed)
    K = len(sizes)
    N = int(sum(sizes))
    mus = rng.normal(size=(K, D)) * 4 + offset
    z = np.repeat(np.arange(K), sizes)
    rng.shuffle(z)
    x = np.empty((N, D))
    covs = []
    for k in range(K):
        A = rng.normal(size=(D, D))
        c = A @ A.T / D + 0.5 * np.eye(D)
        covs.append(c)
        idx = np.flatnonzero(z == k)
        x[idx] = rng.multivariate_normal(mus[k], c, size=idx.size)
    covs = np.array(covs)
    mu = mus + 0.3 * rng.normal(size=mus.shape)
    inv = np.array([np.linalg.inv(c) for c in covs])
    logdet = np.array([np.linalg.slogdet(c)[1] for c in covs])
    w = rng.dirichlet(np.ones(K) * 2)
    mu_lr = mu[:, None, :] + 0.7 * rng.normal(size=(K, 2, D))
    inv_lr = np.repeat(inv[:, None], 2, axis=1) * rng.uniform(0.8, 1.2, size=(K, 2, 1, 1))
    ld_lr = np.array([[-np.linalg.slogdet(inv_lr[k, s])[1] for s in range(2)] for k in range(K)])
    lrw = rng.dirichlet([2, 2], size=K)
    return x, (z + 1).astype(np.int32), (mu, inv, logdet, w, mu_lr, inv_lr, ld_lr, lrw)


def _run(x, labels, params, fused, u, loglik=True, seed=11):
    N, D = x.shape
    K = params[0].shape[0]
    ck = CudaKernel(prior_type.Gaussian, loglik_mode=LL_TC_BF16X3, k_max=32).init(N, x, seed, points_major=True)
    check(lib().dpmm_set_fused_sub_stats(ck.ctx, fused))
    ck.set_gaussian_params(*params)
    ck.set_labels(labels)
    r = ck.create_subclusters_labels(K, uniforms=u, return_loglik=loglik)
    sub = ck.get_sub_labels()
    st = ck.create_sufficient_statistics(np.arange(K))
    ck.release()
    return (None if r is None else np.asarray(r, np.float64)), sub, st


def _check_stats(st, x, labels, sub, K, tag):
    cnt, sm, S = st
    cnt_o, sm_o, S_o = O.suff_stats(x, labels, sub, K)
    np.testing.assert_array_equal(cnt, cnt_o)
    np.testing.assert_allclose(sm, sm_o, atol=1e-6 * (np.abs(sm_o).max() + 1) * 10, rtol=1e-6)
    np.testing.assert_allclose(S, S_o, atol=1e-6 * (np.abs(S_o).max() + 1), rtol=1e-6)
    P.record(tag, max_rel_S=float(np.abs(S - S_o).max() / (np.abs(S_o).max() + 1)),
             max_rel_sum=float(np.abs(sm - sm_o).max() / (np.abs(sm_o).max() + 1)))


@pytest.mark.parametrize("D,offset", [(64, 0.0), (64, 40.0), (48, -20.0), (32, 5.0), (20, 0.0)])
def test_fused_equals_two_kernels_and_fp64(D, offset):
    x, labels, params = _setup(100 + D, D, SIZES, offset)
    N, K = x.shape[0], len(SIZES)
    u = uniforms(2 * N, 5 + D)
    r_f, sub_f, st_f = _run(x, labels, params, 1, u)
    r_s, sub_s, st_s = _run(x, labels, params, 0, u)
    np.testing.assert_array_equal(r_f, r_s)
    np.testing.assert_array_equal(sub_f, sub_s)
    assert set(np.unique(sub_f)) <= {1, 2}
    # r and the draw against FP64
    mu, inv, logdet, w, mu_lr, inv_lr, ld_lr, lrw = params
    _, _, r64 = O.gauss_sub_labels(x, labels, mu_lr, inv_lr, ld_lr, lrw, u.astype(np.float64))
    row_err = P.gauss_ll(r_f, r64, D, ld_lr[labels - 1], 0.0, "fused", f"fused_sub_D{D}")
    P.sub_labels_vs_fp64(sub_f, r64, labels, lrw, u.reshape(N, 2).astype(np.float64), row_err,
                         f"fused_sub_D{D}_vs_fp64")
    _check_stats(st_f, x, labels, sub_f, K, f"fused_stats_D{D}_off{offset}")
    _check_stats(st_s, x, labels, sub_s, K, f"two_kernel_stats_D{D}_off{offset}")
    np.testing.assert_array_equal(st_f[0], st_s[0])
    np.testing.assert_allclose(st_f[2], st_s[2], atol=2e-6 * (np.abs(st_s[2]).max() + 1), rtol=2e-6)


def test_fused_without_loglik_and_internal_rng():
    # the draw path the sampler takes: no r output, uniforms from the context's own generator
    x, labels, params = _setup(7, 64, [3000, 20000, 700, 9000], 0.0)
    _, sub_f, st_f = _run(x, labels, params, 1, None, loglik=False, seed=123)
    _, sub_s, st_s = _run(x, labels, params, 0, None, loglik=False, seed=123)
    np.testing.assert_array_equal(sub_f, sub_s)
    _check_stats(st_f, x, labels, sub_f, 4, "fused_stats_internal_rng")
    np.testing.assert_array_equal(st_f[0], st_s[0])


def test_fused_wait_runs_out_and_the_context_stays_usable():
    # dpmm_set_wait_test: the fused kernel's MMA thread issues nothing, so the sub-label group's waits
    # for its products run out (2 s); the call returns DPMM_ERR_TIMEOUT and the next call works
    import time
    x, labels, params = _setup(9, 64, [5000, 3000], 0.0)
    N, K = x.shape[0], 2
    u = uniforms(2 * N, 3)
    ck = CudaKernel(prior_type.Gaussian, loglik_mode=LL_TC_BF16X3, k_max=8).init(N, x, 1, points_major=True)
    check(lib().dpmm_set_fused_sub_stats(ck.ctx, 1))
    ck.set_gaussian_params(*params)
    ck.set_labels(labels)
    check(lib().dpmm_set_wait_test(ck.ctx, 1))
    t0 = time.perf_counter()
    with pytest.raises(DpmmError) as e:
        ck.create_subclusters_labels(K, uniforms=u, return_loglik=True)
    dt = time.perf_counter() - t0
    check(lib().dpmm_set_wait_test(ck.ctx, 0))
    assert e.value.status == DPMM_ERR_TIMEOUT, e.value
    assert 1.0 <= dt <= 60.0, dt
    for _ in range(2):
        ck.create_subclusters_labels(K, uniforms=u, return_loglik=True)
        sub = ck.get_sub_labels()
        _check_stats(ck.create_sufficient_statistics(np.arange(K)), x, labels, sub, K, "fused_after_timeout")
    ck.release()

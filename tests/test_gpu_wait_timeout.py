"""Bounded device waits: a wait that runs out ends the kernel with an error status, not a hang.

dpmm_set_wait_test makes the tensor-core kernels issue no products, so the waits for them (the
drain warps' and the producer's mbarrier waits of the label kernels, the single waiting thread of the
scan, sub-label and statistics kernels, each bounded by a 2 s limit read from %globaltimer) run out:
the call must return DPMM_ERR_TIMEOUT after about that limit, with the kernel having waited for the
copies it issued and freed its tensor memory -- the next calls on the same context, with the test
switched off, must run and give correct results (they allocate the same tensor memory again).
"""
import ctypes
import time

import numpy as np
import pytest

from conftest import uniforms
from dpmmsubclusters_gpu_b200 import LL_TC_BF16X3, CudaKernel, DpmmError, prior_type
from dpmmsubclusters_gpu_b200.capi import check, lib
from oracle import oracle as O

pytestmark = pytest.mark.gpu

DPMM_ERR_TIMEOUT = 5


def _expect_timeout(ck, K, u):
    check(lib().dpmm_set_wait_test(ck.ctx, 1))
    t0 = time.perf_counter()
    with pytest.raises(DpmmError) as e:
        ck.create_clusters_labels(K, uniforms=u, return_loglik=True)   # return_loglik: the dense kernel runs
    dt = time.perf_counter() - t0
    check(lib().dpmm_set_wait_test(ck.ctx, 0))
    assert e.value.status == DPMM_ERR_TIMEOUT, e.value
    assert 1.0 <= dt <= 60.0, dt        # the wait limit is 2 s
    return dt


def test_gaussian_tensor_core_wait_runs_out_and_the_context_stays_usable():
    rng = np.random.default_rng(1)
    N, D, K = 20000, 64, 9
    mus = rng.normal(size=(K, D)) * 3
    z = rng.integers(0, K, size=N)
    x = mus[z] + rng.normal(size=(N, D))
    inv = np.repeat(np.eye(D)[None], K, 0)
    ck = CudaKernel(prior_type.Gaussian, loglik_mode=LL_TC_BF16X3, k_max=16).init(N, x, 1, points_major=True)
    ck.set_gaussian_params(mus, inv, np.zeros(K), np.full(K, 1.0 / K))
    u = uniforms(2 * N, 3)
    _expect_timeout(ck, K, u)
    for _ in range(2):          # the context works again, twice in a row
        r = ck.create_clusters_labels(K, uniforms=u, return_loglik=True).astype(np.float64)
        lab_o, mg = O.sample_labels(r, u.reshape(N, 2).astype(np.float64))
        bad = ck.get_labels() != lab_o
        assert np.all(mg[bad] < 1e-4)
    ck.release()


def test_multinomial_tensor_core_wait_runs_out_and_the_context_stays_usable():
    rng = np.random.default_rng(2)
    N, D, K = 9000, 200, 6
    theta = rng.dirichlet(np.ones(D) * 0.3, size=K)
    z = rng.integers(0, K, size=N)
    x = np.stack([rng.multinomial(50, theta[k]) for k in z]).astype(np.float64)
    lt = np.log(theta * 0.9 + 0.1 / D)
    ck = CudaKernel(prior_type.Multinomial, loglik_mode=LL_TC_BF16X3, k_max=8).init(N, x, 1, points_major=True)
    ck.set_multinomial_params(lt)
    u = uniforms(2 * N, 4)
    _expect_timeout(ck, K, u)
    r = ck.create_clusters_labels(K, uniforms=u, return_loglik=True).astype(np.float64)
    lab_o, mg = O.sample_labels(r, u.reshape(N, 2).astype(np.float64))
    bad = ck.get_labels() != lab_o
    assert np.all(mg[bad] < 1e-4)
    r64 = np.stack([O.mult_loglik(x, lt[k]) for k in range(K)], 1)
    assert (np.abs(r - r64) / np.maximum(x @ np.abs(lt).T, 1)).max() <= 1e-5
    ck.release()


def _separated(seed, N, D, K):
    rng = np.random.default_rng(seed)
    mus = rng.normal(size=(K, D)) * 3
    z = rng.integers(0, K, size=N)
    x = mus[z] + rng.normal(size=(N, D))
    inv = np.repeat(np.eye(D)[None], K, 0)
    mu_lr = mus[:, None, :] + 0.5 * rng.normal(size=(K, 2, D))
    params = (mus, inv, np.zeros(K), np.full(K, 1.0 / K), mu_lr, np.repeat(inv[:, None], 2, 1), np.zeros((K, 2)),
              np.full((K, 2), 0.5))
    return rng, x, (z + 1).astype(np.int32), params


def _context(x, labels, params, K):
    N = x.shape[0]
    ck = CudaKernel(prior_type.Gaussian, loglik_mode=LL_TC_BF16X3, k_max=16).init(N, x, 1, points_major=True)
    ck.set_gaussian_params(*params)
    ck.set_labels(labels)
    return ck


def _stalled(ck, call):
    check(lib().dpmm_set_wait_test(ck.ctx, 1))
    t0 = time.perf_counter()
    with pytest.raises(DpmmError) as e:
        call()
    dt = time.perf_counter() - t0
    check(lib().dpmm_set_wait_test(ck.ctx, 0))
    assert e.value.status == DPMM_ERR_TIMEOUT, e.value
    assert 1.0 <= dt <= 60.0, dt
    return dt


@pytest.mark.parametrize("step", ["pruned_scan", "sub_labels", "statistics"])
def test_block_synchronous_kernel_wait_runs_out_and_the_context_stays_usable(step):
    # the kernels where one thread waits for the block's products (k_prune_scan1_tc, k_sub_labels_tc,
    # k_slot_stats_tc): with the seam on the wait runs out, the call reports DPMM_ERR_TIMEOUT, and the
    # same context then gives the results of a context that never stalled
    N, D, K = 30000, 64, 10
    rng, x, labels, params = _separated(5, N, D, K)
    u = uniforms(2 * N, 6)
    sub = rng.integers(1, 3, size=N).astype(np.int32)
    ck = _context(x, labels, params, K)
    fresh = _context(x, labels, params, K)
    if step == "pruned_scan":
        for c in (ck, fresh):
            check(lib().dpmm_set_label_pruning(c.ctx, 30.0))

        def run(c):
            c.set_labels(labels)
            c.create_clusters_labels(K, uniforms=u)   # no log-likelihood output: the pruned phase runs
            return [c.get_labels()]
    elif step == "sub_labels":
        def run(c):
            r = c.create_subclusters_labels(K, uniforms=u, return_loglik=True)
            return [np.asarray(r), c.get_sub_labels()]
    else:
        def run(c):
            c.set_sub_labels(sub)
            return list(c.create_sufficient_statistics(np.arange(K)))
    _stalled(ck, lambda: run(ck))
    want = run(fresh)
    for _ in range(2):
        got = run(ck)
        for a, b in zip(got, want):
            np.testing.assert_array_equal(a, b)
    if step == "pruned_scan":
        out = (ctypes.c_double * 6)()
        check(lib().dpmm_label_pruning_stats(ck.ctx, out))
        assert out[1] == 2, list(out)   # both runs after the stall ran pruned
    if step == "statistics":
        cnt, sm, S = O.suff_stats(x, labels, sub, K)
        np.testing.assert_array_equal(want[0], cnt)
        np.testing.assert_allclose(want[2], S, atol=1e-6 * (np.abs(S).max() + 1), rtol=1e-6)
    ck.release()
    fresh.release()

"""The allocation-free entry point dpmm_merge_hastings_static, called through the C ABI.

It serves callers that cannot call cudaMalloc (device memory owned by another framework's pool or
a fixed budget; loops that cannot take cudaMalloc's implicit synchronisation): its scratch is a
file-scope device array and every buffer it touches belongs to the caller.  This file is collected
last, so a run that stops at the first failure has already run every other test; the test works
both alone in a fresh process and after the others.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _stats_layout(cnt, sm, S):
    """(K,3) counts, (K,3,D) sums, (K,3,D,D) scatter -> the device layout: 3K slots of
    (count, sum[D], S[D*D] column-major)."""
    K, _, D = sm.shape
    rows = []
    for k in range(K):
        for s in range(3):
            parts = [np.array([cnt[k, s]], np.float64), sm[k, s]]
            if S is not None:
                parts.append(S[k, s].T.reshape(-1))
            rows.append(np.concatenate(parts))
    return np.concatenate(rows)


def _run(case_seed, gauss):
    import torch
    from dpmmsubclusters_gpu_b200 import CudaKernel, lib, multinomial_hyper, niw_hyperparams, prior_type
    from dpmmsubclusters_gpu_b200.capi import check

    rng = np.random.default_rng(case_seed)
    if gauss:
        N, D, K = 12000, 6, 7
        mus = rng.normal(size=(K, D)) * 3
        z = rng.integers(0, K, size=N)
        x = mus[z] + rng.normal(size=(N, D))
        hyper = niw_hyperparams(1.0, np.zeros(D), D + 3.0, np.eye(D))
        pt = prior_type.Gaussian
    else:
        N, D, K = 6000, 30, 5
        theta = rng.dirichlet(np.ones(D) * 0.5, size=K)
        z = rng.integers(0, K, size=N)
        x = np.stack([rng.multinomial(40, theta[k]) for k in z]).astype(np.float64)
        hyper = multinomial_hyper(np.ones(D))
        pt = prior_type.Multinomial
    ck = CudaKernel(pt).init(N, x, 1, points_major=True)
    ck.set_labels((z + 1).astype(np.int32))
    ck.set_sub_labels(rng.integers(1, 3, size=N).astype(np.int32))
    ck.set_prior(hyper)
    cnt, sm, S = ck.create_sufficient_statistics(np.arange(K))
    alpha = 3.0 + case_seed
    expected = ck.merge_hastings(K, alpha)            # the context-based entry point
    ck.release()

    dev = torch.device("cuda:0")
    stats = torch.tensor(_stats_layout(cnt, sm, S), dtype=torch.float64, device=dev)
    if gauss:
        prior = torch.tensor(np.concatenate([hyper.m, hyper.psi.T.reshape(-1)]), dtype=torch.float64, device=dev)
        k0, v0 = hyper.k, hyper.v
    else:
        prior = torch.tensor(hyper.alpha, dtype=torch.float64, device=dev)
        k0, v0 = 0.0, 0.0
    out = torch.zeros(K * K, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    check(lib().dpmm_merge_hastings_static(int(pt), D, K, alpha, k0, v0, ctypes.c_void_p(prior.data_ptr()),
                                           ctypes.c_void_p(stats.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                           ctypes.c_void_p(stream.cuda_stream)))
    stream.synchronize()
    got = out.cpu().numpy().reshape(K, K)
    assert np.array_equal(np.isnan(got), np.isnan(expected))
    m = ~np.isnan(expected)
    np.testing.assert_allclose(got[m], expected[m], rtol=1e-12, atol=1e-9)
    return got


def test_static_merge_hastings_matches_context_entry_point_twice():
    # two calls in a row: the shared scratch keeps the first call's contents, and the second call
    # (other data, other K) must not depend on them
    a = _run(1, True)
    b = _run(2, True)
    assert a.shape != b.shape or not np.array_equal(np.nan_to_num(a), np.nan_to_num(b))


def test_static_merge_hastings_multinomial_twice():
    _run(3, False)
    _run(4, False)


def test_static_merge_hastings_rejects_oversize():
    import torch
    from dpmmsubclusters_gpu_b200 import lib
    buf = torch.zeros(64, dtype=torch.float64, device="cuda:0")
    p = ctypes.c_void_p(buf.data_ptr())
    st = lib().dpmm_merge_hastings_static(0, 4, 1025, 1.0, 1.0, 7.0, p, p, p, None)
    assert st == 1 and b"1024" in lib().dpmm_last_error()

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


_RESET_CHILD = r"""
import ctypes, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from dpmmsubclusters_gpu_b200 import lib
L = lib()                                   # loads libcudart.so.12 through the library's runpath
rt = ctypes.CDLL("libcudart.so.12")         # the same (already loaded) runtime instance
drv = ctypes.CDLL("libcuda.so.1")
K, D = 3, 4
rng = np.random.default_rng(5)
prior = np.concatenate([np.zeros(D), np.eye(D).reshape(-1)])
slots = []
for k in range(K):
    for s in range(3):
        x = rng.normal(size=(40 + 10 * k + s, D)) + 2.0 * k
        slots.append(np.concatenate([[x.shape[0]], x.sum(0), (x.T @ x).T.reshape(-1)]))
stats = np.concatenate(slots)

def dev(a):
    p = ctypes.c_void_p()
    assert rt.cudaMalloc(ctypes.byref(p), ctypes.c_size_t(a.nbytes)) == 0
    assert rt.cudaMemcpy(p, a.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(a.nbytes), 1) == 0
    return p

def ctx_id():
    c = ctypes.c_void_p()
    i = ctypes.c_ulonglong()
    assert drv.cuCtxGetCurrent(ctypes.byref(c)) == 0 and c.value
    assert drv.cuCtxGetId(c, ctypes.byref(i)) == 0
    return i.value

def call():
    out = np.zeros(K * K)
    dp, ds, do = dev(prior), dev(stats), dev(out)
    st = L.dpmm_merge_hastings_static(0, D, K, 2.0, 1.0, D + 3.0, dp, ds, do, None)
    assert st == 0, L.dpmm_last_error()
    assert rt.cudaDeviceSynchronize() == 0
    assert rt.cudaMemcpy(out.ctypes.data_as(ctypes.c_void_p), do, ctypes.c_size_t(out.nbytes), 2) == 0
    for p in (dp, ds, do):
        rt.cudaFree(p)
    return out

a = call()
id1 = ctx_id()
assert rt.cudaDeviceReset() == 0
z = ctypes.c_void_p()
assert rt.cudaMalloc(ctypes.byref(z), ctypes.c_size_t(256)) == 0    # a new context after the reset
rt.cudaFree(z)
if ctx_id() == id1:
    print("SAME_CONTEXT_ID")
    sys.exit(0)
b = call()
assert np.array_equal(np.isnan(a), np.isnan(b)) and np.array_equal(a[~np.isnan(a)], b[~np.isnan(b)])
assert np.isfinite(a).sum() == K * (K - 1) // 2
print("OK")
"""


def test_static_merge_hastings_after_device_reset():
    """After cudaDeviceReset the library's module is loaded anew in a new context: the entry point
    must look the scratch array's address up again (it keys its cache on the context's id) and give
    the same ratios.  Runs in a child process without torch, since the reset ends the process's
    CUDA state."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", _RESET_CHILD, root], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    if "SAME_CONTEXT_ID" in out.stdout:
        pytest.skip("the driver kept the context id across cudaDeviceReset")
    assert "OK" in out.stdout, out.stdout + out.stderr

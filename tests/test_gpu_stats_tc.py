"""Sub-cluster statistics on the tensor cores (csrc/dpmm_tc.cu k_slot_stats_tc: split-TF32 Gram
products of 32-point tiles, FP64 totals) against the FP64 oracle (oracle.suff_stats, the reference's
niw::create_sufficient_statistics per slot): counts exact, sums and scatter matrices within 1e-6
relative (of the largest entry) -- the bar of the FP32 SIMT kernel.  Data far from the origin, so
the centring at the cluster's mean parameter carries the accuracy; chunk tails of every length."""
import numpy as np
import pytest

from dpmmsubclusters_gpu_b200 import CudaKernel, LL_FP32, prior_type
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _data(seed, N, D, K, offset):
    rng = np.random.default_rng(seed)
    mus = rng.normal(size=(K, D)) * 4.0 + offset
    z = rng.integers(0, K, size=N)
    x = mus[z] + rng.normal(size=(N, D)) * rng.uniform(0.5, 2.0, size=D)
    sub = rng.integers(1, 3, size=N).astype(np.int32)
    return x, z, sub, mus


def _check(kern, x, z, sub, K):
    cnt, sm, S = kern.create_sufficient_statistics(np.arange(K))
    cnt_o, sm_o, S_o = O.suff_stats(x, (z + 1).astype(np.int32), sub, K)
    np.testing.assert_array_equal(cnt, cnt_o)
    np.testing.assert_allclose(sm, sm_o, atol=1e-6 * (np.abs(sm_o).max() + 1), rtol=1e-6)
    np.testing.assert_allclose(S, S_o, atol=1e-6 * (np.abs(S_o).max() + 1), rtol=1e-6)
    return cnt, sm, S


@pytest.mark.parametrize("D,N,K,offset", [(64, 60001, 5, 20.0), (32, 30011, 3, -50.0), (48, 9000, 4, 5.0),
                                          (20, 7000, 6, 100.0), (64, 200, 3, 0.0)])
def test_slot_statistics_match_fp64(D, N, K, offset):
    x, z, sub, mus = _data(D * 7 + N, N, D, K, offset)
    kern = CudaKernel(prior_type.Gaussian, k_max=8).init(N, x.T, seed=1)
    # the mean parameters centre the products (as in the sampler, where they are the last draw)
    rng = np.random.default_rng(1)
    kern.set_gaussian_params(mus + 0.1 * rng.normal(size=mus.shape), np.tile(np.eye(D), (K, 1, 1)),
                             np.zeros(K), np.full(K, 1.0 / K))
    kern.set_labels((z + 1).astype(np.int32))
    kern.set_sub_labels(sub)
    _check(kern, x, z, sub, K)


def test_tensor_core_and_simt_statistics_agree():
    D, N, K = 64, 40000, 4
    x, z, sub, mus = _data(5, N, D, K, 30.0)
    out = []
    for mode in (None, LL_FP32):   # LL_FP32: the SIMT kernel
        kern = CudaKernel(prior_type.Gaussian, k_max=8, loglik_mode=mode).init(N, x.T, seed=1)
        kern.set_gaussian_params(mus, np.tile(np.eye(D), (K, 1, 1)), np.zeros(K), np.full(K, 1.0 / K))
        kern.set_labels((z + 1).astype(np.int32))
        kern.set_sub_labels(sub)
        out.append(_check(kern, x, z, sub, K))
    (c0, s0, S0), (c1, s1, S1) = out
    np.testing.assert_array_equal(c0, c1)
    np.testing.assert_allclose(S0, S1, atol=2e-6 * np.abs(S1).max(), rtol=2e-6)

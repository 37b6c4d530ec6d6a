"""The multinomial label phase on the tensor cores (csrc/dpmm_tc.cu k_mult_labels_tc) through the C ABI.

r_k(x) = sum_d x_d log theta_kd (cudaKernel_multinomial.cu:60-76, no weight term) as one BF16 contraction:
counts exact in BF16, log theta as three BF16 parts (its FP32 value exactly), FP32 accumulation.
Checked against the FP64 oracle: |r - r64| <= 1e-5 * max(sum_d x_d |log theta_kd|, 1) (the FP32 sum of
exact products); labels exact against the oracle's draw on the GPU's own r except at margins below
1e-4, against its draw on FP64 r up to the margin rule of tests/parity.py; argmax labels likewise; the
same labels as the FP32 SIMT form for the same uniforms; counts that BF16 does not hold exactly fall
back to the FP32 SIMT form.
"""
import numpy as np
import pytest

import parity as P
from conftest import uniforms
from dpmmsubclusters_gpu_b200 import LL_FP32, LL_TC_BF16X3, CudaKernel, prior_type
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _data(seed, N, D, K, length=60, alpha=0.3):
    rng = np.random.default_rng(seed)
    theta = rng.dirichlet(np.ones(D) * alpha, size=K)
    z = rng.integers(0, K, size=N)
    lens = rng.poisson(length, size=N) + 1
    x = np.stack([rng.multinomial(lens[i], theta[z[i]]) for i in range(N)]).astype(np.float64)
    lt = np.log(rng.dirichlet(np.ones(D), size=K) * 0.3 + theta * 0.7)
    return x, z, lt


def _check_r(r, x, lt, tag):
    r64 = np.stack([O.mult_loglik(x, lt[k]) for k in range(lt.shape[0])], 1)
    scale = np.maximum(x @ np.abs(lt).T, 1.0)
    err = np.abs(r - r64)
    P.record(tag, abs_max=float(err.max()), rel_max=float((err / scale).max()))
    assert (err / scale).max() <= 1e-5, (err / scale).max()
    return r64, err.max(axis=1)


@pytest.mark.parametrize("D,K,N", [(20, 3, 5000), (100, 50, 12000), (1000, 50, 4000), (300, 150, 3000),
                                   (64, 2, 148 * 128 * 3 + 5)])
def test_multinomial_tensor_core_labels_parity(D, K, N):
    x, z, lt = _data(D * 7 + K, N, D, K)
    ck = CudaKernel(prior_type.Multinomial, loglik_mode=LL_TC_BF16X3, k_max=max(K, 8)).init(N, x, 3, points_major=True)
    ck.set_multinomial_params(lt)
    u = uniforms(2 * N, D + K)
    r = ck.create_clusters_labels(K, uniforms=u, return_loglik=True).astype(np.float64)
    lab = ck.get_labels()
    tag = f"mult_tc_D{D}_K{K}_N{N}"
    r64, row_err = _check_r(r, x, lt, tag)
    u2 = u.reshape(N, 2).astype(np.float64)
    lab_o, mg = O.sample_labels(r, u2)
    bad = lab != lab_o
    assert np.all(mg[bad] < 1e-4) and bad.mean() <= 1e-3, (bad.sum(), mg[bad][:5])
    P.labels_vs_fp64(lab, r64, u2, row_err, tag + "_vs_fp64")
    rf = ck.create_clusters_labels(K, bFinal=True, return_loglik=True).astype(np.float64)
    labf = ck.get_labels()
    lab_of, gap = O.sample_labels(rf, np.zeros((N, 2)), final=True)
    assert np.all((labf == lab_of) | (gap < 1e-5))
    P.labels_vs_fp64(labf, r64, np.zeros((N, 2)), row_err, tag + "_argmax_vs_fp64", final=True)


def test_multinomial_tensor_core_equals_fp32_form():
    N, D, K = 30000, 200, 40
    x, z, lt = _data(5, N, D, K)
    u = uniforms(2 * N, 17)
    out = {}
    for mode in (LL_FP32, LL_TC_BF16X3):
        ck = CudaKernel(prior_type.Multinomial, loglik_mode=mode, k_max=64).init(N, x, 3, points_major=True)
        ck.set_multinomial_params(lt)
        r = ck.create_clusters_labels(K, uniforms=u, return_loglik=True).astype(np.float64)
        out[mode] = (r, ck.get_labels())
        ck.release()
    r32, lab32 = out[LL_FP32]
    rtc, labtc = out[LL_TC_BF16X3]
    scale = np.maximum(x @ np.abs(lt).T, 1.0)
    assert (np.abs(rtc - r32) / scale).max() <= 2e-5
    assert np.mean(lab32 != labtc) <= 1e-3


def test_inexact_counts_fall_back_to_the_fp32_form():
    # counts above 256 that BF16 cannot hold: the tensor-core form is not used, the labels stay exact
    N, D, K = 4000, 30, 4
    x, z, lt = _data(9, N, D, K)
    x[::7, 0] = 257.0
    ck = CudaKernel(prior_type.Multinomial, k_max=8).init(N, x, 3, points_major=True)
    ck.set_multinomial_params(lt)
    u = uniforms(2 * N, 4)
    r = ck.create_clusters_labels(K, uniforms=u, return_loglik=True).astype(np.float64)
    r64, row_err = _check_r(r, x, lt, "mult_fallback")
    P.labels_vs_fp64(ck.get_labels(), r64, u.reshape(N, 2).astype(np.float64), row_err, "mult_fallback_vs_fp64")
    with pytest.raises(Exception):
        c2 = CudaKernel(prior_type.Multinomial, loglik_mode=LL_TC_BF16X3, k_max=8).init(N, x, 3, points_major=True)
        c2.set_multinomial_params(lt)
        c2.create_clusters_labels(K, uniforms=u)

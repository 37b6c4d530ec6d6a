"""Labels of this repository's kernels against the labels of the REFERENCE'S OWN GPU code on the same
points, cluster parameters and random stream.

oracle/_ref/ref_gpu_labels (built by oracle/Makefile from the reference's cudaKernel*.cu and host
sources, sm_100a) runs cudaKernel::create_clusters_labels (cudaKernel.cu:1400-1490: FP64 log-likelihoods,
softmax, Walker alias draw from the per-point XORWOW stream curand_init(seed, point, 0)), then
create_subclusters_labels (cudaKernel.cu:1299-1398) on the labels it drew, then the argmax labels of the
final iterations.  It runs as a child process: its init calls cudaDeviceReset (cudaKernel.cu:615).
This repository's context runs the same three phases in cuRAND-compatible mode (RNG_CURAND_XORWOW, same
seed) through the C ABI.  Labels must be identical point for point except where the FP64 decision margin
is inside what the row's log-likelihood error can move (tests/parity.py); the mismatch count is recorded.
Sub-labels are compared on the points whose cluster label agrees.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import parity as P
from conftest import ROOT
from dpmmsubclusters_gpu_b200 import LL_FP32, LL_TC_BF16X3, RNG_CURAND_XORWOW, CudaKernel, prior_type
from oracle import oracle as O

pytestmark = pytest.mark.gpu

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_labels")


def _run_reference(prior, x, K, seed, dists, w, lrw):
    """x: (N, D) points; dists: per cluster three records (cluster, l, r) of float64 arrays."""
    N, D = x.shape
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            np.array([prior, N, D, K], np.int32).tofile(f)
            np.array([seed], np.uint64).tofile(f)
            np.ascontiguousarray(x, np.float64).tofile(f)
            for rec in dists:
                for a in rec:
                    np.ascontiguousarray(a, np.float64).tofile(f)
            np.ascontiguousarray(w, np.float64).tofile(f)
            np.ascontiguousarray(lrw, np.float64).tofile(f)
        out = subprocess.run([REF_BIN, fin, fout], capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stdout + out.stderr
        res = np.fromfile(fout, np.int32).reshape(3, N)
    return res[0], res[1], res[2]


def _gauss_case(seed, N, D, K, spread):
    rng = np.random.default_rng(seed)
    mus = rng.normal(size=(K, D)) * spread
    covs = []
    z = rng.integers(0, K, size=N)
    x = np.empty((N, D))
    for k in range(K):
        A = rng.normal(size=(D, D))
        C = A @ A.T / D + 0.5 * np.eye(D)
        covs.append(C)
        idx = np.flatnonzero(z == k)
        x[idx] = rng.multivariate_normal(mus[k], C, size=idx.size)
    covs = np.array(covs)
    mu = mus + 0.3 * rng.normal(size=mus.shape)
    inv = np.linalg.inv(covs)
    ld = np.linalg.slogdet(covs)[1]
    mu_lr = mu[:, None, :] + 0.5 * rng.normal(size=(K, 2, D))
    sc = rng.uniform(0.8, 1.25, size=(K, 2))
    inv_lr = inv[:, None] * sc[:, :, None, None]
    ld_lr = ld[:, None] - D * np.log(sc)
    w = rng.dirichlet(np.ones(K) * 2)
    lrw = rng.dirichlet([2, 2], size=K)
    return x, mu, inv, ld, w, mu_lr, inv_lr, ld_lr, lrw


@pytest.mark.skipif(not os.path.exists(REF_BIN), reason="reference GPU build (oracle/_ref) not present")
@pytest.mark.parametrize("D,K,N,mode", [(2, 3, 20000, LL_FP32), (8, 6, 20000, LL_FP32), (32, 10, 12000, LL_TC_BF16X3),
                                        (64, 12, 8000, LL_TC_BF16X3), (64, 12, 8000, LL_FP32)])
def test_gaussian_labels_equal_reference_gpu(D, K, N, mode):
    seed = 1234 + D
    x, mu, inv, ld, w, mu_lr, inv_lr, ld_lr, lrw = _gauss_case(D * 10 + K, N, D, K, 4.0)
    # Eigen matrices are column-major: write inv^T so that the file holds inv column by column
    dists = [((mu[k], inv[k].T, [ld[k]]), (mu_lr[k, 0], inv_lr[k, 0].T, [ld_lr[k, 0]]),
              (mu_lr[k, 1], inv_lr[k, 1].T, [ld_lr[k, 1]])) for k in range(K)]
    dists = [tuple(a for part in rec for a in part) for rec in dists]
    lab_ref, sub_ref, fin_ref = _run_reference(0, x, K, seed, dists, w, lrw)

    def make():
        ck = CudaKernel(prior_type.Gaussian, loglik_mode=mode, rng_kind=RNG_CURAND_XORWOW, k_max=32).init(
            N, x, seed, points_major=True)
        ck.set_gaussian_params(mu, inv, ld, w, mu_lr, inv_lr, ld_lr, lrw)
        return ck
    path = "fp32" if mode == LL_FP32 else "tc"
    tag = f"refgpu_{path}_D{D}_K{K}"
    lab, sub, fin, r, rs, u_lab, u_sub = _our_phases(make, K)
    r64 = np.stack([O.gauss_loglik(x, mu[k], inv[k], ld[k], w[k]) for k in range(K)], 1)
    row_err = P.gauss_ll(r, r64, D, ld, np.log(w), path, tag)
    _, _, r64s = O.gauss_sub_labels(x, lab_ref, mu_lr, inv_lr, ld_lr, lrw, u_sub.reshape(-1).astype(np.float64))
    same = lab == lab_ref
    row_s = np.zeros(N)
    row_s[same] = P.gauss_ll(rs[same], r64s[same], D, ld_lr[lab[same] - 1], 0.0, path, tag + "_sub_ll")
    _compare(lab, sub, fin, lab_ref, sub_ref, fin_ref, r64, r64s, row_err, row_s, u_lab, u_sub, lrw, tag)


def _our_phases(make, K):
    """The three phases on this repository's kernels: once from the device's cuRAND-compatible stream
    and once with the same uniforms read out of that stream (dpmm_draw_uniforms) and passed in, so that
    the oracle can re-run each decision; both give identical labels."""
    ck = make()
    ck.create_clusters_labels(K)
    lab_dev = ck.get_labels()
    ck.create_subclusters_labels(K)
    sub_dev = ck.get_sub_labels()
    ck.release()
    gen = make()
    u_lab = gen.draw_uniforms().astype(np.float64)
    u_sub = gen.draw_uniforms().astype(np.float64)
    gen.release()
    ck = make()
    r = ck.create_clusters_labels(K, uniforms=u_lab.astype(np.float32).reshape(-1), return_loglik=True)
    lab = ck.get_labels()
    rs = ck.create_subclusters_labels(K, uniforms=u_sub.astype(np.float32).reshape(-1), return_loglik=True)
    sub = ck.get_sub_labels()
    ck.create_clusters_labels(K, bFinal=True)
    fin = ck.get_labels()
    ck.release()
    np.testing.assert_array_equal(lab, lab_dev)
    np.testing.assert_array_equal(sub, sub_dev)
    return lab, sub, fin, r.astype(np.float64), rs.astype(np.float64), u_lab, u_sub


def _compare(lab, sub, fin, lab_ref, sub_ref, fin_ref, r64, r64s, row_err, row_s, u_lab, u_sub, lrw, tag):
    N = lab.size
    # 1. the reference's own labels are the oracle's FP64 draw (its log-likelihoods differ from the
    #    oracle's only by cuBLAS rounding): this pins the oracle against the reference's GPU build
    lab64, mg = O.sample_labels(r64, u_lab)
    bad_ref = lab_ref != lab64
    assert np.all(mg[bad_ref] < 1e-9), (tag, int(bad_ref.sum()), mg[bad_ref][:5])
    # 2. ours against the reference: only inside the margin rule of the row's log-likelihood error
    bad = lab != lab_ref
    bound = 4 * r64.shape[1] * (row_err + 1e-6)
    P.record(tag, mismatches_vs_reference=int(bad.sum()), reference_vs_oracle=int(bad_ref.sum()), points=N)
    assert np.all(mg[bad] < bound[bad]), (tag, int(bad.sum()), mg[bad][:5], bound[bad][:5])
    # 3. argmax: only gaps inside twice the row error
    badf = np.flatnonzero(fin != fin_ref)
    gap = np.abs(r64[badf, fin[badf] - 1] - r64[badf, fin_ref[badf] - 1])
    P.record(tag + "_argmax", mismatches_vs_reference=int(badf.size), points=N)
    assert np.all(gap <= 2 * row_err[badf] + 1e-9), (tag, gap[:5])
    # 4. sub-labels where the cluster labels agree: the 2-way draw with the same uniforms
    same = np.flatnonzero(lab == lab_ref)
    sub64 = np.zeros(N, np.int32)
    mgs = np.full(N, np.inf)
    for k in range(lrw.shape[0]):
        idx = same[lab[same] == k + 1]
        if idx.size:
            sub64[idx], mgs[idx] = O.sample_sub_from_loglik(r64s[idx], lrw[k], u_sub[idx])
    bad_sref = sub_ref[same] != sub64[same]
    assert np.all(mgs[same][bad_sref] < 1e-9), (tag, int(bad_sref.sum()))
    bad_s = sub[same] != sub_ref[same]
    bound_s = 8 * (row_s[same] + 1e-6)
    P.record(tag + "_sub", mismatches_vs_reference=int(bad_s.sum()), points=int(same.size))
    assert np.all(mgs[same][bad_s] < bound_s[bad_s]), (tag, int(bad_s.sum()))


@pytest.mark.skipif(not os.path.exists(REF_BIN), reason="reference GPU build (oracle/_ref) not present")
@pytest.mark.parametrize("D,K,N", [(20, 4, 10000), (300, 8, 4000)])
def test_multinomial_labels_equal_reference_gpu(D, K, N):
    rng = np.random.default_rng(D + K)
    theta = rng.dirichlet(np.ones(D) * 0.3, size=K)
    z = rng.integers(0, K, size=N)
    x = np.stack([rng.multinomial(rng.poisson(40) + 1, theta[k]) for k in z]).astype(np.float64)
    lt = np.log(theta * 0.9 + 0.1 / D)
    lt_lr = np.log(rng.dirichlet(np.ones(D), size=(K, 2)) * 0.3 + theta[:, None] * 0.7)
    lrw = rng.dirichlet([3, 3], size=K)
    w = np.full(K, 1.0 / K)
    seed = 77 + D
    dists = [(lt[k], lt_lr[k, 0], lt_lr[k, 1]) for k in range(K)]
    lab_ref, sub_ref, fin_ref = _run_reference(1, x, K, seed, dists, w, lrw)

    def make():
        ck = CudaKernel(prior_type.Multinomial, rng_kind=RNG_CURAND_XORWOW, k_max=16).init(N, x, seed,
                                                                                          points_major=True)
        ck.set_multinomial_params(lt, None, lt_lr, lrw)
        return ck
    lab, sub, fin, r, rs, u_lab, u_sub = _our_phases(make, K)
    r64 = np.stack([O.mult_loglik(x, lt[k]) for k in range(K)], 1)
    row_err = np.abs(r - r64).max(1)
    assert (row_err / np.maximum(np.abs(r64).max(1), 1)).max() <= 1e-5
    _, _, r64s = O.mult_sub_labels(x, lab_ref, lt_lr, lrw, u_sub.reshape(-1))
    row_s = np.abs(rs - r64s).max(1)
    row_s[~np.isfinite(row_s)] = 0
    _compare(lab, sub, fin, lab_ref, sub_ref, fin_ref, r64, r64s, row_err, row_s, u_lab, u_sub, lrw,
             f"refgpu_mult_D{D}_K{K}")

"""The pruned label phase (dpmm_set_label_pruning; csrc/dpmm_kernels.cu k_prune_*) against the dense
phase with the same parameters and caller uniforms.  Left-out clusters are provably more than the
margin (30 nats) below each point's own cluster, so both draw the same label unless a uniform falls
inside < K e^-30 of probability: the labels must be identical.  A state the bound cannot prune (random
current labels) falls back to the dense phase."""
import ctypes

import numpy as np
import pytest

import parity as P
from conftest import uniforms
from oracle import oracle as O
from dpmmsubclusters_gpu_b200 import RNG_CURAND_XORWOW, CudaKernel, LL_FP32, prior_type
from dpmmsubclusters_gpu_b200.capi import check, lib

pytestmark = pytest.mark.gpu


def _mixture(seed, N, D, K, spread):
    rng = np.random.default_rng(seed)
    mus = rng.normal(size=(K, D)) * spread
    covs = []
    z = rng.integers(0, K, size=N)
    x = np.empty((N, D))
    for c in range(K):
        A = rng.normal(size=(D, D))
        C = A @ A.T / D + 0.5 * np.eye(D)
        covs.append(C)
        idx = np.flatnonzero(z == c)
        x[idx] = rng.multivariate_normal(mus[c], C, size=idx.size)
    return x, z, mus, np.array(covs), rng


def _stats(kern):
    out = (ctypes.c_double * 6)()
    check(lib().dpmm_label_pruning_stats(kern.ctx, out))
    return list(out)


# D = 32 / 64 in the default mode: the scan runs on the tensor cores; D = 16 and FP32 mode: SIMT
@pytest.mark.parametrize("D,mode", [(16, None), (64, None), (32, None), (32, LL_FP32)])
def test_pruned_labels_equal_dense_labels(D, mode):
    K, N = 10, 60000
    x, z, mus, covs, rng = _mixture(D, N, D, K, 6.0)
    kern = CudaKernel(prior_type.Gaussian, k_max=16, loglik_mode=mode).init(N, x.T, seed=1)
    mu = mus + 0.05 * rng.normal(size=mus.shape)
    inv = np.array([np.linalg.inv(c) for c in covs])
    ld = np.array([np.linalg.slogdet(c)[1] for c in covs])
    w = rng.dirichlet(np.ones(K) * 3)
    kern.set_gaussian_params(mu, inv, ld, w)
    u = uniforms(2 * N, 5)
    res = {}
    for margin in (30.0, 0.0):
        check(lib().dpmm_set_label_pruning(kern.ctx, margin))
        for final in (False, True):
            kern.set_labels((z + 1).astype(np.int32))
            kern.create_clusters_labels(K, final, None if final else u)
            res[(margin, final)] = kern.get_labels()
    st = _stats(kern)
    assert st[1] == 2, st          # both pruned phases ran pruned
    for final in (False, True):
        np.testing.assert_array_equal(res[(30.0, final)], res[(0.0, final)])
    # and against the oracle's draw on FP64 log-likelihoods (margin rule of tests/parity.py) on a sample
    sel = np.arange(0, N, 5)
    r64 = np.stack([O.gauss_loglik(x[sel], mu[k], inv[k], ld[k], w[k]) for k in range(K)], 1)
    kern.set_labels((z + 1).astype(np.int32))
    r = kern.create_clusters_labels(K, False, u, return_loglik=True)
    path = "fp32" if mode == LL_FP32 or D < 32 else "tc"
    row_err = P.gauss_ll(r[sel], r64, D, ld, np.log(w), path, f"prune_dense_{path}_D{D}")
    u2 = u.reshape(N, 2).astype(np.float64)
    P.labels_vs_fp64(res[(30.0, False)][sel], r64, u2[sel], row_err, f"prune_{path}_D{D}_vs_fp64")
    P.labels_vs_fp64(res[(30.0, True)][sel], r64, u2[sel], row_err, f"prune_argmax_{path}_D{D}_vs_fp64",
                     final=True)


def test_dense_phase_chosen_where_it_costs_less():
    # tensor-core dense phase (D = 64): no attempt below 8 clusters (the scan alone costs more).  At 12
    # heavily overlapping clusters the points keep most other clusters, far more than 12 / 30 per
    # point, so the attempt falls back to the dense phase.  Labels equal the dense phase's either way.
    N, D = 60000, 64
    for K, spread, tried, used in ((4, 6.0, 0, 0), (12, 0.3, 1, 0)):
        x, z, mus, covs, rng = _mixture(29 + K, N, D, K, spread)
        kern = CudaKernel(prior_type.Gaussian, k_max=16).init(N, x.T, seed=1)
        kern.set_gaussian_params(mus, np.array([np.linalg.inv(c) for c in covs]),
                                 np.array([np.linalg.slogdet(c)[1] for c in covs]), np.full(K, 1.0 / K))
        u = uniforms(2 * N, 11)
        lab = {}
        for margin in (30.0, 0.0):
            check(lib().dpmm_set_label_pruning(kern.ctx, margin))
            kern.set_labels((z + 1).astype(np.int32))
            kern.create_clusters_labels(K, False, u)
            lab[margin] = kern.get_labels()
        st = _stats(kern)
        assert st[0] == tried and st[1] == used, (K, st)
        if tried:
            assert st[4] > K / 30.0, st
        np.testing.assert_array_equal(lab[30.0], lab[0.0])
        kern.release()


def test_unprunable_state_falls_back_to_dense():
    K, N, D = 6, 30000, 8
    x, z, mus, covs, rng = _mixture(3, N, D, K, 0.5)    # overlapping clusters
    kern = CudaKernel(prior_type.Gaussian, k_max=16).init(N, x.T, seed=1)
    kern.set_gaussian_params(mus, np.array([np.linalg.inv(c) for c in covs]),
                             np.array([np.linalg.slogdet(c)[1] for c in covs]), np.full(K, 1.0 / K))
    u = uniforms(2 * N, 7)
    lab = {}
    for margin in (30.0, 0.0):
        check(lib().dpmm_set_label_pruning(kern.ctx, margin))
        kern.set_labels(rng.integers(1, K + 1, size=N).astype(np.int32))
        kern.create_clusters_labels(K, False, u)
        lab[margin] = kern.get_labels()
    st = _stats(kern)
    assert st[0] == 1 and st[1] == 0, st
    np.testing.assert_array_equal(lab[30.0], lab[0.0])


@pytest.mark.parametrize("K,N,D,planted", [(30, 200000, 8, 3000), (60, 200000, 64, 1500), (150, 150000, 32, 600),
                                           (200, 200000, 32, 500)])
def test_chunk_over_capacity_is_evaluated_against_every_cluster(K, N, D, planted):
    # separated clusters; points drawn from all of them carry label 1, so the chunk(s) of cluster 0
    # keep more than 16 clusters: those points get every cluster, the rest stay pruned.  At D = 32 / 64
    # the scan runs on the tensor cores: in one pass up to 193 clusters (150: two B tiles), in two
    # passes above (200: the chunk bound first, then more than 128 candidates in two tiles).  With the
    # tensor-core dense phase the pruned one is kept while fewer than K / 30 other clusters per point
    # are kept: cluster 1's chunks (all of them over capacity) hold under N / 30 points.
    x, z, mus, covs, rng = _mixture(17, N, D, K, 8.0)
    kern = CudaKernel(prior_type.Gaussian, k_max=K + 2).init(N, x.T, seed=1)
    kern.set_gaussian_params(mus, np.array([np.linalg.inv(c) for c in covs]),
                             np.array([np.linalg.slogdet(c)[1] for c in covs]), np.full(K, 1.0 / K))
    cur = (z + 1).astype(np.int32)
    cur[rng.choice(N, planted, replace=False)] = 1
    u = uniforms(2 * N, 9)
    lab = {}
    for margin in (30.0, 0.0):
        check(lib().dpmm_set_label_pruning(kern.ctx, margin))
        kern.set_labels(cur)
        kern.create_clusters_labels(K, False, u)
        lab[margin] = kern.get_labels()
    st = _stats(kern)
    assert st[1] == 1 and st[5] >= 1, st
    np.testing.assert_array_equal(lab[30.0], lab[0.0])


def test_stateful_stream_stays_in_step_with_the_dense_phase():
    # cuRAND XORWOW keeps one generator state per point: a pruned phase that settles a point without
    # drawing must still advance it, or the next draws differ from the dense phase's.  Phase 1:
    # separated clusters (every point settled without a draw); phase 2: clusters 0 and 1 made
    # identical, so their points draw 50 / 50 from the advanced states.
    K, N, D = 8, 40000, 16
    x, z, mus, covs, rng = _mixture(23, N, D, K, 6.0)
    inv = np.array([np.linalg.inv(c) for c in covs])
    ld = np.array([np.linalg.slogdet(c)[1] for c in covs])
    mus2, inv2, ld2 = mus.copy(), inv.copy(), ld.copy()
    mus2[1], inv2[1], ld2[1] = mus[0], inv[0], ld[0]
    lab = {}
    for margin in (30.0, 0.0):
        kern = CudaKernel(prior_type.Gaussian, k_max=16, rng_kind=RNG_CURAND_XORWOW).init(N, x.T, seed=3)
        check(lib().dpmm_set_label_pruning(kern.ctx, margin))
        out = []
        for m, iv, l in ((mus, inv, ld), (mus2, inv2, ld2)):
            kern.set_gaussian_params(m, iv, l, np.full(K, 1.0 / K))
            kern.set_labels((z + 1).astype(np.int32))
            kern.create_clusters_labels(K, False, None)
            out.append(kern.get_labels())
        lab[margin] = out
        if margin > 0:
            assert _stats(kern)[1] == 2
    for a, b in zip(lab[30.0], lab[0.0]):
        np.testing.assert_array_equal(a, b)
    moved = (lab[0.0][1] == 2) & (z == 0)
    assert moved.sum() > 1000   # the second phase does draw between clusters 0 and 1

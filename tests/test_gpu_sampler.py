"""Whole-sampler runs through the reference-facing API (dp_parallel_sampling_class) on the GPU:
recovery of the true clusters on synthetic data of the reference's configurations' shapes,
the params-JSON path, and run-to-run determinism."""
import json

import numpy as np
import pytest

from dpmmsubclusters_gpu_b200 import (LL_FP32, dp_parallel_sampling_class, multinomial_hyper, niw_hyperparams,
                                      prior_type)

pytestmark = pytest.mark.gpu


def nmi(a, b):
    a = np.asarray(a); b = np.asarray(b)
    ua, ia = np.unique(a, return_inverse=True)
    ub, ib = np.unique(b, return_inverse=True)
    c = np.zeros((ua.size, ub.size))
    np.add.at(c, (ia, ib), 1)
    p = c / c.sum()
    pa, pb = p.sum(1), p.sum(0)
    h = lambda q: -np.sum(q[q > 0] * np.log(q[q > 0]))
    nz = p > 0
    mi = np.sum(p[nz] * np.log(p[nz] / np.outer(pa, pb)[nz]))
    return 2 * mi / (h(pa) + h(pb))


def gmm(rng, N, D, K, mean_range, cov_scale):
    mus = rng.uniform(-mean_range, mean_range, size=(K, D))
    z = rng.integers(0, K, size=N)
    x = np.empty((N, D))
    for k in range(K):
        A = rng.normal(size=(D, D))
        cov = A @ A.T * cov_scale + (0.5 if cov_scale < 1 else 1.0) * np.eye(D)
        idx = np.where(z == k)[0]
        x[idx] = rng.multivariate_normal(mus[k], cov, size=idx.size)
    return x, z


def test_gaussian_c1_shape_recovers_two_clusters():
    # shape of the first configuration: N=1e5, D=2, 2 true clusters, means U(-100,100), cov AA^T + I
    rng = np.random.default_rng(12345)
    x, z = gmm(rng, 100000, 2, 2, 100.0, 1.0)
    dps = dp_parallel_sampling_class(100000, x.T, 12345, prior_type.Gaussian)
    mi = dps.dp_parallel(niw_hyperparams(1.0, np.zeros(2), 5.0, np.eye(2)), 1.0, iters=100, verbose=False, burnout=15)
    assert len(np.unique(mi.labels)) == 2
    assert nmi(mi.labels, z) > 0.99
    assert mi.iter_count.size == 100 and mi.weights.size == 2
    assert mi.cluster_count_history[-1] == 2


def test_gaussian_d8_many_clusters():
    rng = np.random.default_rng(3)
    x, z = gmm(rng, 60000, 8, 6, 20.0, 1.0 / 8)
    dps = dp_parallel_sampling_class(60000, x.T, 7, prior_type.Gaussian)
    mi = dps.dp_parallel(niw_hyperparams(1.0, np.zeros(8), 11.0, np.eye(8)), 10.0, iters=120, verbose=False,
                         burnout=15, gt=z + 1)
    assert nmi(mi.labels, z) > 0.95
    assert abs(len(np.unique(mi.labels)) - 6) <= 1


def test_plain_fp32_form_matches_quality():
    rng = np.random.default_rng(4)
    x, z = gmm(rng, 40000, 4, 4, 20.0, 0.25)
    dps = dp_parallel_sampling_class(40000, x.T, 9, prior_type.Gaussian, loglik_mode=LL_FP32)
    mi = dps.dp_parallel(niw_hyperparams(1.0, np.zeros(4), 7.0, np.eye(4)), 10.0, iters=80, verbose=False)
    assert nmi(mi.labels, z) > 0.95


def test_multinomial_recovers_components():
    rng = np.random.default_rng(5)
    N, D, K = 30000, 100, 5
    theta = rng.dirichlet(np.ones(D) * 0.1, size=K)
    z = rng.integers(0, K, size=N)
    x = np.stack([rng.multinomial(200, theta[k]) for k in z]).astype(np.float64)
    dps = dp_parallel_sampling_class(N, x.T, 11, prior_type.Multinomial)
    mi = dps.dp_parallel(multinomial_hyper(np.ones(D)), 10.0, iters=60, verbose=False, burnout=15)
    assert nmi(mi.labels, z) > 0.95


def test_deterministic_for_a_seed():
    rng = np.random.default_rng(6)
    x, z = gmm(rng, 20000, 3, 3, 15.0, 0.3)
    out = []
    for _ in range(2):
        dps = dp_parallel_sampling_class(20000, x.T, 321, prior_type.Gaussian)
        out.append(dps.dp_parallel(niw_hyperparams(1.0, np.zeros(3), 6.0, np.eye(3)), 10.0, iters=40, verbose=False))
    np.testing.assert_array_equal(out[0].labels, out[1].labels)
    np.testing.assert_array_equal(out[0].cluster_count_history, out[1].cluster_count_history)


def test_params_json_and_npy_path(tmp_path):
    # the --params_path / --model_path route (dp_parallel_from_file), with // comments, an outlier
    # cluster (ModuleTestFile2.json-like) and float32 npy data
    rng = np.random.default_rng(8)
    x, z = gmm(rng, 20000, 2, 3, 30.0, 1.0)
    npy = tmp_path / "data.npy"
    np.save(npy, x.astype(np.float32))
    params = tmp_path / "params.json"
    params.write_text("""{
  "iterations": 60,
  "initial_clusters": 1,
  "alpha": 10.0,
  "use_verbose": false,
  "burnout_period": 15,
  "max_num_of_clusters": 1000000000,
  "hyper_params": {
    //Example for niw
    "m": [0.0, 0.0],
    "psi": [[1.0, 0.0], [0.0, 1.0]],
    "k": 1,
    "v": 5.0
  },
  "outlier_mod": 0.05,
  "randomSeed": 17
}
""")
    res = tmp_path / "result.json"
    dps = dp_parallel_sampling_class(str(npy), str(params), prior_type.Gaussian)
    mi = dps.dp_parallel_from_file(str(res))
    out = json.loads(res.read_text())
    assert len(out["labels"]) == 20000 and len(out["iter_count"]) == 60
    assert np.array_equal(np.array(out["labels"]), mi.labels)
    inliers = mi.labels != 1
    assert nmi(mi.labels[inliers], z[inliers]) > 0.9

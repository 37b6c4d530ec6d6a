"""Whole-sampler runs through the reference-facing API (dp_parallel_sampling_class) on the GPU:
recovery of the true clusters on synthetic data of the reference's configurations' shapes,
the params-JSON path, and run-to-run determinism."""
import json
import os

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
    # shape of the first configuration: N=1e5, D=2, 2 true clusters, means U(-100,100), cov AA^T + I,
    # alpha = 1.  The sampler is stochastic: like the reference's own end-to-end tests
    # (test/module_tests_test.cpp:48-93 retry up to 3 times) the check is over three seeds.
    rng = np.random.default_rng(12345)
    x, z = gmm(rng, 100000, 2, 2, 100.0, 1.0)
    found = 0
    for seed in (1, 2, 3):
        dps = dp_parallel_sampling_class(100000, x.T, seed, prior_type.Gaussian)
        mi = dps.dp_parallel(niw_hyperparams(1.0, np.zeros(2), 5.0, np.eye(2)), 1.0, iters=100, verbose=False,
                             burnout=15)
        assert mi.iter_count.size == 100 and mi.weights.size == mi.cluster_count_history[-1]
        found += len(np.unique(mi.labels)) == 2 and nmi(mi.labels, z) > 0.99
    assert found >= 2


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
    # with an outlier cluster and one initial cluster, cluster 1 keeps its first (prior) draw for the
    # whole run (local_clusters_actions.cpp:348-351), so whether a run separates all three clusters
    # depends on the seed: the check is that some run separates at least two of them
    best = 0.0
    for seed in (17, 18, 19, 20):
        params = tmp_path / f"params{seed}.json"
        params.write_text("""{
  "iterations": 100,
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
  "randomSeed": %d
}
""" % seed)
        res = tmp_path / f"result{seed}.json"
        dps = dp_parallel_sampling_class(str(npy), str(params), prior_type.Gaussian)
        mi = dps.dp_parallel_from_file(str(res))
        out = json.loads(res.read_text())
        assert len(out["labels"]) == 20000 and len(out["iter_count"]) == 100
        assert np.array_equal(np.array(out["labels"]), mi.labels)
        assert len(out["weights"]) == len(mi.weights)
        inliers = mi.labels != 1
        if len(np.unique(mi.labels[inliers])) > 1:
            best = max(best, nmi(mi.labels[inliers], z[inliers]))
    assert best > 0.7


REF_EXE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "dpmm_ref")


@pytest.mark.skipif(not os.path.exists(REF_EXE), reason="reference executable not built (make -C oracle ref)")
def test_statistical_parity_with_reference_executable(tmp_path):
    """Final K and NMI over seeds: this library against the reference's own executable on the same
    npy + params JSON (the reference cannot be matched draw for draw: its inverse-Wishart draw is
    seeded from std::random_device)."""
    import subprocess
    rng = np.random.default_rng(11)
    x, z = gmm(rng, 20000, 2, 5, 60.0, 1.0)
    npy = tmp_path / "d.npy"
    np.save(npy, x)
    ks_ref, ks_our, nmi_ref, nmi_our = [], [], [], []
    for seed in (1, 2, 3):
        pj = tmp_path / f"p{seed}.json"
        pj.write_text(json.dumps({"alpha": 100000.0, "iterations": 80, "burnout_period": 15, "outlier_mod": 0.0,
                                  "randomSeed": seed, "initial_clusters": 1,
                                  "hyper_params": {"k": 1.0, "m": [0.0, 0.0], "v": 5.0,
                                                   "psi": [[1.0, 0.0], [0.0, 1.0]]}}))
        rj = tmp_path / f"r{seed}.json"
        p = subprocess.run(["timeout", "300", REF_EXE, f"--model_path={npy}", f"--params_path={pj}",
                            "--prior_type=Gaussian", f"--result_path={rj}"], capture_output=True, text=True)
        assert p.returncode == 0, p.stdout[-500:] + p.stderr[-500:]
        lab = np.array(json.loads(rj.read_text())["labels"])
        ks_ref.append(len(np.unique(lab)))
        nmi_ref.append(nmi(lab, z))
        mi = dp_parallel_sampling_class(str(npy), str(pj), prior_type.Gaussian).dp_parallel_from_file()
        ks_our.append(len(np.unique(mi.labels)))
        nmi_our.append(nmi(mi.labels, z))
    assert abs(np.mean(ks_ref) - np.mean(ks_our)) <= 1.5, (ks_ref, ks_our)
    # one-sided: the reference's own runs vary from run to run (unseeded draws); ours must not be worse
    assert np.mean(nmi_our) >= np.mean(nmi_ref) - 0.1, (nmi_ref, nmi_our)

"""Batches of samplers (dpmm_batch_*): many uneven data sets advanced together, the label phase of a
padded dimension as one launch replayed from a CUDA graph.  Each data set's run performs the same
operations as running it alone with the FP32 label kernel (per-point arithmetic does not depend on
the block size; random streams are per data set), so labels and weights must be identical."""
import numpy as np
import pytest

from dpmmsubclusters_gpu_b200 import BatchSampler, capi, niw_hyperparams, prior_type
from dpmmsubclusters_gpu_b200.api import dp_parallel_sampling_class

pytestmark = pytest.mark.gpu


def _data_set(rng, N, D, K):
    mus = rng.uniform(-10, 10, size=(K, D))
    z = rng.integers(0, K, size=N)
    x = np.empty((N, D))
    for c in range(K):
        A = rng.normal(size=(D, D))
        idx = np.flatnonzero(z == c)
        x[idx] = rng.multivariate_normal(mus[c], A @ A.T / D + 0.5 * np.eye(D), size=idx.size)
    return x.T.copy(), z


def test_batch_equals_separate_runs():
    rng = np.random.default_rng(77)
    shapes = [(3000, 2, 3), (9000, 8, 4), (2500, 16, 5), (12000, 2, 6), (4000, 8, 2), (7000, 16, 3), (5000, 64, 4),
              (1500, 8, 2)]
    data = [_data_set(rng, *s) for s in shapes]
    iters = 30
    hyp = [niw_hyperparams(1.0, np.zeros(s[1]), s[1] + 3.0, np.eye(s[1])) for s in shapes]
    b = BatchSampler([x for x, _ in data], hyp, 5.0, iters=iters, init_clusters=1, burnout=5, k_max=32)
    b.step(iters)
    info = b.info()
    assert info["data_sets"] == len(shapes) and info["groups"] == 4, info
    assert info["graph_launches"] > 0 and all(v in (32, 64, 128) for v in info["block_size_by_padded_dim"].values())
    for i, (x, z) in enumerate(data):
        mb = b.model_info(i)
        s = dp_parallel_sampling_class(x.shape[1], x, 1 + i, prior_type.Gaussian, loglik_mode=capi.LL_FP32, k_max=32)
        ms = s.dp_parallel(hyp[i], 5.0, iters=iters, init_clusters=1, verbose=False, burnout=5)
        np.testing.assert_array_equal(mb.labels, ms.labels)
        np.testing.assert_array_equal(mb.weights, ms.weights)
        np.testing.assert_array_equal(mb.cluster_count_history, ms.cluster_count_history)
    b.close()

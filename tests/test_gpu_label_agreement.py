"""Verbose-mode label agreement on the device (dpmm_set_ground_truth / dpmm_label_agreement): the
(label, class) contingency table is counted by a kernel and only it is copied back; NMI and VI must
equal scikit-learn's / numpy's on the downloaded labels.  The sampler's verbose NMI history
(dp_parallel_sampling.cpp:161-179) comes from the same call."""
import numpy as np
import pytest
from sklearn.metrics import normalized_mutual_info_score

from dpmmsubclusters_gpu_b200 import CudaKernel, niw_hyperparams, prior_type
from dpmmsubclusters_gpu_b200.api import dp_parallel_sampling_class

pytestmark = pytest.mark.gpu


# the last case exceeds the shared-memory table (global atomics)
@pytest.mark.parametrize("N,K,G", [(100000, 12, 9), (30011, 200, 3), (20000, 200, 100)])
def test_device_nmi_matches_sklearn(N, K, G):
    rng = np.random.default_rng(N + K)
    x = rng.normal(size=(N, 4))
    kern = CudaKernel(prior_type.Gaussian, k_max=256).init(N, x.T, seed=1)
    gt = rng.integers(0, G, size=N) * 7 - 3          # arbitrary class values
    kern.set_ground_truth(gt)
    for rep in range(2):
        lab = np.where(rng.random(N) < 0.6, (gt + 3) // 7 % K, rng.integers(0, K, size=N)) + 1
        kern.set_labels(lab.astype(np.int32))
        nmi, vi = kern.label_agreement(K)
        assert abs(nmi - normalized_mutual_info_score(gt, kern.get_labels())) <= 1e-12, rep
        assert vi >= 0


def test_sampler_verbose_history_uses_device_scores():
    rng = np.random.default_rng(5)
    N, D, K = 50000, 4, 5
    mus = rng.normal(size=(K, D)) * 10
    z = rng.integers(0, K, size=N)
    x = mus[z] + rng.normal(size=(N, D))
    dps = dp_parallel_sampling_class(N, x.T, 3, prior_type.Gaussian)
    mi = dps.dp_parallel(niw_hyperparams(1.0, np.zeros(D), D + 3.0, np.eye(D)), 10.0, iters=30, verbose=True,
                         burnout=5, gt=z + 1)
    hist = np.asarray(mi.nmi_score_history)
    assert hist.size == 30
    assert abs(hist[-1] - normalized_mutual_info_score(z, mi.labels)) <= 1e-12
    assert np.all((hist >= 0) & (hist <= 1 + 1e-12))

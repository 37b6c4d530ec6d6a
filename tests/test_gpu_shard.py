"""The data-parallel sampler (dpmm_sampler_create_sharded) against one sampler over all the points.

Two shards of one data set run as two samplers on this GPU, each driven by its own host thread and
exchanging their statistics through LocalGroupExchange (host-side sums in rank order; the samplers'
kernels never wait on each other, only the host threads do).  The ranks must hold the same run bit for
bit (cluster counts, weights, log posterior: every decision is replicated from the summed statistics),
and with the same seed the run must reach the single sampler's clustering (see _compare for why equal
outcome, not equal trajectories, is the criterion).
"""
import threading

import numpy as np
import pytest

import parity as P
from dpmmsubclusters_gpu_b200 import LL_FP32, capi, dp_parallel_sampling_class, multinomial_hyper, niw_hyperparams
from dpmmsubclusters_gpu_b200 import prior_type
from dpmmsubclusters_gpu_b200.shard import LocalGroupExchange, ShardedSampler, shard_bounds

pytestmark = pytest.mark.gpu


def _gauss(seed, N, D, K, spread):
    rng = np.random.default_rng(seed)
    mus = rng.normal(size=(K, D)) * spread
    z = rng.integers(0, K, size=N)
    x = np.empty((N, D))
    for k in range(K):
        A = rng.normal(size=(D, D))
        idx = np.flatnonzero(z == k)
        x[idx] = rng.multivariate_normal(mus[k], A @ A.T / D + 0.5 * np.eye(D), size=idx.size)
    return x, z


def _run(x, prior, hyper, world, iters, seed, gt=None, **kw):
    N, D = x.shape
    spc = dp_parallel_sampling_class(N, x.T, seed, prior, **kw)
    out = [None] * world
    errs = []
    group = LocalGroupExchange(world) if world > 1 else None

    def rank(r):
        try:
            off, n = shard_bounds(N, world, r)
            g = None if gt is None else np.ascontiguousarray(gt[off:off + n], np.int32)
            rd, keep = spc.run_desc(hyper, 10.0, iters=iters, init_clusters=1, verbose=gt is not None, burnout=15,
                                    gt=g)
            s = ShardedSampler(rd, np.ascontiguousarray(x[off:off + n]), n, D, off, N, r, world,
                               group.ranks[r] if group else None, keep=keep)
            s.step(iters)
            out[r] = s.model_info()
            s.close()
        except Exception as e:      # pragma: no cover - reported below
            errs.append(e)
            if group:
                group._barrier.abort()

    th = [threading.Thread(target=rank, args=(r,)) for r in range(world)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=600)
    assert not errs, errs
    return out


def _nmi(a, b):
    from sklearn.metrics import normalized_mutual_info_score
    return normalized_mutual_info_score(a, b)


def _compare(single, shards, tag, z=None):
    """Every rank must hold the same run (the replicated decisions are the point of the design): the same
    cluster count after every iteration, the same weights, bit for bit.  Against the single sampler the
    run agrees in outcome: the statistics are summed in another order, so the FP64 sums -- and through the
    parameter draws every later decision -- may differ in the last bits and the trajectories of this
    chaotic sampler may part after some iterations; the final clustering must agree (NMI between the two
    label sets, the same final cluster count within one, NMI against the generating labels within 0.01)."""
    for s in shards[1:]:
        np.testing.assert_array_equal(s.cluster_count_history, shards[0].cluster_count_history)
        np.testing.assert_array_equal(s.weights, shards[0].weights)
        np.testing.assert_array_equal(s.likelihood_history, shards[0].likelihood_history)
    k1, ks = single[0].cluster_count_history, shards[0].cluster_count_history
    same_until = int(np.argmax(k1 != ks)) if np.any(k1 != ks) else len(k1)
    lab_sh = np.concatenate([s.labels for s in shards])
    agree = _nmi(lab_sh, single[0].labels)
    rec = dict(final_clusters_single=int(k1[-1]), final_clusters_sharded=int(ks[-1]),
               count_history_equal_through_iteration=same_until, nmi_between_runs=float(agree),
               label_mismatches=int((lab_sh != single[0].labels).sum()))
    if z is not None:
        rec["nmi_vs_truth_single"] = float(_nmi(z, single[0].labels))
        rec["nmi_vs_truth_sharded"] = float(_nmi(z, lab_sh))
    P.record(tag, **rec)
    assert abs(int(k1[-1]) - int(ks[-1])) <= 1, rec
    assert agree >= 0.95, rec
    if z is not None:
        assert abs(rec["nmi_vs_truth_single"] - rec["nmi_vs_truth_sharded"]) <= 0.01, rec


@pytest.mark.parametrize("D,mode", [(8, None), (32, None), (32, LL_FP32)])
def test_sharded_gaussian_run_equals_single_run(D, mode):
    N, K, iters = 60000, 6, 60
    x, z = _gauss(100 + D, N, D, K, 6.0)
    hyper = niw_hyperparams(1.0, np.zeros(D), D + 3.0, np.eye(D))
    kw = {} if mode is None else {"loglik_mode": mode}
    single = _run(x, prior_type.Gaussian, hyper, 1, iters, 11, **kw)
    shards = _run(x, prior_type.Gaussian, hyper, 2, iters, 11, **kw)
    assert single[0].cluster_count_history[-1] >= K // 2        # the run did split
    _compare(single, shards, f"shard_gauss_D{D}_{'fp32' if mode == LL_FP32 else 'auto'}", z)


def test_sharded_multinomial_run_equals_single_run():
    rng = np.random.default_rng(3)
    N, D, K, iters = 20000, 40, 4, 50
    theta = rng.dirichlet(np.ones(D) * 0.2, size=K)
    z = rng.integers(0, K, size=N)
    x = np.stack([rng.multinomial(60, theta[k]) for k in z]).astype(np.float64)
    hyper = multinomial_hyper(np.ones(D))
    single = _run(x, prior_type.Multinomial, hyper, 1, iters, 5)
    shards = _run(x, prior_type.Multinomial, hyper, 2, iters, 5)
    _compare(single, shards, "shard_mult_D40", z)


def test_sharded_verbose_scores_the_whole_data_set():
    # verbose mode with a ground truth: the NMI history comes from the contingency table summed over the
    # shards, so each shard reports the whole data set's score, equal to the single run's
    N, D, K, iters = 30000, 4, 5, 40
    x, z = _gauss(9, N, D, K, 8.0)
    hyper = niw_hyperparams(1.0, np.zeros(D), D + 3.0, np.eye(D))
    single = _run(x, prior_type.Gaussian, hyper, 1, iters, 21, gt=z)
    shards = _run(x, prior_type.Gaussian, hyper, 2, iters, 21, gt=z)
    _compare(single, shards, "shard_verbose", z)
    # the NMI each rank reports comes from the contingency table summed over the shards: it is the whole
    # data set's score, the one scikit-learn gives for all the labels together
    np.testing.assert_array_equal(shards[0].nmi_score_history, shards[1].nmi_score_history)
    lab_sh = np.concatenate([s.labels for s in shards])
    assert abs(shards[0].nmi_score_history[-1] - _nmi(z, lab_sh)) <= 1e-9

"""The data-parallel sampler (dpmm_sampler_create_sharded) against one sampler over all the points.

Two shards of one data set run as two samplers on this GPU, each driven by its own host thread and
exchanging their statistics through LocalGroupExchange (host-side sums in rank order; the samplers'
kernels never wait on each other, only the host threads do).  With the same seed, the sharded run
must take the same split / merge decisions -- the same cluster count after every iteration -- and draw
the same labels as the single sampler, up to points whose draw sits within rounding of a decision
boundary (the two runs add the statistics in different orders; the count is recorded and bounded).
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


def _compare(single, shards, tag, max_frac=1e-3):
    k1 = single[0].cluster_count_history
    for s in shards:
        np.testing.assert_array_equal(s.cluster_count_history, k1)
    lab_sh = np.concatenate([s.labels for s in shards])
    bad = int((lab_sh != single[0].labels).sum())
    P.record(tag, label_mismatches=bad, points=int(lab_sh.size), final_clusters=int(k1[-1]))
    assert bad <= max(2, int(max_frac * lab_sh.size)), bad
    for s in shards:
        np.testing.assert_allclose(s.weights, single[0].weights, rtol=1e-6, atol=1e-9)


@pytest.mark.parametrize("D,mode", [(8, None), (32, None), (32, LL_FP32)])
def test_sharded_gaussian_run_equals_single_run(D, mode):
    N, K, iters = 60000, 6, 60
    x, z = _gauss(100 + D, N, D, K, 6.0)
    hyper = niw_hyperparams(1.0, np.zeros(D), D + 3.0, np.eye(D))
    kw = {} if mode is None else {"loglik_mode": mode}
    single = _run(x, prior_type.Gaussian, hyper, 1, iters, 11, **kw)
    shards = _run(x, prior_type.Gaussian, hyper, 2, iters, 11, **kw)
    assert single[0].cluster_count_history[-1] >= K // 2        # the run did split
    _compare(single, shards, f"shard_gauss_D{D}_{'fp32' if mode == LL_FP32 else 'auto'}")


def test_sharded_multinomial_run_equals_single_run():
    rng = np.random.default_rng(3)
    N, D, K, iters = 20000, 40, 4, 50
    theta = rng.dirichlet(np.ones(D) * 0.2, size=K)
    z = rng.integers(0, K, size=N)
    x = np.stack([rng.multinomial(60, theta[k]) for k in z]).astype(np.float64)
    hyper = multinomial_hyper(np.ones(D))
    single = _run(x, prior_type.Multinomial, hyper, 1, iters, 5)
    shards = _run(x, prior_type.Multinomial, hyper, 2, iters, 5)
    _compare(single, shards, "shard_mult_D40")


def test_sharded_verbose_scores_the_whole_data_set():
    # verbose mode with a ground truth: the NMI history comes from the contingency table summed over the
    # shards, so each shard reports the whole data set's score, equal to the single run's
    N, D, K, iters = 30000, 4, 5, 40
    x, z = _gauss(9, N, D, K, 8.0)
    hyper = niw_hyperparams(1.0, np.zeros(D), D + 3.0, np.eye(D))
    single = _run(x, prior_type.Gaussian, hyper, 1, iters, 21, gt=z)
    shards = _run(x, prior_type.Gaussian, hyper, 2, iters, 21, gt=z)
    _compare(single, shards, "shard_verbose")
    for s in shards:
        np.testing.assert_allclose(s.nmi_score_history, single[0].nmi_score_history, atol=1e-6)
        np.testing.assert_allclose(s.likelihood_history, single[0].likelihood_history, rtol=1e-9, atol=1e-6)

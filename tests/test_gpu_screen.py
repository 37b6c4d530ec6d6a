"""GPU parity of the learned split/merge screen (csrc/dpmm_screen.cu) against its FP64 oracle
(oracle/screen_oracle.py), through the C ABI, and the screen inside the sampler.

Tolerances (stated per check):
  * features (FP32 outputs of FP64 arithmetic; the NIW inverse Cholesky factor is stored in FP32):
    |f - f64| <= 2e-4 + 2e-4 |f64|;  proxy log ratio: |P - P64| <= 0.5 + 1e-5 |P64|
  * MLP scores (BF16-rounded weights, FP32 accumulate) vs FP64 with the same rounded weights:
    |z - z64| <= 1e-4 + 1e-4 |z64|
  * loss and gradient (FP32) vs FP64: loss within 1e-5 relative, gradient within 1e-4 of its norm
  * one Adam step (FP32) vs FP64: within 1e-3 lr + 1e-7 per parameter
  * selection and exact list ratios: exact (same rule / the same FP64 arithmetic as the full launch)
"""
import numpy as np
import pytest

from dpmmsubclusters_gpu_b200 import CudaKernel, capi, multinomial_hyper, niw_hyperparams, prior_type
from dpmmsubclusters_gpu_b200 import screen as SC
from dpmmsubclusters_gpu_b200.api import dp_parallel_sampling_class
from oracle import screen_oracle as S

pytestmark = pytest.mark.gpu


def _slot_rows(cnt, sm, Smat):
    """create_sufficient_statistics output -> oracle slot rows (count, sum, S column-major)"""
    n = cnt.shape[0]
    rows = []
    for q in range(n):
        for s in range(3):
            r = [np.array([cnt[q, s]], np.float64), sm[q, s]]
            if Smat is not None:
                r.append(Smat[q, s].T.reshape(-1))
            rows.append(np.concatenate(r))
    return np.array(rows)


def _gauss_kernel(seed, N=30000, D=8, K=7):
    """K labels over a mixture where labels 0 and 1 are random halves of one component (a pair whose
    merge ratio is near acceptance) and the rest are components of their own."""
    rng = np.random.default_rng(seed)
    comps = K - 1
    mus = rng.normal(size=(comps, D)) * 3.0
    z = rng.integers(0, comps, size=N)
    x = np.empty((N, D))
    for c in range(comps):
        A = rng.normal(size=(D, D))
        idx = np.flatnonzero(z == c)
        x[idx] = rng.multivariate_normal(mus[c], A @ A.T / D + 0.5 * np.eye(D), size=idx.size)
    lab = z + 1
    lab[(z == 0) & (rng.random(N) < 0.5)] = 0
    lab = lab.astype(np.int32)                       # 0..K-1
    sub = rng.integers(1, 3, size=N).astype(np.int32)
    kern = CudaKernel(prior_type.Gaussian, k_max=32).init(N, x.T, seed=seed)
    kern.set_labels(lab + 1)
    kern.set_sub_labels(sub)
    hyper = niw_hyperparams(1.0, np.zeros(D), D + 3.0, np.eye(D))
    kern.set_prior(hyper)
    cnt, sm, Smat = kern.create_sufficient_statistics(np.arange(K))
    prior = S.Prior(True, D, k0=1.0, m0=np.zeros(D), v0=D + 3.0, psi0=np.eye(D))
    return kern, _slot_rows(cnt, sm, Smat), prior, K


def _dir_kernel(seed, N=20000, D=60, K=6):
    rng = np.random.default_rng(seed)
    theta = rng.dirichlet(np.full(D, 0.3), size=K - 1)
    z = rng.integers(0, K - 1, size=N)
    x = np.zeros((N, D))
    for c in range(K - 1):
        idx = np.flatnonzero(z == c)
        x[idx] = rng.multinomial(80, theta[c], size=idx.size)
    lab = z + 1
    lab[(z == 0) & (rng.random(N) < 0.5)] = 0
    sub = rng.integers(1, 3, size=N).astype(np.int32)
    kern = CudaKernel(prior_type.Multinomial, k_max=32).init(N, x.T, seed=seed)
    kern.set_labels((lab + 1).astype(np.int32))
    kern.set_sub_labels(sub)
    alpha0 = np.ones(D)
    kern.set_prior(multinomial_hyper(alpha0))
    cnt, sm, _ = kern.create_sufficient_statistics(np.arange(K))
    return kern, _slot_rows(cnt, sm, None), S.Prior(False, D, alpha0=alpha0), K


@pytest.mark.parametrize("family", ["gauss", "dir"])
@pytest.mark.parametrize("kind", [capi.SCREEN_SPLIT, capi.SCREEN_MERGE])
def test_features_match_oracle(family, kind):
    kern, st, prior, K = _gauss_kernel(11) if family == "gauss" else _dir_kernel(12)
    alpha = 10.0
    f, P = kern.screen_features(K, kind, alpha)
    f64, P64 = (S.merge_features if kind == capi.SCREEN_MERGE else S.split_features)(st, K, prior, alpha)
    assert np.all(np.isfinite(f))
    err = np.abs(f - f64) - (2e-4 + 2e-4 * np.abs(f64))
    assert err.max() <= 0, (np.unravel_index(err.argmax(), err.shape), f.ravel()[err.argmax()], f64.ravel()[err.argmax()])
    assert np.all(np.abs(P - P64) <= 0.5 + 1e-5 * np.abs(P64)), np.abs(P - P64).max()
    if kind == capi.SCREEN_MERGE:
        # the pair of halves of one component is the most mergeable
        assert int(np.argmax(P)) == 0


def test_mlp_forward_matches_oracle():
    rng = np.random.default_rng(4)
    X = rng.normal(size=(1500, capi.SCREEN_FEATURES)).astype(np.float32)
    p = S.init_params(9)
    p[S.OFF_B1:S.OFF_W2] = rng.normal(size=S.H).astype(np.float32) * 0.1
    z = SC.forward(X, p)
    z64, _, _ = S.forward(S.deployed(p), X.astype(np.float64))
    assert np.all(np.abs(z - z64) <= 1e-4 + 1e-4 * np.abs(z64)), np.abs(z - z64).max()


def test_loss_grad_matches_oracle():
    rng = np.random.default_rng(5)
    X = rng.normal(size=(333, capi.SCREEN_FEATURES)).astype(np.float32)
    t = rng.normal(size=333).astype(np.float32)
    p = S.init_params(3)
    loss, g = SC.loss_grad(X, t, p)
    l64, g64 = S.loss_grad(p.astype(np.float64), X.astype(np.float64), t.astype(np.float64))
    assert abs(loss - l64) <= 1e-5 * abs(l64)
    assert np.linalg.norm(g - g64) <= 1e-4 * np.linalg.norm(g64)


def test_train_one_step_is_adam():
    rng = np.random.default_rng(6)
    X = rng.normal(size=(128, capi.SCREEN_FEATURES)).astype(np.float32)
    t = rng.normal(size=128).astype(np.float32)
    p = S.init_params(2)
    lr = 1e-3
    q, losses = SC.train(X, t, p, epochs=1, batch=128, lr=lr, seed=1)
    _, g64 = S.loss_grad(p.astype(np.float64), X.astype(np.float64), t.astype(np.float64))
    q64, _, _ = S.adam_step(p.astype(np.float64), np.zeros(S.NPARAM), np.zeros(S.NPARAM), g64, 1, lr)
    assert np.all(np.abs(q - q64) <= 1e-3 * lr + 1e-7), np.abs(q - q64).max()


def test_train_reduces_loss_on_learnable_target():
    rng = np.random.default_rng(8)
    X = rng.normal(size=(20000, capi.SCREEN_FEATURES)).astype(np.float32)
    w = rng.normal(size=capi.SCREEN_FEATURES)
    t = np.tanh(X @ w / 4).astype(np.float32)
    p0 = SC.init_params(0)
    l0, _ = SC.loss_grad(X, t, p0)
    p, losses = SC.train(X, t, p0, epochs=8, batch=256, lr=2e-3, seed=3)
    l1, _ = SC.loss_grad(X, t, p)
    assert losses[-1] < losses[0] and l1 < 0.05 * l0, (l0, l1, losses)


@pytest.mark.parametrize("kind", [capi.SCREEN_SPLIT, capi.SCREEN_MERGE])
def test_select_matches_rule(kind):
    kern, st, prior, K = _gauss_kernel(21)
    kern.screen_set_params(S.init_params(5))
    elig = np.ones(K, np.uint8)
    elig[3] = 0
    for top in (1, 4, 16):
        sel, scores = kern.screen_select(K, kind, 10.0, elig, top)
        rows_ok = S.merge_row_eligibility(elig, K) if kind == capi.SCREEN_MERGE else elig.astype(bool)
        assert sel.tolist() == S.select_top(scores, rows_ok, top).tolist()


def test_list_ratios_equal_full_launch():
    kern, st, prior, K = _gauss_kernel(31)
    lml, split_full = kern.split_hastings(K, 10.0)
    merge_full = kern.merge_hastings(K, 10.0)
    ks = np.array([5, 0, 3], np.int32)
    np.testing.assert_array_equal(kern.split_hastings_list(K, 10.0, ks), split_full[ks])
    pairs = np.array([[0, 1], [2, 5], [1, 6], [3, 4]], np.int32)
    got = kern.merge_hastings_list(K, 10.0, pairs)
    np.testing.assert_array_equal(got, merge_full[pairs[:, 0], pairs[:, 1]])


def _mixture(seed, N, D, K, spread):
    rng = np.random.default_rng(seed)
    mus = rng.normal(size=(K, D)) * spread
    z = rng.integers(0, K, size=N)
    x = np.empty((N, D))
    for c in range(K):
        A = rng.normal(size=(D, D))
        idx = np.flatnonzero(z == c)
        x[idx] = rng.multivariate_normal(mus[c], A @ A.T / D + 0.5 * np.eye(D), size=idx.size)
    return x, z


def _nmi(a, b):
    from sklearn.metrics import normalized_mutual_info_score
    return normalized_mutual_info_score(a, b)


def test_sampler_log_mode_records_candidates():
    x, z = _mixture(41, 20000, 4, 4, 6.0)
    s = dp_parallel_sampling_class(x.shape[0], x.T, 5, prior_type.Gaussian, screen_mode=capi.SCREEN_LOG)
    mi = s.dp_parallel(niw_hyperparams(1.0, np.zeros(4), 7.0, np.eye(4)), 10.0, iters=30, init_clusters=10,
                       verbose=False, burnout=5)
    f, hr, kind, it = mi.screen_log
    assert f.shape[1] == 32 and np.all(np.isfinite(f)) and np.all(np.isfinite(hr))
    assert (kind == 1).sum() > 0 and (kind == 0).sum() > 0 and it.min() >= 1
    assert mi.screen_stats["merge_exact"] == mi.screen_stats["merge_candidates"]


def _run(x, z, seed, mode, params=None, sweep=2):
    D = x.shape[1]
    s = dp_parallel_sampling_class(x.shape[0], x.T, seed, prior_type.Gaussian, screen_mode=mode, screen_params=params,
                                   screen_sweep_every=sweep, screen_split_min=1)
    mi = s.dp_parallel(niw_hyperparams(1.0, np.zeros(D), D + 3.0, np.eye(D)), 10.0, iters=60, init_clusters=24,
                       verbose=False, burnout=5)
    return mi, _nmi(z, mi.labels)


def test_screen_in_sampler_saves_exact_ratios_and_keeps_quality():
    # many initial clusters over 6 true ones: merges are frequent and must be found by the screen
    x, z = _mixture(51, 60000, 8, 6, 4.0)
    mi_off, nmi_off = _run(x, z, 3, capi.SCREEN_OFF)
    mi_on, nmi_on = _run(x, z, 3, capi.SCREEN_ON, SC.load_params())
    st = mi_on.screen_stats
    assert st["merge_exact"] < st["merge_candidates"], st
    assert st["split_exact"] < st["split_candidates"] or st["split_candidates"] <= 16, st
    assert abs(nmi_on - nmi_off) <= 0.05 and nmi_on > 0.85, (nmi_on, nmi_off, st)


def test_trained_network_ranking_against_proxy_and_untrained_at_d64():
    """What the trained network adds, on a shape it was not trained on (the C5 generative shape at N = 1e5,
    D = 64, every candidate logged with its exact FP64 ratio): the share of the candidates worth an exact
    ratio (log ratio > -1) that the top 16 of each (iteration, kind) group holds.  The trained network
    must beat an untrained network of the same shape and a random order clearly; against its strongest
    single input (feature 2, the proxy log ratio) it is about even -- the comparison is recorded, not
    asserted (the network does not beat the proxy consistently)."""
    import parity as P
    from dpmmsubclusters_gpu_b200.train_screen import log_run, ranking_report
    f, hr, kind, it = log_run("c5", 7, 50, 25)
    g = it.astype(np.int64) * 2 + kind
    groups = [np.flatnonzero(g == v) for v in np.unique(g)]
    rng = np.random.default_rng(0)
    net = ranking_report(groups, SC.forward(f, SC.load_params()), hr)
    proxy = ranking_report(groups, f[:, 2].astype(np.float64), hr)
    untrained = ranking_report(groups, SC.forward(f, SC.init_params(123)), hr)
    rand = ranking_report(groups, rng.random(hr.size), hr)
    P.record("screen_ranking_c5_shape", trained=net["recall_at_16"], proxy=proxy["recall_at_16"],
             untrained=untrained["recall_at_16"], random=rand["recall_at_16"])
    assert net["candidates"] > 0
    assert net["recall_at_16"] >= untrained["recall_at_16"] + 0.05, (net, untrained)
    assert net["recall_at_16"] >= rand["recall_at_16"] + 0.1, (net, rand)
    assert net["recall_at_16"] >= 0.75, net

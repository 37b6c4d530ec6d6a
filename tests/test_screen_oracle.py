"""CPU checks of the learned-screen oracle (oracle/screen_oracle.py): its MLP gradient against
central finite differences, the proxy merge ratio against the exact FP64 ratio where its
approximations are exact or close, and the selection rule."""
import numpy as np

from oracle import screen_oracle as S


def _stats_from_points(groups, D):
    """3K slots (cluster, l, r) of (count, sum, S col-major) from per-cluster point arrays, each
    cluster's points split in half for its sub-clusters."""
    rows = []
    for x in groups:
        h = x.shape[0] // 2
        for part in (x, x[:h], x[h:]):
            rows.append(np.concatenate([[part.shape[0]], part.sum(0), (part.T @ part).T.reshape(-1)]))
    return np.array(rows)


def test_mlp_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = S.init_params(1).astype(np.float64)
    p[S.OFF_B1:S.OFF_W2] = rng.normal(size=S.H) * 0.1
    X = rng.normal(size=(40, S.F))
    t = rng.normal(size=40)
    loss, g = S.loss_grad(p, X, t)
    idx = rng.choice(S.NPARAM, size=60, replace=False)
    h = 1e-6
    for e in np.concatenate([idx, [S.OFF_B3]]):
        q = p.copy()
        q[e] += h
        lp, _ = S.loss_grad(q, X, t)
        q[e] -= 2 * h
        lm, _ = S.loss_grad(q, X, t)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[e]) <= 1e-6 + 1e-5 * abs(fd), (e, fd, g[e])


def test_adam_first_step_moves_by_lr():
    p = np.zeros(4)
    g = np.array([1e-3, -2.0, 5.0, 0.0])
    q, m, v = S.adam_step(p, np.zeros(4), np.zeros(4), g, 1, 0.01)
    assert np.allclose(q[:3], -0.01 * np.sign(g[:3]), rtol=1e-4)
    assert q[3] == 0.0


def test_merge_proxy_tracks_exact_ratio_for_same_shape_clusters():
    # two halves of one Gaussian cluster, and two well separated clusters of the same shape: the
    # proxy's Minkowski bound is tight for proportional scatters, so it follows the exact ratio
    rng = np.random.default_rng(5)
    D = 6
    A = rng.normal(size=(D, D))
    cov = A @ A.T / D + 0.5 * np.eye(D)
    x = rng.multivariate_normal(np.zeros(D), cov, size=8000)
    y = rng.multivariate_normal(np.full(D, 6.0), cov, size=5000)
    prior = S.Prior(True, D, k0=1.0, m0=np.zeros(D), v0=D + 3.0, psi0=np.eye(D))
    for groups in ([x[:4000], x[4000:]], [x, y]):
        st = _stats_from_points(groups, D)
        _, prox = S.merge_features(st, 2, prior, alpha=10.0)
        exact = S.exact_merge_log_hr(st, 0, 1, prior, 10.0)
        assert abs(prox[0] - exact) <= 0.01 * abs(exact) + 8.0, (prox[0], exact)
    # and the ranking: the same-cluster halves rank above the separated pair
    st = _stats_from_points([x[:4000], x[4000:], y], D)
    _, prox = S.merge_features(st, 3, prior, alpha=10.0)
    assert prox[0] > prox[1] and prox[0] > prox[2]


def test_dirichlet_proxy_uses_stirling_terms():
    rng = np.random.default_rng(2)
    D = 30
    th = rng.dirichlet(np.ones(D))
    groups = [rng.multinomial(200, th, size=3000).astype(np.float64), rng.multinomial(200, th, size=2000).astype(np.float64)]
    rows = []
    for x in groups:
        h = x.shape[0] // 2
        for part in (x, x[:h], x[h:]):
            rows.append(np.concatenate([[part.shape[0]], part.sum(0)]))
    st = np.array(rows)
    prior = S.Prior(False, D, alpha0=np.ones(D))
    f, prox = S.merge_features(st, 2, prior, alpha=10.0)
    assert np.all(np.isfinite(f)) and f[0, 0] == 1.0 and f[0, 1] == -1.0
    # Stirling's error cancels to a few nats in the difference of marginal likelihoods
    exact = S.exact_merge_log_hr(st, 0, 1, prior, 10.0)
    assert abs(prox[0] - exact) < 0.05 * abs(exact) + 50.0, (prox[0], exact)
    fs, _ = S.split_features(st, 2, prior, alpha=10.0)
    assert np.all(np.isfinite(fs)) and np.all(fs[:, 0] == -1.0)


def test_select_top_rule():
    s = np.array([0.5, np.nan, 2.0, 2.0, -1.0, 3.0])
    elig = np.array([1, 1, 1, 1, 1, 0], bool)
    assert S.select_top(s, elig, 2).tolist() == [2, 3]
    assert S.select_top(s, elig, 3).tolist() == [0, 2, 3]
    assert S.select_top(s, elig, 10).tolist() == [0, 1, 2, 3, 4]
    assert S.merge_row_eligibility([1, 0, 1], 3).tolist() == [False, True, False]

"""The FP64 oracle pinned against the reference's own golden vectors (its GoogleTest files,
extracted by tests/golden/make_golden.py) and against the reference's compiled host code."""
import math

import numpy as np
import pytest

from conftest import eigen, inits
from oracle import oracle as O

PREFIX_G = "cudaKernel_gaussian_test::"


def _near(exp, got):
    for e, g in zip(exp, got):
        assert abs(e["value"] - g) <= e["tol"] + 1e-12, (e, g)


@pytest.mark.parametrize("name", ["log_likelihood", "log_likelihood_ignore_weight"])
def test_gaussian_loglik_goldens(goldens, name):
    # test/cudaKernel_gaussian_test.cpp:748-829
    t = goldens[PREFIX_G + name]
    I = inits(t)
    x = eigen(I["x"][0], 2, 10).T
    r = O.gauss_loglik(x, I["mu"][0], eigen(I["invSigma"][0], 2, 2), t["scalars"]["logdetSigma"],
                       t["scalars"]["weight"])
    exp = [e for e in t["expect"] if e["kind"] == "near"]
    assert len(exp) == 10
    _near(exp, r)


def test_gaussian_loglik_identity(goldens):
    # test/cudaKernel_gaussian_test.cpp:831-872: Sigma = I against the closed form
    t = goldens[PREFIX_G + "log_likelihood_sigma_is_identity"]
    I = inits(t)
    x = eigen(I["x"][0], 2, 10).T
    mu = I["mu"][0]
    r = O.gauss_loglik(x, mu, np.eye(2), t["scalars"]["logdetSigma"], 1.0)
    z = x - mu
    scalar = -((4 * math.log(2 * math.pi) + t["scalars"]["logdetSigma"]) / 2)   # sigma.size() == 4
    np.testing.assert_allclose(r, scalar - (z * z).sum(1) / 2, atol=1e-4)


def test_multinomial_loglik_golden(goldens):
    # test/cudaKernel_multinomial_test.cpp:18-55
    t = goldens["cudaKernel_multinomial_test::log_likelihood_labels"]
    x = eigen(inits(t)["x"][0], 2, 10).T
    r = O.mult_loglik(x, np.array(t["alpha_push"]))
    _near([e for e in t["expect"] if e["kind"] == "near"], r)


def _check_exprs(t, env):
    n = 0
    for e in t["expect"]:
        expr = e["expr"].replace("->", ".")
        try:
            got = eval(expr, {}, env)
        except Exception:
            continue
        tol = e.get("tol", 0.0)
        assert abs(got - e["value"]) <= tol + 1e-9, (expr, got, e["value"])
        n += 1
    return n


class _Obj:
    def __init__(self, **kw):
        self.__dict__.update(kw)


class _Vec:
    """callable + indexable wrapper so golden expressions like m(0) and S(0, 1) evaluate."""

    def __init__(self, a):
        self.a = np.asarray(a)

    def __call__(self, *i):
        return float(self.a[i])


def _ss(n, sm, S=None):
    return _Obj(N=int(n), points_sum=_Vec(sm), S=_Vec(S) if S is not None else None)


def _hp(k, m, v, psi):
    return _Obj(k=k, m=_Vec(m), v=v, psi=_Vec(psi))


def test_update_suff_stats_posterior_golden(goldens):
    # test/local_clusters_actions_test.cpp:15-172: N, sum x, S and posterior of cluster / l / r
    t = goldens["local_clusters_actions_test::update_suff_stats_posterior"]
    I = inits(t)
    x = eigen(I["points"][0], 2, 10).T
    labels = np.array(t["int_vectors"]["labels"], np.int32)
    sub = np.array(t["int_vectors"]["sub_labels"], np.int32)
    cnt, sm, S = O.suff_stats(x, labels, sub, 1)
    m0, psi0 = I["m"][0], eigen(I["psi"][0], 2, 2)
    env = {}
    names = ["", "_l", "_r"]
    for s in range(3):
        k, m, v, psi = O.niw_posterior(1.0, m0, 5.0, psi0, cnt[0, s], sm[0, s], S[0, s])
        env["ss" + names[s]] = _ss(cnt[0, s], sm[0, s], S[0, s])
        env["hyper" + names[s]] = _hp(k, m, v, psi)
    env["localCluster"] = _Obj(cluster_params=_Obj(
        cluster_params_l=_Obj(suff_statistics=env["ss_l"]), cluster_params_r=_Obj(suff_statistics=env["ss_r"])))
    assert _check_exprs(t, env) == 45


def test_create_suff_stats_dict_worker_golden(goldens):
    # test/local_clusters_actions_test.cpp:281-315
    t = goldens["local_clusters_actions_test::create_suff_stats_dict_worker"]
    I = inits(t)
    x = eigen(I["group_pts"][0], 2, 10).T
    cnt, sm, _ = O.suff_stats(x, t["int_vectors"]["labels"], t["int_vectors"]["sub_labels"], 1)
    actual = {0: _Obj(cluster_suff=_ss(cnt[0, 0], sm[0, 0]), l_suff=_ss(cnt[0, 1], sm[0, 1]),
                      r_suff=_ss(cnt[0, 2], sm[0, 2]))}
    n = 0
    for e in t["expect"]:
        expr = e["expr"].replace("->", ".").replace("actual[0]", "actual0")
        got = eval(expr, {}, {"actual0": actual[0]})
        assert abs(got - e["value"]) <= e.get("tol", 0) + 1e-9, (expr, got)
        n += 1
    assert n == 8


def test_niw_suff_stats_and_posterior_goldens(goldens):
    # test/niw_test.cpp:13-58
    t = goldens["niw_test::CreateSufficientStatistics"]
    I = inits(t)
    x = eigen(I["points"][0], 2, 10).T
    cnt, sm, S = O.suff_stats(x, np.ones(10, np.int32), np.ones(10, np.int32), 1)
    assert _check_exprs(t, {"result": _ss(cnt[0, 0], sm[0, 0], S[0, 0])}) == 7
    t = goldens["niw_test::CalcPosterior"]
    I = inits(t)
    k, m, v, psi = O.niw_posterior(1.0, I["m"][0], 5.0, eigen(I["psi"][0], 2, 2), int(t["ss_ctor_N"][0]),
                                   I["points_sum"][0], eigen(I["S"][0], 2, 2))
    assert _check_exprs(t, {"result": _hp(k, m, v, psi)}) == 4


@pytest.mark.parametrize("name,D", [("LogMarginalLikelihood_Dim3", 3), ("LogMarginalLikelihood_Dim50", 50)])
def test_niw_lml_goldens(goldens, name, D):
    # test/niw_test.cpp:184-224
    t = goldens["niw_test::" + name]
    psi_post = eigen(inits(t)["psi_posterior"][0], D, D)
    ctor = t["niw_ctor"][1]
    lml = O.niw_lml(1.0, float(D), np.eye(D), float(ctor[0]), float(ctor[2]), psi_post, int(t["ss_ctor_N"][0]))
    e = t["expect"][0]
    assert abs(lml - e["value"]) <= e["tol"], (lml, e)


def test_multinomial_prior_goldens(goldens):
    # test/multinomial_prior_test.cpp:14-103
    t = goldens["multinomial_prior_test::CreateSufficientStatistics"]
    x = eigen(inits(t)["points"][0], 2, 10).T
    cnt, sm, _ = O.suff_stats(x, np.ones(10, np.int32), np.ones(10, np.int32), 1, with_S=False)
    assert _check_exprs(t, {"result": _ss(cnt[0, 0], sm[0, 0])}) == 3
    t = goldens["multinomial_prior_test::LogMarginalLikelihood"]
    I = inits(t)
    post = O.mult_posterior(I["alpha_prior"][0], I["points_sum"][0], int(t["ss_ctor_N"][0]))
    lml = O.mult_lml(I["alpha_prior"][0], I["alpha_posterior"][0])
    assert abs(lml - t["expect"][0]["value"]) <= t["expect"][0]["tol"]
    np.testing.assert_allclose(post, I["alpha_prior"][0] + I["points_sum"][0])
    t = goldens["multinomial_prior_test::AggregateSuffStats"]
    I = inits(t)
    agg = _ss(10 + 12, I["points_l_sum"][0] + I["points_r_sum"][0])
    assert _check_exprs(t, {"suff_out": agg}) == 3


def test_should_split_local_golden(goldens):
    # test/local_clusters_actions_test.cpp:174-279: log_HR ~ 0.52088, accepted with the
    # scripted generator (uniform 0.5)
    t = goldens["local_clusters_actions_test::should_split_local"]
    I = inits(t)
    sums, Ss = I["suff_statistics->points_sum"], I["suff_statistics->S"]
    N = t["suff_N"]
    psi0 = np.eye(2)
    lml = []
    for s in range(3):
        k, m, v, psi = O.niw_posterior(1.0, np.zeros(2), 5.0, psi0, N[s], sums[s], eigen(Ss[s], 2, 2))
        lml.append(O.niw_lml(1.0, 5.0, psi0, k, v, psi, N[s]))
    hr = O.split_log_hr(10.0, N[0], N[1], N[2], lml[0], lml[1], lml[2])
    assert abs(hr - 0.5208818912506104) < 1e-3
    assert hr > math.log(0.5)


def test_alias_draw_distribution():
    # the alias table reproduces the probabilities it was built from (cudaKernel.cu:27-124)
    rng = np.random.default_rng(3)
    for k in (1, 2, 3, 7, 30):
        p = rng.dirichlet(np.ones(k))
        n = 40000
        u = rng.random((n, 2))
        u[u == 0] = 1.0
        lab = np.array([O.alias_draw(p, a, b)[0] for a, b in u])
        assert lab.min() >= 1 and lab.max() <= k
        freq = np.bincount(lab - 1, minlength=k) / n
        assert np.abs(freq - p).max() < 0.015, (k, freq, p)


def test_alias_exact_boundaries():
    # two categories: column 1 keeps label 1 iff u2 <= 2 p1 (p1 < 0.5); column 2 always 2
    p = np.array([0.3, 0.7])
    assert O.alias_draw(p, 0.2, 0.59)[0] == 1
    assert O.alias_draw(p, 0.2, 0.61)[0] == 2
    assert O.alias_draw(p, 0.9, 0.99)[0] == 2
    # equal weights: every column keeps its own label
    q = np.array([0.5, 0.5])
    assert O.alias_draw(q, 0.1, 1.0)[0] == 1 and O.alias_draw(q, 0.9, 1.0)[0] == 2


def test_relabel_rules():
    # cudaKernel.cu:172-263
    lab = np.array([1, 1, 2, 2, 3, 3], np.int32)
    sub = np.array([1, 2, 1, 2, 1, 2], np.int32)
    bits = np.array([0, 1, 2, 3, 4, 5], np.uint32)
    l2, s2 = O.split_cluster(lab, sub, 0, 3, bits)
    assert list(l2) == [1, 4, 2, 2, 3, 3] and list(s2) == [1, 2, 1, 2, 1, 2]
    l3, s3 = O.merge_clusters(lab, sub, 0, 2)
    assert list(l3) == [1, 1, 2, 2, 1, 1] and list(s3) == [1, 1, 1, 2, 2, 2]
    assert list(O.remove_empty_cluster(lab, 1)) == [1, 1, 1, 1, 2, 2]
    s4 = O.reset_bad_cluster(lab, sub, 1, np.array([7, 7, 7, 8, 7, 7], np.uint32))
    assert list(s4) == [1, 2, 2, 1, 1, 2]
    assert list(O.sample_labels_init(np.array([0.01, 0.5, 1.0]), 3, 0.0)) == [1, 2, 3]
    assert list(O.sample_labels_init(np.array([0.01, 1.0]), 3, 0.05)) == [2, 4]


# ------------------------------------------------------------------ against the compiled reference
ref_needed = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (make -C oracle ref)")


def _rand_stats(rng, D, n):
    x = rng.normal(size=(n, D)) * rng.uniform(0.5, 3) + rng.normal(size=D) * 5
    return x.sum(0), x.T @ x


@ref_needed
@pytest.mark.parametrize("D", [2, 5, 16])
def test_oracle_matches_reference_niw(D):
    import ctypes
    R = O.ref()
    rng = np.random.default_rng(D)
    m0 = rng.normal(size=D)
    A = rng.normal(size=(D, D))
    psi0 = A @ A.T / D + np.eye(D)
    k0, v0 = 1.3, D + 3.0
    pd = lambda a: np.ascontiguousarray(a, np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    for n in (0, 1, 7, 500):
        sm, S = _rand_stats(rng, D, n) if n else (np.zeros(D), np.zeros((D, D)))
        ko, mo, vo, po = ctypes.c_double(), np.empty(D), ctypes.c_double(), np.empty(D * D)
        R.ref_niw_posterior(D, k0, pd(m0), v0, pd(psi0.T), n, pd(sm), pd(S.T), ctypes.byref(ko), pd(mo),
                            ctypes.byref(vo), pd(po))
        k, m, v, psi = O.niw_posterior(k0, m0, v0, psi0, n, sm, S)
        assert k == ko.value and v == vo.value
        np.testing.assert_allclose(m, mo, rtol=1e-13, atol=1e-12)
        np.testing.assert_allclose(psi, po.reshape(D, D).T, rtol=1e-12, atol=1e-12)
        ref_lml = R.ref_niw_lml(D, k0, pd(m0), v0, pd(psi0.T), k, pd(m), v, pd(psi.T), n)
        assert abs(O.niw_lml(k0, v0, psi0, k, v, psi, n) - ref_lml) <= 1e-9 * max(1, abs(ref_lml))


@ref_needed
def test_oracle_matches_reference_lgamma_and_mvgamma():
    R = O.ref()
    for x in (0.5, 1.0, 2.5, 10.0, 1234.5, 1e6):
        assert abs(math.lgamma(x) - R.ref_r8_gamma_log(x)) <= 1e-12 * max(1, abs(math.lgamma(x)))
    for x, d in ((3.5, 2), (40.0, 16), (5000.0, 64)):
        a, b = O.log_multivariate_gamma(x, d), R.ref_log_multivariate_gamma(x, d)
        assert abs(a - b) <= 1e-10 * max(1, abs(b))


def _hastings_inputs(rng, D, n_each, sep):
    xs = [rng.normal(size=(n, D)) + sep * rng.normal(size=D) for n in n_each]
    return xs


@ref_needed
@pytest.mark.parametrize("D,sep", [(2, 0.3), (2, 6.0), (8, 1.0), (8, 5.0)])
def test_split_and_merge_ratio_match_reference(D, sep):
    """log Hastings ratios and decisions against should_split_local / should_merge compiled from
    the reference (the merge ratio has no golden vector in the reference's own tests)."""
    import ctypes
    R = O.ref()
    rng = np.random.default_rng(int(D * 10 + sep))
    m0, psi0, k0, v0, alpha = np.zeros(D), np.eye(D), 1.0, D + 3.0, 10.0
    pd = lambda a: np.ascontiguousarray(a, np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    for trial in range(4):
        xl, xr = _hastings_inputs(rng, D, [rng.integers(5, 300), rng.integers(5, 300)], sep)
        parts = [np.vstack([xl, xr]), xl, xr]
        n = np.array([len(p) for p in parts], np.int32)
        sm = np.stack([p.sum(0) for p in parts])
        S = np.stack([(p.T @ p).T for p in parts])
        lml = []
        for s in range(3):
            k, m, v, psi = O.niw_posterior(k0, m0, v0, psi0, n[s], sm[s], S[s])
            lml.append(O.niw_lml(k0, v0, psi0, k, v, psi, n[s]))
        hr_o = O.split_log_hr(alpha, n[0], n[1], n[2], *lml)
        dec, u = ctypes.c_int(), ctypes.c_double()
        hr_r = R.ref_split_log_hr(0, D, k0, pd(m0), v0, pd(psi0), None, alpha,
                                  n.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), pd(sm), pd(S), 1234 + trial, 0,
                                  ctypes.byref(dec), ctypes.byref(u))
        assert abs(hr_o - hr_r) <= 1e-8 * max(1.0, abs(hr_r)), (hr_o, hr_r)
        assert dec.value == int(hr_r > math.log(u.value))
        # merge of the two halves
        mhr_o = O.merge_log_hr(alpha, n[1], n[2], lml[1], lml[2], lml[0])
        for uu in (1e-6, 0.3, 0.999999):
            mdec = ctypes.c_int()
            n2 = np.ascontiguousarray(n[1:], np.int32)
            mhr_r = R.ref_merge_log_hr(0, D, k0, pd(m0), v0, pd(psi0), None, alpha,
                                       n2.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), pd(sm[1:]), pd(S[1:]), uu,
                                       0, ctypes.byref(mdec))
            assert abs(mhr_o - mhr_r) <= 1e-8 * max(1.0, abs(mhr_r)), (mhr_o, mhr_r)
            assert mdec.value == int(mhr_r > math.log(uu))


@ref_needed
def test_multinomial_ratio_matches_reference():
    import ctypes
    R = O.ref()
    rng = np.random.default_rng(9)
    D, alpha = 20, 5.0
    a0 = np.ones(D)
    pd = lambda a: np.ascontiguousarray(a, np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    xl = rng.poisson(rng.dirichlet(np.ones(D)) * 50, size=(40, D)).astype(float)
    xr = rng.poisson(rng.dirichlet(np.ones(D)) * 50, size=(60, D)).astype(float)
    parts = [np.vstack([xl, xr]), xl, xr]
    n = np.array([len(p) for p in parts], np.int32)
    sm = np.stack([p.sum(0) for p in parts])
    lml = [O.mult_lml(a0, O.mult_posterior(a0, sm[s], n[s])) for s in range(3)]
    dec, u = ctypes.c_int(), ctypes.c_double()
    hr_r = R.ref_split_log_hr(1, D, 0.0, None, 0.0, None, pd(a0), alpha, n.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                              pd(sm), None, 7, 0, ctypes.byref(dec), ctypes.byref(u))
    hr_o = O.split_log_hr(alpha, n[0], n[1], n[2], *lml)
    assert abs(hr_o - hr_r) <= 1e-8 * max(1, abs(hr_r))
    mdec = ctypes.c_int()
    n2 = np.ascontiguousarray(n[1:], np.int32)
    mhr_r = R.ref_merge_log_hr(1, D, 0.0, None, 0.0, None, pd(a0), alpha, n2.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                               pd(sm[1:]), None, 0.5, 0, ctypes.byref(mdec))
    assert abs(O.merge_log_hr(alpha, n[1], n[2], lml[1], lml[2], lml[0]) - mhr_r) <= 1e-8 * max(1, abs(mhr_r))

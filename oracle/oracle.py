"""ctypes front-end of the FP64 CPU oracle (dpmm_oracle.c) and of the reference shim.

TEST INFRASTRUCTURE ONLY.  The product never imports this module; tests/,
__graft_entry__.smoke() and bench.py (cpu_baseline and the reference arm) use it as
the checker.  Every function mirrors a routine of the reference's per-iteration path;
the C file cites the reference file:line of each.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_double, c_int, c_int64, c_uint32, c_ulonglong

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libdpmm_oracle.so")
REF_LIB_PATH = os.path.join(HERE, "_ref", "libdpmm_ref_host.so")

_lib = None
_ref = None


def reference_dir():
    """The reference's DPMMSubClusters/ source directory: $DPMM_REFERENCE_DIR, else a `reference/`
    checkout beside this repository; None when neither exists (e.g. on a machine that only runs the
    prebuilt checkers in _ref/)."""
    cands = [os.environ.get("DPMM_REFERENCE_DIR"),
             os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference", "DPMMSubClusters")]
    for c in cands:
        if c and os.path.isdir(c):
            return os.path.abspath(c)
    return None

_pd = POINTER(c_double)
_pi32 = POINTER(ctypes.c_int32)
_pi64 = POINTER(c_int64)
_pu32 = POINTER(c_uint32)


def build() -> str:
    """Compile the C restatement (make -C oracle) if it is missing or stale."""
    src = os.path.join(HERE, "dpmm_oracle.c")
    if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-C", HERE], check=True, capture_output=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        sig = {
            "or_gauss_loglik": (None, [c_int64, c_int, _pd, _pd, _pd, c_double, c_double, c_int, _pd]),
            "or_mult_loglik": (None, [c_int64, c_int, _pd, _pd, _pd]),
            "or_softmax_rows": (None, [c_int64, c_int, _pd]),
            "or_alias_draw": (c_int, [c_int, _pd, c_double, c_double, _pd, _pd, POINTER(c_int)]),
            "or_sample_labels": (None, [c_int64, c_int, _pd, _pd, c_int, _pi32, _pd]),
            "or_sample_sub_from_loglik": (None, [c_int64, _pd, _pd, _pd, _pi32, _pd]),
            "or_gauss_sub_labels": (None, [c_int64, c_int, _pd, _pi32, c_int, _pd, _pd, _pd, _pd, _pd,
                                           _pi32, _pd, _pd]),
            "or_mult_sub_labels": (None, [c_int64, c_int, _pd, _pi32, c_int, _pd, _pd, _pd, _pi32, _pd, _pd]),
            "or_suff_stats": (None, [c_int64, c_int, _pd, _pi32, _pi32, c_int, _pi64, _pd, _pd]),
            "or_sample_labels_init": (None, [c_int64, _pd, c_int, c_double, _pi32]),
            "or_sample_sub_labels_init": (None, [c_int64, _pd, _pi32]),
            "or_split_cluster": (None, [c_int64, _pi32, _pi32, c_int, c_int, _pu32]),
            "or_merge_clusters": (None, [c_int64, _pi32, _pi32, c_int, c_int]),
            "or_reset_bad_cluster": (None, [c_int64, _pi32, _pi32, c_int, _pu32]),
            "or_remove_empty_cluster": (None, [c_int64, _pi32, c_int]),
            "or_sub_labels_count": (None, [c_int64, _pi32, POINTER(c_int), POINTER(c_int)]),
            "or_niw_posterior": (None, [c_int, c_double, _pd, c_double, _pd, c_int64, _pd, _pd, _pd, _pd, _pd, _pd]),
            "or_logdet_chol": (c_double, [c_int, _pd]),
            "or_log_multivariate_gamma": (c_double, [c_double, c_int]),
            "or_niw_lml": (c_double, [c_int, c_double, c_double, _pd, c_double, c_double, _pd, c_int64]),
            "or_mult_posterior": (None, [c_int, _pd, _pd, c_int64, _pd]),
            "or_mult_lml": (c_double, [c_int, _pd, _pd]),
            "or_split_log_hr": (c_double, [c_double, c_int64, c_int64, c_int64, c_double, c_double, c_double]),
            "or_merge_log_hr": (c_double, [c_double, c_int64, c_int64, c_double, c_double, c_double]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_pd)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


# ---------------------------------------------------------------- per-point phases
def gauss_loglik(x, mu, inv_sigma, logdet_sigma, weight=1.0, add_log_weight=True):
    """x: (N, D) point-major.  inv_sigma: (D, D).  Returns r (N,)."""
    x = _f64(x)
    n, d = x.shape
    r = np.empty(n)
    lib().or_gauss_loglik(n, d, _d(x), _d(_f64(mu)), _d(_f64(np.asarray(inv_sigma).T)),
                          logdet_sigma, weight, int(add_log_weight), _d(r))
    return r


def mult_loglik(x, log_theta):
    x = _f64(x)
    n, d = x.shape
    r = np.empty(n)
    lib().or_mult_loglik(n, d, _d(x), _d(_f64(log_theta)), _d(r))
    return r


def alias_draw(p, u1, u2):
    p = _f64(p)
    k = p.shape[0]
    y = np.empty(k + 2)
    iw = (c_int * (2 * (k + 2)))()
    mg = c_double()
    lab = lib().or_alias_draw(k, _d(p), u1, u2, ctypes.byref(mg), _d(y), iw)
    return lab, mg.value


def sample_labels(r_nk, u, final=False):
    """r_nk: (N, K) log-likelihoods; u: (N, 2) uniforms.  Returns (labels int32, margin)."""
    r = np.asfortranarray(_f64(r_nk))           # column-major N x K like d_r
    n, k = r.shape
    buf = np.array(r.T, dtype=np.float64, copy=True).reshape(-1)   # column j contiguous
    lab = np.empty(n, np.int32)
    mg = np.empty(n)
    lib().or_sample_labels(n, k, _d(buf), _d(_f64(u).reshape(-1)), int(final),
                           lab.ctypes.data_as(_pi32), _d(mg))
    return lab, mg


def sample_sub_from_loglik(r_m2, lr_weights, u):
    r = _f64(r_m2)
    m = r.shape[0]
    buf = np.array(r.T, dtype=np.float64, copy=True).reshape(-1)
    sub = np.empty(m, np.int32)
    mg = np.empty(m)
    lib().or_sample_sub_from_loglik(m, _d(buf), _d(_f64(lr_weights)), _d(_f64(u).reshape(-1)),
                                    sub.ctypes.data_as(_pi32), _d(mg))
    return sub, mg


def gauss_sub_labels(x, labels, mu_lr, inv_sigma_lr, logdet_lr, lr_weights, u, sub_init=None):
    """mu_lr: (K, 2, D); inv_sigma_lr: (K, 2, D, D); logdet_lr/lr_weights: (K, 2)."""
    x = _f64(x)
    n, d = x.shape
    k = np.asarray(mu_lr).shape[0]
    sub = np.array(sub_init if sub_init is not None else np.zeros(n), dtype=np.int32)
    mg = np.full(n, np.inf)
    rr = np.full((n, 2), np.nan)
    inv_t = np.ascontiguousarray(np.swapaxes(_f64(inv_sigma_lr), -1, -2))   # column-major per matrix
    lib().or_gauss_sub_labels(n, d, _d(x), _i32(labels).ctypes.data_as(_pi32), k, _d(_f64(mu_lr)),
                              _d(inv_t), _d(_f64(logdet_lr)), _d(_f64(lr_weights)),
                              _d(_f64(u).reshape(-1)), sub.ctypes.data_as(_pi32), _d(mg), _d(rr))
    return sub, mg, rr


def mult_sub_labels(x, labels, log_theta_lr, lr_weights, u, sub_init=None):
    x = _f64(x)
    n, d = x.shape
    k = np.asarray(log_theta_lr).shape[0]
    sub = np.array(sub_init if sub_init is not None else np.zeros(n), dtype=np.int32)
    mg = np.full(n, np.inf)
    rr = np.full((n, 2), np.nan)
    lib().or_mult_sub_labels(n, d, _d(x), _i32(labels).ctypes.data_as(_pi32), k, _d(_f64(log_theta_lr)),
                             _d(_f64(lr_weights)), _d(_f64(u).reshape(-1)), sub.ctypes.data_as(_pi32),
                             _d(mg), _d(rr))
    return sub, mg, rr


def suff_stats(x, labels, sub_labels, k, with_S=True):
    """Returns count (K,3), sum (K,3,D), S (K,3,D,D) for cluster / l / r."""
    x = _f64(x)
    n, d = x.shape
    cnt = np.empty(3 * k, np.int64)
    sm = np.empty(3 * k * d)
    S = np.empty(3 * k * d * d) if with_S else None
    lib().or_suff_stats(n, d, _d(x), _i32(labels).ctypes.data_as(_pi32),
                        _i32(sub_labels).ctypes.data_as(_pi32), k, cnt.ctypes.data_as(_pi64), _d(sm),
                        _d(S) if with_S else None)
    out_S = S.reshape(k, 3, d, d).swapaxes(-1, -2).copy() if with_S else None
    return cnt.reshape(k, 3), sm.reshape(k, 3, d), out_S


def split_cluster(labels, sub, index, new_index, bits):
    labels = _i32(labels).copy(); sub = _i32(sub).copy()
    lib().or_split_cluster(labels.size, labels.ctypes.data_as(_pi32), sub.ctypes.data_as(_pi32), index,
                           new_index, np.ascontiguousarray(bits, np.uint32).ctypes.data_as(_pu32))
    return labels, sub


def merge_clusters(labels, sub, index, new_index):
    labels = _i32(labels).copy(); sub = _i32(sub).copy()
    lib().or_merge_clusters(labels.size, labels.ctypes.data_as(_pi32), sub.ctypes.data_as(_pi32), index,
                            new_index)
    return labels, sub


def reset_bad_cluster(labels, sub, index, bits):
    sub = _i32(sub).copy()
    lib().or_reset_bad_cluster(sub.size, _i32(labels).ctypes.data_as(_pi32), sub.ctypes.data_as(_pi32),
                               index, np.ascontiguousarray(bits, np.uint32).ctypes.data_as(_pu32))
    return sub


def remove_empty_cluster(labels, limit):
    labels = _i32(labels).copy()
    lib().or_remove_empty_cluster(labels.size, labels.ctypes.data_as(_pi32), limit)
    return labels


def sample_labels_init(u, initial_clusters, outlier_mod):
    u = _f64(u)
    out = np.empty(u.size, np.int32)
    lib().or_sample_labels_init(u.size, _d(u), initial_clusters, outlier_mod, out.ctypes.data_as(_pi32))
    return out


def sample_sub_labels_init(u):
    u = _f64(u)
    out = np.empty(u.size, np.int32)
    lib().or_sample_sub_labels_init(u.size, _d(u), out.ctypes.data_as(_pi32))
    return out


# ---------------------------------------------------------------- host maths
def niw_posterior(k, m, v, psi, count, sm, S):
    m = _f64(m); d = m.size
    ko, vo = c_double(), c_double()
    mo = np.empty(d); po = np.empty(d * d)
    lib().or_niw_posterior(d, k, _d(m), v, _d(_f64(np.asarray(psi).T)), int(count), _d(_f64(sm)),
                           _d(_f64(np.asarray(S).T)), ctypes.byref(ko), _d(mo), ctypes.byref(vo), _d(po))
    return ko.value, mo, vo.value, po.reshape(d, d).T.copy()


def logdet_chol(a):
    a = _f64(a)
    return lib().or_logdet_chol(a.shape[0], _d(_f64(a.T)))


def log_multivariate_gamma(x, d):
    return lib().or_log_multivariate_gamma(x, d)


def niw_lml(k0, v0, psi0, kp, vp, psip, count):
    psi0 = _f64(psi0)
    return lib().or_niw_lml(psi0.shape[0], k0, v0, _d(_f64(psi0.T)), kp, vp, _d(_f64(np.asarray(psip).T)),
                            int(count))


def mult_posterior(alpha, sm, count):
    alpha = _f64(alpha)
    out = np.empty(alpha.size)
    lib().or_mult_posterior(alpha.size, _d(alpha), _d(_f64(sm)), int(count), _d(out))
    return out


def mult_lml(alpha0, alphap):
    alpha0 = _f64(alpha0)
    return lib().or_mult_lml(alpha0.size, _d(alpha0), _d(_f64(alphap)))


def split_log_hr(alpha, n, nl, nr, lml, lml_l, lml_r):
    return lib().or_split_log_hr(alpha, int(n), int(nl), int(nr), lml, lml_l, lml_r)


def merge_log_hr(alpha, ni, nj, lml_i, lml_j, lml_ij):
    return lib().or_merge_log_hr(alpha, int(ni), int(nj), lml_i, lml_j, lml_ij)


# ---------------------------------------------------------------- reference shim
def ref_available() -> bool:
    return os.path.exists(REF_LIB_PATH)


def ref():
    """The reference's own compiled host code (oracle/_ref), or None when not built."""
    global _ref
    if _ref is None and ref_available():
        R = ctypes.CDLL(REF_LIB_PATH)
        R.ref_r8_gamma_log.restype = c_double
        R.ref_r8_gamma_log.argtypes = [c_double]
        R.ref_log_multivariate_gamma.restype = c_double
        R.ref_log_multivariate_gamma.argtypes = [c_double, c_int]
        R.ref_niw_posterior.restype = None
        R.ref_niw_posterior.argtypes = [c_int, c_double, _pd, c_double, _pd, c_int, _pd, _pd, _pd, _pd, _pd, _pd]
        R.ref_niw_lml.restype = c_double
        R.ref_niw_lml.argtypes = [c_int, c_double, _pd, c_double, _pd, c_double, _pd, c_double, _pd, c_int]
        R.ref_mult_posterior.restype = None
        R.ref_mult_posterior.argtypes = [c_int, _pd, c_int, _pd, _pd]
        R.ref_mult_lml.restype = c_double
        R.ref_mult_lml.argtypes = [c_int, _pd, _pd]
        R.ref_split_log_hr.restype = c_double
        R.ref_split_log_hr.argtypes = [c_int, c_int, c_double, _pd, c_double, _pd, _pd, c_double,
                                       POINTER(c_int), _pd, _pd, c_ulonglong, c_int, POINTER(c_int), _pd]
        R.ref_merge_log_hr.restype = c_double
        R.ref_merge_log_hr.argtypes = [c_int, c_int, c_double, _pd, c_double, _pd, _pd, c_double,
                                       POINTER(c_int), _pd, _pd, c_double, c_int, POINTER(c_int)]
        _ref = R
    return _ref

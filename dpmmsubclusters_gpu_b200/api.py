"""Host-side mirror of the reference's API for the sampler path.

Names, argument order and meaning follow the reference (DPMMSubClusters/):
  prior_type                         global_params.h:11-15
  niw_hyperparams(k, m, v, psi)      priors/niw_hyperparams.h:9-43
  multinomial_hyper(alpha)           priors/multinomial_hyper.h:9-29
  ModelInfo                          modelInfo.h:8-56
  dp_parallel_sampling_class         dp_parallel_sampling.h:9-38 (both constructors,
                                     dp_parallel, dp_parallel_from_file)
  CudaKernel                         cudaKernel.cuh:31-138 -- the device back-end, one method per
                                     reference method, over the C ABI (include/dpmm_capi.h)
Points follow the reference's Eigen layout: a D x N matrix (one column per point).
Errors raise capi.DpmmError (the reference printf()s and exit()s instead).
"""
from __future__ import annotations

import ctypes
import enum
import sys
from ctypes import byref, c_double, c_float, c_int32, c_int64, c_uint32, c_void_p
from typing import Optional, Sequence

import numpy as np

from . import capi
from .capi import check, lib

DBL_MAX = sys.float_info.max


class prior_type(enum.IntEnum):
    Gaussian = capi.PRIOR_GAUSSIAN
    Multinomial = capi.PRIOR_MULTINOMIAL


class niw_hyperparams:
    def __init__(self, k: float, m, v: float, psi):
        self.k = float(k)
        self.m = np.ascontiguousarray(m, dtype=np.float64).reshape(-1)
        self.v = float(v)
        self.psi = np.asarray(psi, dtype=np.float64).reshape(self.m.size, self.m.size)

    def clone(self):
        return niw_hyperparams(self.k, self.m.copy(), self.v, self.psi.copy())


class multinomial_hyper:
    def __init__(self, alpha):
        self.alpha = np.ascontiguousarray(alpha, dtype=np.float64).reshape(-1)

    def clone(self):
        return multinomial_hyper(self.alpha.copy())


class ModelInfo:
    """labels (1-based, N), weights, iter_count (seconds per iteration), histories."""

    def __init__(self):
        self.labels = np.zeros(0, np.int32)
        self.weights = np.zeros(0)
        self.iter_count = np.zeros(0)
        self.nmi_score_history = np.zeros(0)
        self.likelihood_history = np.zeros(0)
        self.cluster_count_history = np.zeros(0, np.int32)
        # learned split/merge screen (no counterpart in the reference): counters and the log of
        # DPMM_SCREEN_LOG runs (features (rows, 32), exact log ratios, kinds 0 split / 1 merge, iterations)
        self.screen_stats = {}
        self.screen_log = None

    @staticmethod
    def _from_handle(h) -> "ModelInfo":
        L = lib()
        mi = ModelInfo()
        n = L.dpmm_model_info_n(h)
        it = L.dpmm_model_info_iterations(h)
        nw = L.dpmm_model_info_num_weights(h)
        mi.labels = np.ctypeslib.as_array(L.dpmm_model_info_labels(h), shape=(n,)).copy() if n else mi.labels
        mi.weights = np.ctypeslib.as_array(L.dpmm_model_info_weights(h), shape=(nw,)).copy() if nw else mi.weights
        if it:
            mi.iter_count = np.ctypeslib.as_array(L.dpmm_model_info_iter_count(h), shape=(it,)).copy()
            mi.likelihood_history = np.ctypeslib.as_array(L.dpmm_model_info_likelihood_history(h), shape=(it,)).copy()
            mi.cluster_count_history = np.ctypeslib.as_array(L.dpmm_model_info_cluster_count_history(h),
                                                             shape=(it,)).copy()
            p = L.dpmm_model_info_nmi_history(h)
            if p:
                mi.nmi_score_history = np.ctypeslib.as_array(p, shape=(it,)).copy()
        st = np.zeros(8, np.int64)
        check(L.dpmm_model_info_screen_stats(h, st.ctypes.data_as(ctypes.POINTER(c_int64))))
        keys = ("split_candidates", "split_exact", "merge_candidates", "merge_exact", "sweeps", "sweep_accepts",
                "sweep_hits", "disabled_at")
        mi.screen_stats = {k: int(v) for k, v in zip(keys, st)}
        rows = L.dpmm_model_info_screen_log_rows(h)
        if rows:
            mi.screen_log = (
                np.ctypeslib.as_array(L.dpmm_model_info_screen_log_features(h), shape=(rows, capi.SCREEN_FEATURES)).copy(),
                np.ctypeslib.as_array(L.dpmm_model_info_screen_log_hr(h), shape=(rows,)).copy(),
                np.ctypeslib.as_array(L.dpmm_model_info_screen_log_kind(h), shape=(rows,)).copy(),
                np.ctypeslib.as_array(L.dpmm_model_info_screen_log_iter(h), shape=(rows,)).copy())
        return mi


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(c_double)) if a is not None else None


def _fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(c_float)) if a is not None else None


def _iptr(a):
    return a.ctypes.data_as(ctypes.POINTER(c_int32)) if a is not None else None


def nmi_from_table(table):
    """(NMI, variation of information in nats) from a K x G table of counts (host only)."""
    t = np.ascontiguousarray(table, np.int64)
    if t.ndim != 2:
        raise ValueError("table must be 2-D")
    nmi, vi = ctypes.c_double(), ctypes.c_double()
    check(lib().dpmm_nmi_from_table(t.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), t.shape[0], t.shape[1],
                                    ctypes.byref(nmi), ctypes.byref(vi)))
    return nmi.value, vi.value


def _points_major(all_data, numLabels=None) -> np.ndarray:
    """D x N (reference layout) -> contiguous N x D float64."""
    x = np.asarray(all_data, dtype=np.float64)
    if x.ndim != 2:
        raise ValueError("points must be a 2-D D x N matrix")
    if numLabels is not None and x.shape[1] != numLabels:
        raise ValueError(f"points matrix must be D x N with N = {numLabels}")
    return np.ascontiguousarray(x.T)


class dp_parallel_sampling_class:
    """dp_parallel_sampling_class(numLabels, all_data (D x N), randomSeed, priorType) or
    dp_parallel_sampling_class(modelDataFileName (.npy, N x D), modelParamsFileName (JSON), priorType)."""

    def __init__(self, a, b, c=None, d=None, *, loglik_mode: int = capi.LL_AUTO, rng_kind: int = capi.RNG_PHILOX,
                 k_max: int = 0, device: int = 0, screen_mode: int = capi.SCREEN_OFF, screen_params=None,
                 screen_top: int = 16, screen_sweep_every: int = 10, screen_min_recall: float = 0.5,
                 screen_split_min: int = 256, host_param_draws: bool = False):
        """screen_*: the learned split/merge screen (no counterpart in the reference); screen_params
        defaults to the trained parameters shipped with the package when screen_mode is SCREEN_ON."""
        self._from_file = isinstance(a, str)
        self.loglik_mode, self.rng_kind, self.k_max, self.device = loglik_mode, rng_kind, k_max, device
        self.screen_mode, self.screen_top = screen_mode, screen_top
        self.screen_sweep_every, self.screen_min_recall = screen_sweep_every, screen_min_recall
        self.screen_split_min = screen_split_min
        self.host_param_draws = host_param_draws
        if screen_mode == capi.SCREEN_ON and screen_params is None:
            from .screen import load_params
            screen_params = load_params()
        self.screen_params = None if screen_params is None else np.ascontiguousarray(screen_params, np.float32)
        if self._from_file:
            self.model_path, self.params_path = a, b
            self.prior = prior_type(c if c is not None else prior_type.Gaussian)
        else:
            self.numLabels = int(a)
            self.points = _points_major(b, self.numLabels)
            self.random_seed = int(c or 0)
            self.prior = prior_type(d if d is not None else prior_type.Gaussian)

    def dp_parallel(self, local_hyper_params, alpha_param: float, iters: int = 100, init_clusters: int = 1,
                    verbose: bool = True, draw_labels: bool = False, save_model: bool = False, burnout: int = 15,
                    gt: Optional[Sequence[int]] = None, max_clusters: float = DBL_MAX, outlier_weight: float = 0,
                    outlier_params=None) -> ModelInfo:
        if self._from_file:
            raise RuntimeError("dp_parallel needs the (numLabels, all_data, seed, prior) constructor")
        n, dim = self.points.shape
        rd, keep = self.run_desc(local_hyper_params, alpha_param, iters, init_clusters, verbose, burnout, gt,
                                 max_clusters, outlier_weight, outlier_params)
        h = c_void_p()
        check(lib().dpmm_dp_parallel(byref(rd), n, dim, _dptr(self.points), byref(h)))
        try:
            return ModelInfo._from_handle(h)
        finally:
            lib().dpmm_model_info_free(h)

    def run_desc(self, local_hyper_params, alpha_param: float, iters: int = 100, init_clusters: int = 1,
                 verbose: bool = True, burnout: int = 15, gt: Optional[Sequence[int]] = None,
                 max_clusters: float = DBL_MAX, outlier_weight: float = 0, outlier_params=None):
        """The dpmm_run_desc of a dp_parallel call, and the arrays it points into (keep them alive)."""
        rd = capi.dpmm_run_desc()
        rd.prior_type = int(self.prior)
        rd.iterations = iters
        rd.initial_clusters = init_clusters
        rd.burnout = burnout
        rd.alpha = alpha_param
        rd.max_clusters = max_clusters if max_clusters < DBL_MAX else 0
        rd.outlier_weight = outlier_weight
        rd.seed = self.random_seed
        rd.verbose = int(verbose)
        rd.loglik_mode = self.loglik_mode
        rd.rng_kind = self.rng_kind
        rd.k_max = self.k_max
        rd.device = self.device
        self._put_screen(rd)
        keep = []

        def put(h, prefix):
            if h is None:
                return
            if isinstance(h, niw_hyperparams):
                m, psi = np.ascontiguousarray(h.m), np.ascontiguousarray(h.psi.T)   # column-major
                keep.extend([m, psi])
                setattr(rd, prefix + "niw_k", h.k)
                setattr(rd, prefix + "niw_v", h.v)
                setattr(rd, prefix + "niw_m", _dptr(m))
                setattr(rd, prefix + "niw_psi", _dptr(psi))
            else:
                a = np.ascontiguousarray(h.alpha)
                keep.append(a)
                setattr(rd, prefix + "mult_alpha", _dptr(a))

        put(local_hyper_params, "")
        put(outlier_params, "out_")
        if gt is not None:
            g = np.ascontiguousarray(gt, dtype=np.int32)
            keep.append(g)
            rd.gt = _iptr(g)
        if self.screen_params is not None:
            keep.append(self.screen_params)
        return rd, keep

    def _put_screen(self, rd):
        rd.screen_mode = self.screen_mode
        rd.screen_top = self.screen_top
        rd.screen_sweep_every = self.screen_sweep_every
        rd.screen_min_recall = self.screen_min_recall
        rd.screen_split_min = self.screen_split_min
        rd.host_param_draws = int(self.host_param_draws)
        if self.screen_params is not None:
            if self.screen_params.size != capi.SCREEN_PARAMS:
                raise ValueError(f"screen_params must hold {capi.SCREEN_PARAMS} values")
            rd.screen_params = _fptr(self.screen_params)

    def dp_parallel_from_file(self, result_path: Optional[str] = None) -> ModelInfo:
        if not self._from_file:
            raise RuntimeError("dp_parallel_from_file needs the (npy, params, prior) constructor")
        rd = capi.dpmm_run_desc()
        rd.loglik_mode = self.loglik_mode
        rd.rng_kind = self.rng_kind
        rd.k_max = self.k_max
        rd.device = self.device
        self._put_screen(rd)
        h = c_void_p()
        check(lib().dpmm_dp_parallel_from_file(self.model_path.encode(), self.params_path.encode(), int(self.prior),
                                               byref(rd), byref(h)))
        try:
            if result_path:
                check(lib().dpmm_model_info_write_json(h, result_path.encode()))
            return ModelInfo._from_handle(h)
        finally:
            lib().dpmm_model_info_free(h)


class CudaKernel:
    """The device back-end (the reference's cudaKernel / cudaKernel_gaussian / cudaKernel_multinomial)
    over the C ABI.  init() mirrors cudaKernel::init(numLabels, points (D x N), seed, verbose,
    forceKernel); forceKernel 1 selects the FP32 SIMT contraction, 2 the tensor cores."""

    def __init__(self, prior: int = prior_type.Gaussian, rng_kind: int = capi.RNG_PHILOX, k_max: int = 0,
                 loglik_mode: Optional[int] = None, device: int = 0):
        self.prior = int(prior)
        self.rng_kind = rng_kind
        self.k_max = k_max
        self.loglik_mode = loglik_mode
        self.device = device
        self.ctx = None

    # -------------------------------------------------------------- lifetime (cudaKernel.cu:537-720)
    def init(self, numLabels: int, points, seed: int = 0, verbose: bool = False, forceKernel: int = 0,
             points_major: bool = False):
        x = np.ascontiguousarray(points, np.float64) if points_major else _points_major(points, numLabels)
        self.N, self.D = x.shape
        mode = self.loglik_mode
        if mode is None:
            mode = {1: capi.LL_FP32, 2: capi.LL_TC_BF16X3}.get(forceKernel, capi.LL_AUTO)
        d = capi.dpmm_desc()
        d.n_points, d.dim, d.prior_type = self.N, self.D, self.prior
        d.k_max, d.rng_kind, d.seed = self.k_max, self.rng_kind, int(seed or 0)
        d.loglik_mode, d.device, d.verbose = mode, self.device, int(verbose)
        h = c_void_p()
        check(lib().dpmm_create(byref(d), byref(h)))
        self.ctx = h
        check(lib().dpmm_upload_points(self.ctx, _dptr(x)))
        return self

    def release(self):
        if self.ctx:
            lib().dpmm_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    # -------------------------------------------------------------- labels (cudaKernel.cu:1093-1257)
    @staticmethod
    def _u(u, n):
        if u is None:
            return None
        u = np.ascontiguousarray(u, dtype=np.float32).reshape(-1)
        if u.size != n:
            raise ValueError(f"expected {n} uniforms, got {u.size}")
        return u

    def sample_labels(self, initial_clusters: int, outlier_mod: float, uniforms=None):
        u = self._u(uniforms, self.N)
        check(lib().dpmm_sample_labels(self.ctx, initial_clusters, outlier_mod, _fptr(u)))

    def sample_sub_labels(self, uniforms=None):
        u = self._u(uniforms, self.N)
        check(lib().dpmm_sample_sub_labels(self.ctx, _fptr(u)))

    def draw_uniforms(self):
        """The (N, 2) uniforms the next label / sub-label draw would take from the context's generator;
        the generator advances as that draw would (dpmm_draw_uniforms)."""
        u = np.empty(2 * self.N, np.float32)
        check(lib().dpmm_draw_uniforms(self.ctx, _fptr(u)))
        return u.reshape(self.N, 2)

    def set_labels(self, labels):
        a = np.ascontiguousarray(labels, np.int32)
        check(lib().dpmm_set_labels(self.ctx, _iptr(a)))

    def set_sub_labels(self, sub):
        a = np.ascontiguousarray(sub, np.int32)
        check(lib().dpmm_set_sub_labels(self.ctx, _iptr(a)))

    def get_labels(self) -> np.ndarray:
        out = np.empty(self.N, np.int32)
        check(lib().dpmm_get_labels(self.ctx, _iptr(out)))
        return out

    def set_ground_truth(self, gt):
        """Upload one int32 ground-truth value per point (None clears it) for label_agreement."""
        if gt is None:
            check(lib().dpmm_set_ground_truth(self.ctx, None))
            return
        a = np.ascontiguousarray(gt, np.int32)
        if a.size != self.N:
            raise ValueError("ground truth needs one value per point")
        check(lib().dpmm_set_ground_truth(self.ctx, _iptr(a)))

    def label_agreement(self, K: int):
        """(NMI, variation of information in nats) of the current labels 1..K against the ground
        truth, counted on the device (the verbose-mode score of dp_parallel_sampling.cpp:161-179)."""
        nmi, vi = ctypes.c_double(), ctypes.c_double()
        check(lib().dpmm_label_agreement(self.ctx, int(K), ctypes.byref(nmi), ctypes.byref(vi)))
        return nmi.value, vi.value

    def get_sub_labels(self) -> np.ndarray:
        out = np.empty(self.N, np.int32)
        check(lib().dpmm_get_sub_labels(self.ctx, _iptr(out)))
        return out

    def get_sub_labels_count(self):
        l, r = c_int32(), c_int32()
        check(lib().dpmm_get_sub_labels_count(self.ctx, byref(l), byref(r)))
        return l.value, r.value

    # -------------------------------------------------------------- matrix helpers
    def inverse_matrix(self, A) -> np.ndarray:
        """cudaKernel::inverse_matrix (cudaKernel.cu:1558-1598): A^-1 of a square FP64 matrix,
        computed on the device."""
        A = np.asfortranarray(A, np.float64)
        n = A.shape[0]
        if A.ndim != 2 or A.shape[1] != n:
            raise ValueError("inverse_matrix: A must be square")
        B = np.empty((n, n), np.float64, order="F")
        check(lib().dpmm_inverse_matrix(self.ctx, n, _dptr(A), _dptr(B)))
        return B

    def multiplie_matrix_for_inverseWishart(self, A, B) -> np.ndarray:
        """cudaKernel::multiplie_matrix_for_inverseWishart (cudaKernel.cu:980-1016): (A B)(A B)^T,
        computed on the device."""
        A = np.asfortranarray(A, np.float64)
        B = np.asfortranarray(B, np.float64)
        if A.ndim != 2 or B.ndim != 2 or A.shape[1] != B.shape[0]:
            raise ValueError("multiplie_matrix_for_inverseWishart: A (m, n) and B (n, k) required")
        m, n = A.shape
        k = B.shape[1]
        C = np.empty((m, m), np.float64, order="F")
        check(lib().dpmm_multiply_for_inverse_wishart(self.ctx, m, n, k, _dptr(A), _dptr(B), _dptr(C)))
        return C

    # -------------------------------------------------------------- parameters
    def set_gaussian_params(self, mu, inv_sigma, logdet_sigma, weights, mu_lr=None, inv_sigma_lr=None,
                            logdet_sigma_lr=None, lr_weights=None, factors=False):
        """mu (K, D); inv_sigma (K, D, D) -- or precision factors W with inv_sigma = W W^T when
        factors=True; logdet_sigma (K,); weights (K,); *_lr with a leading (K, 2) for l / r."""
        mu = np.ascontiguousarray(mu, np.float64)
        K = mu.shape[0]
        colmaj = lambda a: None if a is None else np.ascontiguousarray(np.swapaxes(np.asarray(a, np.float64), -1, -2))
        arrs = [mu, colmaj(inv_sigma), np.ascontiguousarray(logdet_sigma, np.float64),
                np.ascontiguousarray(weights, np.float64),
                None if mu_lr is None else np.ascontiguousarray(mu_lr, np.float64),
                colmaj(inv_sigma_lr),
                None if logdet_sigma_lr is None else np.ascontiguousarray(logdet_sigma_lr, np.float64),
                None if lr_weights is None else np.ascontiguousarray(lr_weights, np.float64)]
        fn = lib().dpmm_set_gaussian_factors if factors else lib().dpmm_set_gaussian_params
        check(fn(self.ctx, K, *[_dptr(a) for a in arrs]))
        self._keep = arrs

    def set_multinomial_params(self, log_theta, weights=None, log_theta_lr=None, lr_weights=None):
        lt = np.ascontiguousarray(log_theta, np.float64)
        K = lt.shape[0]
        w = np.ones(K) if weights is None else np.ascontiguousarray(weights, np.float64)
        ltlr = None if log_theta_lr is None else np.ascontiguousarray(log_theta_lr, np.float64)
        lrw = None if lr_weights is None else np.ascontiguousarray(lr_weights, np.float64)
        check(lib().dpmm_set_multinomial_params(self.ctx, K, _dptr(lt), _dptr(w), _dptr(ltlr), _dptr(lrw)))
        self._keep = [lt, w, ltlr, lrw]

    # -------------------------------------------------------------- phases
    def create_clusters_labels(self, K: int, bFinal: bool = False, uniforms=None, return_loglik=False):
        u = self._u(uniforms, 2 * self.N)
        r = np.empty((self.N, K), np.float32) if return_loglik else None
        check(lib().dpmm_create_clusters_labels(self.ctx, K, int(bFinal), _fptr(u), _fptr(r)))
        return r

    def create_subclusters_labels(self, K: int, uniforms=None, return_loglik=False):
        u = self._u(uniforms, 2 * self.N)
        r = np.empty((self.N, 2), np.float32) if return_loglik else None
        check(lib().dpmm_create_subclusters_labels(self.ctx, K, _fptr(u), _fptr(r)))
        return r

    def create_sufficient_statistics(self, indices):
        """-> count (n, 3), sum (n, 3, D), S (n, 3, D, D) or None, slots cluster / l / r."""
        idx = np.ascontiguousarray(indices, np.int32)
        n, D = idx.size, self.D
        cnt = np.empty(3 * n, np.int64)
        sm = np.empty(3 * n * D)
        S = np.empty(3 * n * D * D) if self.prior == prior_type.Gaussian else None
        check(lib().dpmm_create_sufficient_statistics(self.ctx, n, _iptr(idx), cnt.ctypes.data_as(ctypes.POINTER(c_int64)),
                                                      _dptr(sm), _dptr(S)))
        S = None if S is None else S.reshape(n, 3, D, D).swapaxes(-1, -2).copy()
        return cnt.reshape(n, 3), sm.reshape(n, 3, D), S

    def split_cluster_local_worker(self, index, newIndex, bits=None):
        i = np.atleast_1d(np.asarray(index, np.int32))
        j = np.atleast_1d(np.asarray(newIndex, np.int32))
        b = None if bits is None else np.ascontiguousarray(bits, np.uint32)
        check(lib().dpmm_split_clusters(self.ctx, i.size, _iptr(i), _iptr(j),
                                        None if b is None else b.ctypes.data_as(ctypes.POINTER(c_uint32))))

    def merge_clusters_worker(self, index, newIndex):
        i = np.atleast_1d(np.asarray(index, np.int32))
        j = np.atleast_1d(np.asarray(newIndex, np.int32))
        check(lib().dpmm_merge_clusters(self.ctx, i.size, _iptr(i), _iptr(j)))

    def reset_bad_clusters_worker(self, index, bits=None):
        i = np.atleast_1d(np.asarray(index, np.int32))
        b = None if bits is None else np.ascontiguousarray(bits, np.uint32)
        check(lib().dpmm_reset_bad_clusters(self.ctx, i.size, _iptr(i),
                                            None if b is None else b.ctypes.data_as(ctypes.POINTER(c_uint32))))

    def remove_empty_clusters_worker(self, limit):
        lim = np.atleast_1d(np.asarray(limit, np.int32))
        check(lib().dpmm_remove_empty_clusters(self.ctx, lim.size, _iptr(lim)))

    # -------------------------------------------------------------- test seams (test/myCudaKernel.h)
    def log_likelihood_labels(self, weight, mu, inv_sigma=None, logdet_sigma=0.0, log_theta=None):
        r = np.empty(self.N)
        if self.prior == prior_type.Gaussian:
            m = np.ascontiguousarray(mu, np.float64)
            s = np.ascontiguousarray(np.asarray(inv_sigma, np.float64).T)
            check(lib().dpmm_log_likelihood_labels_gaussian(self.ctx, _dptr(m), _dptr(s), logdet_sigma, weight, _dptr(r)))
        else:
            lt = np.ascontiguousarray(log_theta if log_theta is not None else mu, np.float64)
            check(lib().dpmm_log_likelihood_labels_multinomial(self.ctx, _dptr(lt), _dptr(r)))
        return r

    def sample_log_cat_array(self, log_likelihood_array, uniforms=None):
        a = np.asarray(log_likelihood_array, np.float64)       # N x K
        K = a.shape[1]
        buf = np.ascontiguousarray(a.T)                         # column-major N x K
        u = self._u(uniforms, 2 * self.N)
        check(lib().dpmm_sample_log_cat_array(self.ctx, K, _dptr(buf), _fptr(u)))

    def sample_log_cat_array_sub_cluster(self, log_likelihood_array, indices, lr_weights, uniforms=None):
        a = np.asarray(log_likelihood_array, np.float64)       # m x 2
        buf = np.ascontiguousarray(a.T)
        idx = np.ascontiguousarray(indices, np.int32)
        lw = np.ascontiguousarray(lr_weights, np.float64)
        u = self._u(uniforms, 2 * self.N)
        check(lib().dpmm_sample_log_cat_array_sub_cluster(self.ctx, idx.size, _dptr(buf), _iptr(idx), _dptr(lw), _fptr(u)))

    # -------------------------------------------------------------- Hastings (one launch each)
    def set_prior(self, hyper):
        if isinstance(hyper, niw_hyperparams):
            m = np.ascontiguousarray(hyper.m)
            psi = np.ascontiguousarray(hyper.psi.T)
            check(lib().dpmm_set_prior_niw(self.ctx, hyper.k, _dptr(m), hyper.v, _dptr(psi)))
        else:
            a = np.ascontiguousarray(hyper.alpha)
            check(lib().dpmm_set_prior_multinomial(self.ctx, _dptr(a)))

    def split_hastings(self, K: int, alpha: float):
        lml = np.empty(3 * K)
        hr = np.empty(K)
        check(lib().dpmm_split_hastings(self.ctx, K, alpha, _dptr(lml), _dptr(hr)))
        return lml.reshape(K, 3), hr

    def merge_hastings(self, K: int, alpha: float):
        hr = np.empty(K * K)
        check(lib().dpmm_merge_hastings(self.ctx, K, alpha, _dptr(hr)))
        return hr.reshape(K, K)

    # -------------------------------------------------------------- learned screen (no reference counterpart)
    def screen_set_params(self, params):
        p = np.ascontiguousarray(params, np.float32)
        if p.size != capi.SCREEN_PARAMS:
            raise ValueError(f"params must hold {capi.SCREEN_PARAMS} values")
        check(lib().dpmm_screen_set_params(self.ctx, _fptr(p)))

    @staticmethod
    def _rows(K, kind):
        return K * (K - 1) // 2 if kind == capi.SCREEN_MERGE else K

    def screen_features(self, K: int, kind: int, alpha: float):
        """-> features (rows, 32) float32, proxy log ratios (rows,)"""
        rows = self._rows(K, kind)
        f = np.empty((rows, capi.SCREEN_FEATURES), np.float32)
        p = np.empty(rows)
        check(lib().dpmm_screen_features(self.ctx, K, kind, alpha, _fptr(f), _dptr(p)))
        return f, p

    def screen_select(self, K: int, kind: int, alpha: float, eligible, top: int = 16):
        """-> selected rows (ascending), scores of every row"""
        e = np.ascontiguousarray(eligible, np.uint8)
        sel = np.empty(capi.SCREEN_MAX_TOP, np.int32)
        n = c_int32()
        sc = np.empty(self._rows(K, kind), np.float32)
        check(lib().dpmm_screen_select(self.ctx, K, kind, alpha, e.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), top,
                                       _iptr(sel), byref(n), _fptr(sc)))
        return sel[:n.value].copy(), sc

    def split_hastings_list(self, K: int, alpha: float, clusters):
        c = np.ascontiguousarray(clusters, np.int32)
        out = np.empty(c.size)
        check(lib().dpmm_split_hastings_list(self.ctx, K, alpha, c.size, _iptr(c), _dptr(out)))
        return out

    def merge_hastings_list(self, K: int, alpha: float, pairs):
        pr = np.ascontiguousarray(pairs, np.int32).reshape(-1, 2)
        out = np.empty(pr.shape[0])
        check(lib().dpmm_merge_hastings_list(self.ctx, K, alpha, pr.shape[0], _iptr(pr), _dptr(out)))
        return out

    # -------------------------------------------------------------- device parameter draws
    def sample_gaussian_params(self, K: int, seed: int, draw: int, weights, lr_weights):
        """NIW draws of every slot on the device (into the label-phase parameters); -> lml (K, 3)"""
        w = np.ascontiguousarray(weights, np.float64)
        lw = np.ascontiguousarray(lr_weights, np.float64).reshape(-1)
        lml = np.empty(3 * K)
        check(lib().dpmm_sample_gaussian_params(self.ctx, K, seed, draw, _dptr(w), _dptr(lw), _dptr(lml)))
        return lml.reshape(K, 3)

    def sample_multinomial_params(self, K: int, seed: int, draw: int, lr_weights):
        """Dirichlet draws of every slot on the device (into the label-phase parameters); -> lml (K, 3)"""
        lw = np.ascontiguousarray(lr_weights, np.float64).reshape(-1)
        lml = np.empty(3 * K)
        check(lib().dpmm_sample_multinomial_params(self.ctx, K, seed, draw, _dptr(lw), _dptr(lml)))
        return lml.reshape(K, 3)

    def get_multinomial_params(self, K: int):
        """log theta (K, 3, D) of the cluster / l / r slots as the label phases use them"""
        out = np.empty(3 * K * self.D, np.float32)
        check(lib().dpmm_get_multinomial_params(self.ctx, K, _fptr(out)))
        return out.reshape(K, 3, self.D)

    def merge_statistics(self, index, new_index):
        i = np.atleast_1d(np.asarray(index, np.int32))
        j = np.atleast_1d(np.asarray(new_index, np.int32))
        check(lib().dpmm_merge_statistics(self.ctx, i.size, _iptr(i), _iptr(j)))

    def compact_statistics(self, keep):
        k = np.ascontiguousarray(keep, np.int32)
        check(lib().dpmm_compact_statistics(self.ctx, k.size, _iptr(k)))

    def statistics_counts(self, indices):
        idx = np.ascontiguousarray(indices, np.int32)
        out = np.empty(3 * idx.size, np.int64)
        check(lib().dpmm_statistics_counts(self.ctx, idx.size, _iptr(idx), out.ctypes.data_as(ctypes.POINTER(c_int64))))
        return out.reshape(-1, 3)

    def gaussian_params(self, K: int):
        """-> W (3K, D, D), b (3K, D), c (3K,), mu - shift (3K, D) as packed on the device"""
        Dp = 4
        while Dp < self.D:
            Dp *= 2
        S = 3 * K
        wt = np.empty((S, Dp, Dp), np.float32)
        b = np.empty((S, Dp), np.float32)
        c = np.empty(S, np.float32)
        mu = np.empty((S, Dp), np.float32)
        check(lib().dpmm_get_gaussian_params(self.ctx, K, _fptr(wt), _fptr(b), _fptr(c), _fptr(mu)))
        D = self.D
        return np.swapaxes(wt, 1, 2)[:, :D, :D].copy(), b[:, :D].copy(), c, mu[:, :D].copy()

    def synchronize(self):
        check(lib().dpmm_synchronize(self.ctx))


class BatchSampler:
    """Many independent samplers advanced together (dpmm_batch_* of the C ABI; no counterpart in the
    reference, which runs one sampler per process).  datasets: list of D x N matrices (reference
    layout); hypers: one niw_hyperparams per data set (or one for all); every data set runs `iters`
    iterations with the same alpha / init_clusters / burnout; seeds: per data set (default 1 + index)."""

    def __init__(self, datasets, hypers, alpha: float, iters: int = 100, init_clusters: int = 1, burnout: int = 15,
                 seeds=None, k_max: int = 64, device: int = 0):
        B = len(datasets)
        self._keep = []
        runs = (capi.dpmm_run_desc * B)()
        pts = (ctypes.POINTER(c_double) * B)()
        n = np.empty(B, np.int64)
        d = np.empty(B, np.int32)
        for i, x in enumerate(datasets):
            xp = _points_major(x)
            h = hypers[i] if isinstance(hypers, (list, tuple)) else hypers
            m, psi = np.ascontiguousarray(h.m), np.ascontiguousarray(h.psi.T)
            self._keep += [xp, m, psi]
            r = runs[i]
            r.prior_type = capi.PRIOR_GAUSSIAN
            r.iterations, r.initial_clusters, r.burnout = iters, init_clusters, burnout
            r.alpha = alpha
            r.seed = int(seeds[i]) if seeds is not None else 1 + i
            r.loglik_mode, r.rng_kind, r.k_max, r.device = capi.LL_FP32, capi.RNG_PHILOX, k_max, device
            r.niw_k, r.niw_v, r.niw_m, r.niw_psi = h.k, h.v, _dptr(m), _dptr(psi)
            pts[i] = _dptr(xp)
            n[i], d[i] = xp.shape
        self._n = n
        self.h = c_void_p()
        check(lib().dpmm_batch_create(B, runs, n.ctypes.data_as(ctypes.POINTER(c_int64)),
                                      d.ctypes.data_as(ctypes.POINTER(c_int32)), pts, byref(self.h)))
        self.count = B

    def step(self, n_iters: int):
        check(lib().dpmm_batch_step(self.h, n_iters))

    def info(self) -> dict:
        out = np.zeros(10, np.int64)
        check(lib().dpmm_batch_info(self.h, out.ctypes.data_as(ctypes.POINTER(c_int64))))
        return {"data_sets": int(out[0]), "groups": int(out[1]), "batched_label_launches": int(out[2]),
                "graph_launches": int(out[3]),
                "block_size_by_padded_dim": {dp: int(v) for dp, v in zip((4, 8, 16, 32, 64, 128), out[4:]) if v}}

    def model_info(self, i: int) -> ModelInfo:
        h = c_void_p()
        check(lib().dpmm_batch_model_info(self.h, i, byref(h)))
        try:
            return ModelInfo._from_handle(h)
        finally:
            lib().dpmm_model_info_free(h)

    def close(self):
        if self.h:
            lib().dpmm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

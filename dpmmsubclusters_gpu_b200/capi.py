"""ctypes bindings of include/dpmm_capi.h (the library's C ABI).

Loading fails loudly when the native library is missing: there is no Python or CPU
fallback for any compute entry point.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import (POINTER, Structure, c_char_p, c_double, c_float, c_int, c_int8, c_int32, c_int64, c_uint8,
                    c_uint32, c_uint64, c_void_p)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdpmm_b200.so")

DPMM_OK = 0
STATUS_NAMES = {0: "DPMM_OK", 1: "DPMM_ERR_INVALID_ARG", 2: "DPMM_ERR_OOM", 3: "DPMM_ERR_CUDA", 4: "DPMM_ERR_NOT_PD",
                5: "DPMM_ERR_TIMEOUT", 6: "DPMM_ERR_NUMERIC", 7: "DPMM_ERR_STATE", 8: "DPMM_ERR_IO",
                9: "DPMM_ERR_NO_DEVICE", 10: "DPMM_ERR_EXCHANGE"}

PRIOR_GAUSSIAN, PRIOR_MULTINOMIAL = 0, 1
RNG_PHILOX, RNG_CURAND_XORWOW = 0, 1
LL_FP32, LL_TC_BF16X3, LL_AUTO = 0, 1, 2
SCREEN_OFF, SCREEN_ON, SCREEN_LOG = 0, 1, 2
SCREEN_SPLIT, SCREEN_MERGE = 0, 1
SCREEN_FEATURES, SCREEN_HIDDEN, SCREEN_PARAMS, SCREEN_MAX_TOP = 32, 64, 6337, 256


class DpmmError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class dpmm_desc(Structure):
    _fields_ = [("n_points", c_int64), ("dim", c_int32), ("prior_type", c_int32), ("k_max", c_int32),
                ("rng_kind", c_int32), ("seed", c_uint64), ("loglik_mode", c_int32), ("device", c_int32),
                ("verbose", c_int32), ("reserved", c_int32 * 7)]


_PD = POINTER(c_double)


class dpmm_run_desc(Structure):
    _fields_ = [("prior_type", c_int32), ("iterations", c_int32), ("initial_clusters", c_int32),
                ("burnout", c_int32), ("alpha", c_double), ("max_clusters", c_double),
                ("outlier_weight", c_double), ("seed", c_uint64), ("verbose", c_int32),
                ("loglik_mode", c_int32), ("rng_kind", c_int32), ("k_max", c_int32),
                ("niw_k", c_double), ("niw_v", c_double), ("niw_m", _PD), ("niw_psi", _PD), ("mult_alpha", _PD),
                ("out_niw_k", c_double), ("out_niw_v", c_double), ("out_niw_m", _PD), ("out_niw_psi", _PD),
                ("out_mult_alpha", _PD), ("gt", POINTER(c_int32)), ("device", c_int32),
                ("screen_mode", c_int32), ("screen_top", c_int32), ("screen_sweep_every", c_int32),
                ("screen_min_recall", c_float), ("screen_params", POINTER(c_float)), ("screen_split_min", c_int32),
                ("host_param_draws", c_int32), ("label_prune_margin", c_float), ("reserved", c_int32 * 1)]


# dpmm_allreduce_fn: int (*)(void* user, double* buf, int64_t count, void* stream)
ALLREDUCE_FN = ctypes.CFUNCTYPE(c_int, c_void_p, c_void_p, c_int64, c_void_p)


class dpmm_shard(Structure):
    _fields_ = [("rank", c_int32), ("world", c_int32), ("point_offset", c_int64), ("n_total", c_int64),
                ("allreduce", ALLREDUCE_FN), ("user", c_void_p)]


# every symbol include/dpmm_capi.h declares, with its ctypes signature
_PI32 = POINTER(c_int32)
_PI64 = POINTER(c_int64)
_PF = POINTER(c_float)
_PU32 = POINTER(c_uint32)
_CTX = c_void_p
SIGNATURES = {
    "dpmm_status_string": (c_char_p, [c_int]),
    "dpmm_last_error": (c_char_p, []),
    "dpmm_capi_version": (c_int, []),
    "dpmm_create": (c_int, [POINTER(dpmm_desc), POINTER(c_void_p)]),
    "dpmm_destroy": (c_int, [_CTX]),
    "dpmm_upload_points": (c_int, [_CTX, _PD]),
    "dpmm_upload_points_f32": (c_int, [_CTX, _PF]),
    "dpmm_sample_labels": (c_int, [_CTX, c_int, c_double, _PF]),
    "dpmm_sample_sub_labels": (c_int, [_CTX, _PF]),
    "dpmm_draw_uniforms": (c_int, [_CTX, _PF]),
    "dpmm_set_labels": (c_int, [_CTX, _PI32]),
    "dpmm_set_sub_labels": (c_int, [_CTX, _PI32]),
    "dpmm_get_labels": (c_int, [_CTX, _PI32]),
    "dpmm_get_sub_labels": (c_int, [_CTX, _PI32]),
    "dpmm_get_sub_labels_count": (c_int, [_CTX, _PI32, _PI32]),
    "dpmm_inverse_matrix": (c_int, [_CTX, c_int, _PD, _PD]),
    "dpmm_multiply_for_inverse_wishart": (c_int, [_CTX, c_int, c_int, c_int, _PD, _PD, _PD]),
    "dpmm_set_gaussian_params": (c_int, [_CTX, c_int, _PD, _PD, _PD, _PD, _PD, _PD, _PD, _PD]),
    "dpmm_set_gaussian_factors": (c_int, [_CTX, c_int, _PD, _PD, _PD, _PD, _PD, _PD, _PD, _PD]),
    "dpmm_set_multinomial_params": (c_int, [_CTX, c_int, _PD, _PD, _PD, _PD]),
    "dpmm_create_clusters_labels": (c_int, [_CTX, c_int, c_int, _PF, _PF]),
    "dpmm_create_subclusters_labels": (c_int, [_CTX, c_int, _PF, _PF]),
    "dpmm_create_sufficient_statistics": (c_int, [_CTX, c_int, _PI32, _PI64, _PD, _PD]),
    "dpmm_split_clusters": (c_int, [_CTX, c_int, _PI32, _PI32, _PU32]),
    "dpmm_merge_clusters": (c_int, [_CTX, c_int, _PI32, _PI32]),
    "dpmm_reset_bad_clusters": (c_int, [_CTX, c_int, _PI32, _PU32]),
    "dpmm_remove_empty_clusters": (c_int, [_CTX, c_int, _PI32]),
    "dpmm_log_likelihood_labels_gaussian": (c_int, [_CTX, _PD, _PD, c_double, c_double, _PD]),
    "dpmm_log_likelihood_labels_multinomial": (c_int, [_CTX, _PD, _PD]),
    "dpmm_sample_log_cat_array": (c_int, [_CTX, c_int, _PD, _PF]),
    "dpmm_sample_log_cat_array_sub_cluster": (c_int, [_CTX, c_int, _PD, _PI32, _PD, _PF]),
    "dpmm_set_prior_niw": (c_int, [_CTX, c_double, _PD, c_double, _PD]),
    "dpmm_set_prior_multinomial": (c_int, [_CTX, _PD]),
    "dpmm_split_hastings": (c_int, [_CTX, c_int, c_double, _PD, _PD]),
    "dpmm_merge_hastings": (c_int, [_CTX, c_int, c_double, _PD]),
    "dpmm_synchronize": (c_int, [_CTX]),
    "dpmm_dp_parallel": (c_int, [POINTER(dpmm_run_desc), c_int64, c_int32, _PD, POINTER(c_void_p)]),
    "dpmm_dp_parallel_from_file": (c_int, [c_char_p, c_char_p, c_int32, POINTER(dpmm_run_desc), POINTER(c_void_p)]),
    "dpmm_model_info_n": (c_int64, [c_void_p]),
    "dpmm_model_info_labels": (_PI32, [c_void_p]),
    "dpmm_model_info_num_weights": (c_int32, [c_void_p]),
    "dpmm_model_info_weights": (_PD, [c_void_p]),
    "dpmm_model_info_iterations": (c_int32, [c_void_p]),
    "dpmm_model_info_iter_count": (_PD, [c_void_p]),
    "dpmm_model_info_likelihood_history": (_PD, [c_void_p]),
    "dpmm_model_info_nmi_history": (_PD, [c_void_p]),
    "dpmm_model_info_cluster_count_history": (_PI32, [c_void_p]),
    "dpmm_model_info_write_json": (c_int, [c_void_p, c_char_p]),
    "dpmm_model_info_free": (None, [c_void_p]),
    "dpmm_sampler_create": (c_int, [POINTER(dpmm_run_desc), c_int64, c_int32, c_void_p, c_int32, POINTER(c_void_p)]),
    "dpmm_sampler_create_sharded": (c_int, [POINTER(dpmm_run_desc), c_int64, c_int32, c_void_p, c_int32,
                                            POINTER(dpmm_shard), POINTER(c_void_p)]),
    "dpmm_set_shard": (c_int, [_CTX, POINTER(dpmm_shard)]),
    "dpmm_sampler_step": (c_int, [c_void_p, c_int32]),
    "dpmm_sampler_num_clusters": (c_int, [c_void_p, _PI32]),
    "dpmm_sampler_stream": (c_void_p, [c_void_p]),
    "dpmm_sampler_model_info": (c_int, [c_void_p, POINTER(c_void_p)]),
    "dpmm_sampler_destroy": (c_int, [c_void_p]),
    "dpmm_sampler_context": (c_void_p, [c_void_p]),
    "dpmm_kernel_launch_count": (c_uint64, []),
    "dpmm_transfer_bytes": (None, [POINTER(c_uint64), POINTER(c_uint64)]),
    "dpmm_phase_times": (c_int, [_CTX, c_int, _PD, _PI64]),
    "dpmm_merge_hastings_static": (c_int, [c_int32, c_int32, c_int32, c_double, c_double, c_double, c_void_p,
                                           c_void_p, c_void_p, c_void_p]),
    "dpmm_screen_set_params": (c_int, [_CTX, _PF]),
    "dpmm_screen_features": (c_int, [_CTX, c_int, c_int, c_double, _PF, _PD]),
    "dpmm_screen_select": (c_int, [_CTX, c_int, c_int, c_double, POINTER(c_uint8), c_int, _PI32, _PI32, _PF]),
    "dpmm_split_hastings_list": (c_int, [_CTX, c_int, c_double, c_int, _PI32, _PD]),
    "dpmm_merge_hastings_list": (c_int, [_CTX, c_int, c_double, c_int, _PI32, _PD]),
    "dpmm_screen_forward": (c_int, [_PF, c_int64, _PF, _PF, c_int32]),
    "dpmm_screen_loss_grad": (c_int, [_PF, _PF, c_int32, _PF, _PF, _PF, c_int32]),
    "dpmm_screen_train": (c_int, [_PF, _PF, c_int64, c_int32, c_int32, c_float, c_uint64, _PF, _PF, c_int32]),
    "dpmm_model_info_screen_stats": (c_int, [c_void_p, _PI64]),
    "dpmm_model_info_screen_log_rows": (c_int64, [c_void_p]),
    "dpmm_model_info_screen_log_features": (_PF, [c_void_p]),
    "dpmm_model_info_screen_log_hr": (_PD, [c_void_p]),
    "dpmm_model_info_screen_log_kind": (POINTER(c_int8), [c_void_p]),
    "dpmm_model_info_screen_log_iter": (_PI32, [c_void_p]),
    "dpmm_sample_gaussian_params": (c_int, [_CTX, c_int, c_uint64, c_uint64, _PD, _PD, _PD]),
    "dpmm_sample_multinomial_params": (c_int, [_CTX, c_int, c_uint64, c_uint64, _PD, _PD]),
    "dpmm_merge_statistics": (c_int, [_CTX, c_int, _PI32, _PI32]),
    "dpmm_compact_statistics": (c_int, [_CTX, c_int, _PI32]),
    "dpmm_statistics_counts": (c_int, [_CTX, c_int, _PI32, _PI64]),
    "dpmm_get_gaussian_params": (c_int, [_CTX, c_int, _PF, _PF, _PF, _PF]),
    "dpmm_get_multinomial_params": (c_int, [_CTX, c_int, _PF]),
    "dpmm_set_wait_test": (c_int, [_CTX, c_int32]),
    "dpmm_set_fused_sub_stats": (c_int, [_CTX, c_int32]),
    "dpmm_set_outlier_prior_niw": (c_int, [_CTX, c_double, _PD, c_double, _PD]),
    "dpmm_set_outlier_prior_multinomial": (c_int, [_CTX, _PD]),
    "dpmm_set_cluster_priors": (c_int, [_CTX, c_int, ctypes.POINTER(ctypes.c_uint8)]),
    "dpmm_set_label_pruning": (c_int, [_CTX, c_double]),
    "dpmm_label_pruning_stats": (c_int, [_CTX, _PD]),
    "dpmm_set_ground_truth": (c_int, [_CTX, _PI32]),
    "dpmm_label_agreement": (c_int, [_CTX, c_int, _PD, _PD]),
    "dpmm_nmi_from_table": (c_int, [_PI64, c_int, c_int, _PD, _PD]),
    "dpmm_batch_create": (c_int, [c_int32, POINTER(dpmm_run_desc), _PI64, _PI32, POINTER(_PD), POINTER(c_void_p)]),
    "dpmm_batch_step": (c_int, [c_void_p, c_int32]),
    "dpmm_batch_info": (c_int, [c_void_p, _PI64]),
    "dpmm_batch_model_info": (c_int, [c_void_p, c_int32, POINTER(c_void_p)]),
    "dpmm_batch_destroy": (c_int, [c_void_p]),
}

_lib = None


def lib():
    """The loaded native library.  Raises if it was not built (no fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"native library {LIB_PATH} is missing; build it with "
                              "`python -m dpmmsubclusters_gpu_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != DPMM_OK:
        msg = lib().dpmm_last_error()
        raise DpmmError(status, msg.decode() if msg else "")

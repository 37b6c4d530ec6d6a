"""B200-native (sm_100a) per-iteration path of the sub-cluster DPMM sampler.

The compute path is the native library libdpmm_b200.so (C ABI in include/dpmm_capi.h):
hand-written CUDA kernels for the label / sub-label draws, the sufficient-statistic
reduction and the split / merge Hastings ratios, driven by a C++ host loop with the
reference's iteration semantics.  This package mirrors the reference's API
(dp_parallel_sampling_class, niw_hyperparams, multinomial_hyper, ModelInfo, prior_type) and
exposes the device back-end (CudaKernel) for kernel-level use.
"""
from .api import (DBL_MAX, BatchSampler, CudaKernel, ModelInfo, dp_parallel_sampling_class,  # noqa: F401
                  multinomial_hyper, niw_hyperparams, prior_type)
from .capi import (LL_AUTO, LL_FP32, LL_TC_BF16X3, RNG_CURAND_XORWOW, RNG_PHILOX, DpmmError,  # noqa: F401
                   lib)

__all__ = ["BatchSampler", "CudaKernel", "ModelInfo", "dp_parallel_sampling_class", "multinomial_hyper", "niw_hyperparams",
           "prior_type", "DpmmError", "lib", "LL_AUTO", "LL_FP32", "LL_TC_BF16X3", "RNG_PHILOX",
           "RNG_CURAND_XORWOW", "DBL_MAX"]

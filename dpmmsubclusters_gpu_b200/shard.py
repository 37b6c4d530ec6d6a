"""Data-parallel sampler over a data set split by points across ranks (one GPU per rank).

No counterpart in the reference, whose multi-device code is inactive (cudaKernel.cu:553-554 keeps one
device).  The path shards naturally: labels, sub-labels and every per-point phase stay on the rank that
holds the points, and the only exchange is a sum of the per-cluster sufficient statistics (plus a few
counts) after each statistics phase.  The native sampler (dpmm_sampler_create_sharded) calls the
exchange through a C callback, `dpmm_allreduce_fn`; this module provides

  * shard_bounds          the contiguous split of N points over `world` ranks;
  * TorchDistributedExchange
                          the exchange over a torch.distributed process group: NCCL on device buffers
                          (the sampler's own buffers, summed in place), gloo on host buffers;
  * LocalGroupExchange    the exchange between `world` samplers driven from threads of one process
                          (host-side sums in rank order), for running a sharded data set on one GPU;
  * ShardedSampler        one rank's sampler.

Every rank runs the same host loop with the same seed; after each exchange the statistics are
identical on all ranks, so every split / merge decision and parameter draw is identical too.
"""
from __future__ import annotations

import ctypes
import threading
from typing import Optional

import numpy as np

from . import capi
from .capi import check, lib


def shard_bounds(n_total: int, world: int, rank: int):
    """(point_offset, n_local) of `rank`'s contiguous shard: the first n_total % world ranks take one
    point more, so every point belongs to exactly one shard."""
    if world < 1 or not 0 <= rank < world or n_total < world:
        raise ValueError("need 0 <= rank < world <= n_total")
    base, extra = divmod(n_total, world)
    off = rank * base + min(rank, extra)
    return off, base + (1 if rank < extra else 0)


class _Exchange:
    """Holds the ctypes callback (it must outlive every sampler that uses it)."""

    def __init__(self):
        self.calls = 0
        self.values = 0
        self.callback = capi.ALLREDUCE_FN(self._entry)

    def _entry(self, user, buf, count, stream):
        try:
            self.allreduce(buf, int(count), stream)
            self.calls += 1
            self.values += int(count)
            return 0
        except Exception as e:   # the sampler turns a non-zero return into DPMM_ERR_EXCHANGE
            self.error = e
            return 1

    def allreduce(self, buf, count, stream):
        raise NotImplementedError


def _cudart():
    # the CUDA runtime the library itself is linked against (same instance: already loaded)
    lib()
    return ctypes.CDLL("libcudart.so.12")


class _CudaBuffer:
    """A device buffer of doubles seen by torch through __cuda_array_interface__ (no copy)."""

    def __init__(self, ptr, count):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f8", "data": (ptr, False), "version": 3,
                                         "strides": None, "stream": None}


class TorchDistributedExchange(_Exchange):
    """Sum over a torch.distributed process group.  device=True: the buffers are the sampler's device
    buffers, reduced in place by the group's backend (NCCL over NVLink / NVSwitch); the sampler's stream
    is drained first and the reduction is complete on return.  device=False: host buffers (gloo)."""

    def __init__(self, group=None, device: bool = True):
        super().__init__()
        self.group = group
        self.device = device
        self._rt = _cudart() if device else None

    def allreduce(self, buf, count, stream):
        import torch
        import torch.distributed as dist
        if self.device:
            if self._rt.cudaStreamSynchronize(ctypes.c_void_p(stream)) != 0:
                raise RuntimeError("cudaStreamSynchronize failed")
            t = torch.as_tensor(_CudaBuffer(buf, count), device=torch.device("cuda", torch.cuda.current_device()))
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
            torch.cuda.current_stream().synchronize()
        else:
            a = np.ctypeslib.as_array(ctypes.cast(buf, ctypes.POINTER(ctypes.c_double)), shape=(count,))
            t = torch.from_numpy(a)
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)


class LocalGroupExchange:
    """The exchange between `world` samplers driven from `world` threads of one process: each rank's
    buffer is copied to the host, the sums are formed in rank order (so every rank gets the same
    values) and copied back.  device=False: the buffers are host memory."""

    def __init__(self, world: int, device: bool = True, timeout: float = 300.0):
        self.world = world
        self.device = device
        self._rt = _cudart() if device else None
        # a rank that never arrives (it failed, or took another path) breaks the exchange after `timeout`
        # seconds: the waiting ranks' samplers then report DPMM_ERR_EXCHANGE instead of waiting forever
        self._barrier = threading.Barrier(world, timeout=timeout)
        self._parts = [None] * world
        self._sum = None
        self.ranks = [self._Rank(self, r) for r in range(world)]

    class _Rank(_Exchange):
        def __init__(self, group, rank):
            super().__init__()
            self.group, self.rank = group, rank

        def allreduce(self, buf, count, stream):
            self.group._reduce(self.rank, buf, count, stream)

    def _copy(self, dst, src, nbytes, kind):
        if self._rt.cudaMemcpy(ctypes.c_void_p(dst), ctypes.c_void_p(src), ctypes.c_size_t(nbytes), kind) != 0:
            raise RuntimeError("cudaMemcpy failed")

    def _reduce(self, rank, buf, count, stream):
        if self.device:
            if self._rt.cudaStreamSynchronize(ctypes.c_void_p(stream)) != 0:
                raise RuntimeError("cudaStreamSynchronize failed")
            a = np.empty(count, np.float64)
            self._copy(a.ctypes.data, buf, a.nbytes, 2)            # device -> host
        else:
            a = np.ctypeslib.as_array(ctypes.cast(buf, ctypes.POINTER(ctypes.c_double)), shape=(count,)).copy()
        self._parts[rank] = a
        if self._barrier.wait() == 0:
            s = self._parts[0].copy()
            for p in self._parts[1:]:
                if p.shape != s.shape:
                    raise RuntimeError("ranks exchanged different sizes")
                s += p
            self._sum = s
        self._barrier.wait()
        s = self._sum
        if self.device:
            self._copy(buf, s.ctypes.data, s.nbytes, 1)             # host -> device
        else:
            np.ctypeslib.as_array(ctypes.cast(buf, ctypes.POINTER(ctypes.c_double)), shape=(count,))[:] = s
        self._barrier.wait()


class ShardedSampler:
    """One rank's sampler over its shard of a data set split by points.

    points: this rank's (n_local, D) points, point-major, as a host numpy array (float64 / float32) or
    a device address (int, with points_f32 saying the type).  run: a dpmm_run_desc (e.g. from
    dp_parallel_sampling_class.run_desc) with an explicit seed, the same on every rank."""

    def __init__(self, run, points, n_local: int, dim: int, point_offset: int, n_total: int, rank: int, world: int,
                 exchange: Optional[_Exchange], points_f32: Optional[bool] = None, keep=()):
        self._keep = (run, points, exchange, keep)
        if isinstance(points, np.ndarray):
            f32 = points.dtype == np.float32
            if not f32:
                points = np.ascontiguousarray(points, np.float64)
            self._keep = (run, points, exchange, keep)
            ptr = points.ctypes.data
        else:
            f32 = bool(points_f32)
            ptr = int(points)
        sh = capi.dpmm_shard()
        sh.rank, sh.world, sh.point_offset, sh.n_total = rank, world, point_offset, n_total
        if exchange is not None:
            sh.allreduce = exchange.callback
        self._shard = sh
        self.exchange = exchange
        self.n_local = n_local
        h = ctypes.c_void_p()
        check(lib().dpmm_sampler_create_sharded(ctypes.byref(run), n_local, dim, ctypes.c_void_p(ptr), int(f32),
                                                ctypes.byref(sh), ctypes.byref(h)))
        self.h = h

    def step(self, n: int = 1):
        check(lib().dpmm_sampler_step(self.h, n))

    def num_clusters(self) -> int:
        k = ctypes.c_int32()
        check(lib().dpmm_sampler_num_clusters(self.h, ctypes.byref(k)))
        return k.value

    def model_info(self):
        from .api import ModelInfo
        mi = ctypes.c_void_p()
        check(lib().dpmm_sampler_model_info(self.h, ctypes.byref(mi)))
        try:
            return ModelInfo._from_handle(mi)
        finally:
            lib().dpmm_model_info_free(mi)

    @property
    def stream(self):
        return lib().dpmm_sampler_stream(self.h)

    @property
    def context(self):
        return lib().dpmm_sampler_context(self.h)

    def close(self):
        if self.h:
            check(lib().dpmm_sampler_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

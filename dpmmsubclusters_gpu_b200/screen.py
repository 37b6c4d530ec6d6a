"""Learned split/merge screen: parameter files and the device MLP entry points.

The screen has no counterpart in the reference (which evaluates the exact Hastings ratio of every
split candidate and every cluster pair, local_clusters_actions.cpp:244-321).  A 32 -> 64 -> 64 -> 1
ReLU MLP scores each candidate from 32 features of the sufficient statistics; the sampler computes
the exact FP64 ratio only for the top-scored candidates (dpmm_run_desc.screen_*).  Training and
inference run on the device through the C ABI (dpmm_screen_train / _loss_grad / _forward).

Parameter vector (FP32, DPMM_SCREEN_PARAMS = 6337 values): W1[64][32], b1[64], W2[64][64], b2[64],
w3[64], b3.  The trained vector ships as ``screen_params.f32`` (raw little-endian FP32) next to this
file; ``train_screen.py`` regenerates it.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import capi
from .capi import check, lib

HERE = os.path.dirname(os.path.abspath(__file__))
PARAMS_PATH = os.path.join(HERE, "screen_params.f32")

F, H, NPARAM = capi.SCREEN_FEATURES, capi.SCREEN_HIDDEN, capi.SCREEN_PARAMS


def target(log_hr, lo: float = -30.0, hi: float = 10.0) -> np.ndarray:
    """Regression target of a candidate: its exact log Hastings ratio clamped to [lo, hi], / 10."""
    return (np.clip(np.asarray(log_hr, dtype=np.float64), lo, hi) / 10.0).astype(np.float32)


def init_params(seed: int) -> np.ndarray:
    """He-uniform weights, zero biases."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, np.float64)
    o1, o2, o3 = 0, H * F + H, H * F + H + H * H + H
    p[o1:o1 + H * F] = rng.uniform(-1, 1, H * F) * np.sqrt(6.0 / F)
    p[o2:o2 + H * H] = rng.uniform(-1, 1, H * H) * np.sqrt(6.0 / H)
    p[o3:o3 + H] = rng.uniform(-1, 1, H) * np.sqrt(6.0 / H)
    return p.astype(np.float32)


def load_params(path: str = PARAMS_PATH) -> np.ndarray:
    p = np.fromfile(path, dtype="<f4")
    if p.size != NPARAM:
        raise ValueError(f"{path}: expected {NPARAM} FP32 values, found {p.size}")
    return p


def save_params(p, path: str = PARAMS_PATH) -> None:
    np.ascontiguousarray(p, dtype="<f4").tofile(path)


def _f(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def forward(features, params, device: int = 0) -> np.ndarray:
    """Scores of features (rows, 32) with the deployed (BF16-weight) parameters, on the device."""
    X = np.ascontiguousarray(features, np.float32).reshape(-1, F)
    p = np.ascontiguousarray(params, np.float32)
    out = np.empty(X.shape[0], np.float32)
    check(lib().dpmm_screen_forward(_f(X), X.shape[0], _f(p), _f(out), device))
    return out


def loss_grad(features, targets, params, device: int = 0):
    """Mean squared error of the FP32 parameters over all rows and its gradient, on the device."""
    X = np.ascontiguousarray(features, np.float32).reshape(-1, F)
    t = np.ascontiguousarray(targets, np.float32)
    p = np.ascontiguousarray(params, np.float32)
    loss = np.zeros(1, np.float32)
    g = np.empty(NPARAM, np.float32)
    check(lib().dpmm_screen_loss_grad(_f(X), _f(t), X.shape[0], _f(p), _f(loss), _f(g), device))
    return float(loss[0]), g


def train(features, targets, params, epochs: int = 30, batch: int = 256, lr: float = 2e-3, seed: int = 0,
          device: int = 0):
    """Adam training on the device; returns (trained parameters, mean loss per epoch)."""
    X = np.ascontiguousarray(features, np.float32).reshape(-1, F)
    t = np.ascontiguousarray(targets, np.float32)
    p = np.ascontiguousarray(params, np.float32).copy()
    losses = np.zeros(epochs, np.float32)
    check(lib().dpmm_screen_train(_f(X), _f(t), X.shape[0], epochs, batch, lr, seed, _f(p), _f(losses), device))
    return p, losses

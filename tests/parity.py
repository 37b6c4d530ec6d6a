"""Parity criteria shared by the GPU tests: log-likelihoods against the FP64 oracle and labels against
the oracle's draw on FP64 log-likelihoods with the same uniforms.

Log-likelihoods.  The reference's Gaussian r carries the constant -D^2 ln(2 pi)/2
(cudaKernel_gaussian.cu:75, :108), 3764 nats at D = 64, which would hide any error if it entered the
denominator.  The checks here take it out and state three figures per case:
  * abs      max |r - r64| in nats;
  * density  |r - r64| / max(|log N(x; mu, Sigma)|, 1), with the Gaussian's own D ln(2 pi)/2 constant:
             the relative error against FP64 of the log-likelihood;
  * quad     |r - r64| / max((x - mu)^T Sigma^-1 (x - mu) / 2, 1): relative to the data term alone, with
             an absolute floor of 1e-4 nats where the point sits at the mean.
Each test asserts density <= LL_REL and quad <= LL_REL (LL_REL = 1e-4); the absolute error grows with
the data term (far clusters, whose probability is negligible, carry the largest one) and is recorded.

Labels.  A label drawn on the GPU's r may differ from the oracle's draw on FP64 r (same uniforms) only
where the FP64 alias construction had a decision margin (oracle's `margin`: the closest y - 1 or
y - u2 comparison) smaller than what the row's log-likelihood error can move: each y = K p changes by
at most about 2 K p |dr| and the carried deficits by their sum, so 4 K (row error + 1e-6) bounds the
change (1e-6: the draw's own FP32 softmax).  argmax labels: a flip needs a gap below twice the row
error.  Every mismatch must satisfy its bound; the count is returned and recorded.

With DPMM_PARITY_REPORT=<file> every check appends one JSON line with its figures to that file.
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

from oracle import oracle as O

LOG2PI = math.log(2 * math.pi)
LL_REL = 1e-4

def record(label, **fig):
    path = os.environ.get("DPMM_PARITY_REPORT")
    if not path:
        return
    out = {"check": label}
    for k, v in fig.items():
        out[k] = float(v) if isinstance(v, (np.floating, float)) else v
    with open(path, "a") as f:
        f.write(json.dumps(out) + "\n")


def gauss_ll(r_gpu, r64, D, logdet, logw, path, label):
    """r_gpu (N, K): the GPU's r (the device omits the -D^2 ln(2 pi)/2 constant); r64 (N, K): the oracle's
    FP64 values (with it); logdet (K,) log det Sigma_k; logw (K,) the log weight inside r (0 for the
    sub-cluster r).  Asserts both relative bounds; returns the per-row absolute error (nats)."""
    r_gpu = np.asarray(r_gpu, np.float64).reshape(r64.shape)
    err = np.abs(r_gpu - D * D * LOG2PI / 2 - r64)
    half_q = (-D * D * LOG2PI / 2 - np.asarray(logdet) / 2 + np.asarray(logw)) - r64
    dens = -D * LOG2PI / 2 - np.asarray(logdet) / 2 - half_q
    rel_d = float((err / np.maximum(np.abs(dens), 1.0)).max())
    rel_q = float((err / np.maximum(half_q, 1.0)).max())
    record(label, path=path, D=D, abs_max=float(err.max()), rel_density_max=rel_d, rel_quad_max=rel_q)
    assert rel_d <= LL_REL, (label, "relative to the log density", rel_d)
    assert rel_q <= LL_REL, (label, "relative to the data term", rel_q)
    return err.max(axis=1)


def labels_vs_fp64(lab_gpu, r64, u, row_err, label, final=False):
    """The GPU's labels against the oracle's draw (or argmax) on FP64 r with the same uniforms u (N, 2).
    Returns the number of mismatches (each one inside its margin bound)."""
    K = r64.shape[1]
    lab64, mg = O.sample_labels(r64, u, final=final)
    bound = (2 * row_err + 1e-9) if final else 4 * K * (row_err + 1e-6)
    bad = lab_gpu != lab64
    record(label, mismatches=int(bad.sum()), points=int(bad.size), final=bool(final),
           worst_margin_over_bound=float((mg[bad] / bound[bad]).max()) if bad.any() else 0.0)
    assert np.all(mg[bad] < bound[bad]), (label, int(bad.sum()), mg[bad][:5], bound[bad][:5])
    return int(bad.sum())


def sub_labels_vs_fp64(sub_gpu, r64_2, labels, lrw, u, row_err, label):
    """Sub-labels drawn on the GPU against the oracle's two-way draw on FP64 sub-cluster r (N, 2) of each
    point's cluster, same uniforms; bound 8 (row error + 1e-6) per point (K = 2)."""
    n = sub_gpu.size
    sub64 = np.zeros(n, np.int32)
    mg = np.full(n, np.inf)
    for k in range(lrw.shape[0]):
        idx = np.flatnonzero(labels == k + 1)
        if idx.size:
            sub64[idx], mg[idx] = O.sample_sub_from_loglik(r64_2[idx], lrw[k], u[idx])
    bound = 8 * (row_err + 1e-6)
    bad = sub_gpu != sub64
    record(label, mismatches=int(bad.sum()), points=int(n),
           worst_margin_over_bound=float((mg[bad] / bound[bad]).max()) if bad.any() else 0.0)
    assert np.all(mg[bad] < bound[bad]), (label, int(bad.sum()), mg[bad][:5], bound[bad][:5])
    return int(bad.sum())

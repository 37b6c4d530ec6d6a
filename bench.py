#!/usr/bin/env python
"""Benchmark: sampler throughput (points x iterations / s) of the sub-cluster DPMM sampler.

Workload (default): the large overlapping Gaussian configuration -- N = 10,000,000 points,
D = 64, 100 true clusters, means ~ N(0, 5^2 I), covariances A A^T / D + 0.5 I, Dirichlet(2)
weights, float32 data; NIW(kappa=1, m=0, nu=67, Psi=I), alpha = 10, 300 iterations.  Data are
seeded synthetic draws of that generative model, generated on the device.

A "step" is one sampler iteration (local_clusters_actions::group_step: parameter draws, label
phase, sub-label + statistics phase, split and merge tests, relabels).  The sampler starts from the
reference's default of one cluster and runs `--burnin` untimed iterations (130: the split schedule
doubles the clusters every ~15 iterations and reaches the configuration's 100 by about iteration 120),
then W warm-up iterations, then exactly K timed iterations bracketed by a barrier and device
synchronisation, timed with CUDA events on the sampler's stream.  Inputs (2.56 GB) are larger than L2.

The metric compares the product path ("mixed": split-BF16 / split-TF32 tensor-core contractions, pruned
label phase, device parameter draws, learned split / merge screen) with the plain FP32 form ("plain":
dense FP32 SIMT label phase, SIMT statistics, host parameter draws, every candidate exact) run on the
same data, seed and iteration counts in the same invocation: vs_baseline = value / plain's value, and
both NMIs against the generating labels are reported.  --ablation adds the intermediate arms.

--gpus N (under torchrun): by default one data set of N x 1e7 points (one generative model, each rank
drawing its own 1e7 points) sharded by points over the ranks: per-point phases on each rank, the
per-cluster statistics summed over the ranks with NCCL after each statistics phase, every host
decision replicated (weak scaling; value = all ranks' points x iterations over the max elapsed time).
--multi-gpu replicas runs N independent samplers instead.

--impl reference times the reference's per-point path on the host cores: the reference has no CPU
implementation of these phases (every one dispatches to its CUDA back-end), so its FP64
restatement (oracle/) runs in a pool of all host threads on a bounded sample per step.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "sampler points*iters/sec at N=1e7 D=64: mixed+learned vs plain FP32, NMI within 0.01"
UNIT = "points*iters/s"
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    except Exception:
        return dict(FALLBACK_PEAKS), "fallback"


# ----------------------------------------------------------------------------- workload
# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of single-launch ncu captures of the
# timed kernels on a smaller case of the same workload (N = 1e6 points, D = 64; `ncu --set full
# --clock-control none -k regex:<kernel> -c 1` of the C5 generator at N = 1e6), with the number of
# points (and clusters) of that capture.  bench.py scales them to the timed launch by the kernel's
# traffic model; they are a cross-check of the algorithmic bytes, not a live measurement.
NCU_TRAFFIC = {
    "k_gauss_labels_tc": {"dram_bytes": 619413504, "points": 1_000_000, "clusters": 95},
    "k_prune_scan1_tc": {"dram_bytes": 270950144, "points": 1_000_000},
    "k_slot_stats_tc": {"dram_bytes": 288693760, "points": 1_000_000},
    "k_mult_labels_tc": {"dram_bytes": 417898240, "points": 200_000},
}


def label_kernel_traffic(N, K):
    """DRAM bytes per launch of the dense tensor-core label kernel, scaled from its ncu capture by
    the kernel's traffic model N * (256 B packed points + 4 K B of r + 16 B partials)."""
    c = NCU_TRAFFIC["k_gauss_labels_tc"]
    model = lambda n, k: n * (256.0 + 4.0 * k + 16.0)
    return c["dram_bytes"] * model(N, K) / model(c["points"], c["clusters"])


def per_point_traffic(kernel, N):
    """DRAM bytes per launch of a kernel that reads each point once, scaled from its capture by N."""
    c = NCU_TRAFFIC[kernel]
    return c["dram_bytes"] * N / c["points"]


def padded(d):
    p = 4
    while p < d:
        p *= 2
    return p


def kernel_rooflines(ph_ms, ph_calls, N, D, k_mean, kept, pk, pk_src, tc, fused=False):
    """Per timed kernel (CUDA events around each launch on its stream): algorithmic work per launch,
    achieved rate and the fraction of the measured peak of its bound.  tc: the pruned scan and the
    sub-cluster statistics ran on the tensor cores (padded dimension 32 / 64, mixed mode); fused: the
    sub-labels and statistics ran as one kernel (k_sub_stats_tc, timed in the statistics slot)."""
    Dp = padded(D)
    hbm = pk.get("hbm_gbs", FALLBACK_PEAKS["hbm_gbs"])
    bf16 = pk.get("bf16_tflops", FALLBACK_PEAKS["bf16_tflops"])
    out = {}

    def add(name, slot, bound, work, unit, peak, peak_key, note, traffic=None):
        if ph_calls[slot] == 0:
            return
        ms = ph_ms[slot] / ph_calls[slot]
        scale = 1e12 if unit == "TFLOP/s" else 1e9
        ach = work / (ms / 1e3) / scale if ms > 0 else None
        out[name] = {"bound": bound, "achieved": ach, "peak": peak, "unit": unit,
                     "frac": ach / peak if ach else None, "traffic": traffic, "launch_ms": ms,
                     "launches": int(ph_calls[slot]), "total_ms": ph_ms[slot],
                     "peak_source": f"{peak_key} of {pk_src}", "algorithmic": note}

    add("k_gauss_labels_tc", 7, "tensor", 2.0 * N * k_mean * D * D, "TFLOP/s", bf16, "bf16_tflops",
        f"2*N*K*D^2 FLOP per launch (one product; the split form issues 3), K mean {k_mean:.1f}",
        label_kernel_traffic(N, k_mean))
    if tc:
        one_pass = k_mean <= 193   # k_prune_scan1_tc; above, the two-pass k_prune_scan_tc
        add("k_prune_scan1_tc" if one_pass else "k_prune_scan_tc", 8, "hbm", N * (Dp * 4.0 + 12), "GB/s", hbm,
            "hbm_gbs",
            "N*(Dp*4 + 12) B per launch: every point read once from HBM, its permutation index, r_h written; "
            "tensor-core products 3 x 2*N*Dp*(64 + K - 1) FLOP (one pass: r_h and every cluster's bound "
            "direction)",
            per_point_traffic("k_prune_scan1_tc", N) if Dp == 64 and one_pass else None)
        if fused:
            add("k_sub_stats_tc", 10, "hbm", N * (Dp * 4.0 + 8), "GB/s", hbm, "hbm_gbs",
                "N*(Dp*4 + 8) B per launch: every point gathered once (its row), its permutation index read "
                "and its sub-label written; tensor-core products 3 x 2*N*128*64 FLOP (sub-labels, split BF16) "
                "+ 3 x 2*N*128*(Dp+32) FLOP (statistics, split TF32)")
        else:
            add("k_slot_stats_tc", 10, "hbm", N * (Dp * 4.0 + 8), "GB/s", hbm, "hbm_gbs",
                "N*(Dp*4 + 8) B per launch: every point, its permutation index and sub-label read once; "
                "split-TF32 Gram products 3 x 2*N*128*(Dp+32) FLOP",
                per_point_traffic("k_slot_stats_tc", N) if Dp == 64 else None)
    else:
        add("k_prune_scan", 8, "hbm", N * (2.0 * Dp * 4 + 8), "GB/s", hbm, "hbm_gbs",
            "N*(2*Dp*4 + 8) B per launch: every point read twice (its own cluster's r, then the per-point "
            "bound), its permutation index and r written; FP32 SIMT work 2*N*Dp^2 FLOP + the bounds")
        add("k_gauss_slot_stats", 10, "hbm", N * (2.0 * Dp * 4 + 12), "GB/s", hbm, "hbm_gbs",
            "N*(2*Dp*4 + 12) B per launch: every point read once per sub-cluster pass, permutation, "
            "sub-label; FP32 products N*Dp*(Dp+1)")
    add("k_prune_settle+k_prune_draw", 9, "hbm", N * 12.0, "GB/s", hbm, "hbm_gbs",
        "N*12 B (permutation entry, own-cluster r, label) per launch: a lower bound, the rows of the few "
        "chunks that keep other clusters (%.3f other clusters kept per point in the last attempt) are "
        "not counted" % kept)
    return out


def c3_config(args):
    return dict(prior="multinomial", N=args.c3_n, D=1000, K_true=50, alpha=10.0, prior_alpha=1.0, iterations=150,
                burnout=15, theta_dirichlet=0.1, length_mean=200.0)


def generate_c3_torch(cfg, seed, device):
    """Seeded draws of the C3 shape on the device: theta ~ Dirichlet(0.1)^D per component, weights ~
    Dirichlet(1), vector lengths ~ Poisson(200), counts ~ Multinomial(length, theta_z); returned as float32
    counts (N x D, every value an integer that BF16 holds exactly below 257) and the component labels."""
    import torch
    torch.manual_seed(seed)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    N, D, K = cfg["N"], cfg["D"], cfg["K_true"]
    theta = torch.distributions.Dirichlet(torch.full((D,), cfg["theta_dirichlet"])).sample((K,)).to(device)
    w = torch.distributions.Dirichlet(torch.ones(K)).sample().to(device)
    z = torch.multinomial(w, N, replacement=True, generator=g)
    lens = torch.poisson(torch.full((N,), cfg["length_mean"], device=device), generator=g).long()
    x = torch.zeros(N, D, device=device, dtype=torch.float32)
    L = int(lens.max().item())
    for a in range(0, N, 50_000):
        b = min(N, a + 50_000)
        cat = torch.multinomial(theta[z[a:b]], L, replacement=True, generator=g)     # (n, L) categories
        keep = (torch.arange(L, device=device)[None, :] < lens[a:b, None]).float()
        x[a:b].scatter_add_(1, cat, keep)
    return x.contiguous(), z


def mult_kernel_rooflines(ph_ms, ph_calls, N, D, k_mean, pk, pk_src):
    """The multinomial label kernel's roofline: HBM-bound, it reads every point's counts once (BF16,
    padded to whole 64-category blocks) and writes its K values of r and the draw's partials."""
    hbm = pk.get("hbm_gbs", FALLBACK_PEAKS["hbm_gbs"])
    out = {}
    if ph_calls[7]:
        ms = ph_ms[7] / ph_calls[7]
        Dk = (D + 63) // 64 * 64
        work = N * (2.0 * Dk + 4.0 * k_mean + 16.0)
        ach = work / (ms / 1e3) / 1e9
        out["k_mult_labels_tc"] = {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                                   "traffic": per_point_traffic("k_mult_labels_tc", N) if D == 1000 else None, "launch_ms": ms, "launches": int(ph_calls[7]),
                                   "total_ms": ph_ms[7], "peak_source": f"hbm_gbs of {pk_src}",
                                   "algorithmic": "N*(2*Dk + 4*K + 16) B per launch: BF16 counts (Dk = D padded to "
                                                  "64), r written cluster-major, the draw's partials; tensor-core "
                                                  "products 3 x 2*N*Dk*Kp FLOP"}
    return out


def c5_config(args):
    return dict(N=args.n, D=args.d, K_true=args.k_true, alpha=10.0, nu=args.d + 3.0, kappa=1.0, iterations=300,
                mean_sd=5.0, dirichlet=2.0)


def generate_c5_torch(cfg, seed, device, point_seed=None):
    """Seeded draws of the configuration's generative model on the device: the model (weights, means,
    covariances) from `seed`, the points (and their generating labels) from `point_seed` (default: the
    same seed), so shards of one data set share the model and differ in their points."""
    import torch
    torch.manual_seed(seed)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    N, D, K = cfg["N"], cfg["D"], cfg["K_true"]
    w = torch.distributions.Dirichlet(torch.full((K,), cfg["dirichlet"])).sample()
    mus = torch.randn(K, D, device=device, generator=g) * cfg["mean_sd"]
    Ls = []
    for k in range(K):
        A = torch.randn(D, D, device=device, generator=g, dtype=torch.float64)
        cov = A @ A.T / D + 0.5 * torch.eye(D, device=device, dtype=torch.float64)
        Ls.append(torch.linalg.cholesky(cov).float())
    if point_seed is not None:
        g.manual_seed(point_seed)
    z = torch.multinomial(w.to(device), N, replacement=True, generator=g)
    x = torch.empty(N, D, device=device, dtype=torch.float32)
    order = torch.argsort(z)
    counts = torch.bincount(z, minlength=K).tolist()
    start = 0
    for k in range(K):
        n = counts[k]
        e = torch.randn(n, D, device=device, generator=g)
        x[order[start:start + n]] = e @ Ls[k].T + mus[k]
        start += n
    return x.contiguous(), z


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        if self.index < 0:
            return self
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [v.strip() for v in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------- CPU baseline
def _cpu_sample_worker(payload):
    import numpy as np
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    x, mu, inv, logdet, w, u, mu_lr, inv_lr, ld_lr, lrw = payload
    K = mu.shape[0]
    t0 = time.perf_counter()
    r = np.stack([O.gauss_loglik(x, mu[k], inv[k], logdet[k], w[k]) for k in range(K)], 1)
    lab, _ = O.sample_labels(r, u)
    sub, _, _ = O.gauss_sub_labels(x, lab, mu_lr, inv_lr, ld_lr, lrw, u.reshape(-1))
    O.suff_stats(x, lab, sub, K)
    return time.perf_counter() - t0


def cpu_sample_payload(x_np, n, seed, K, D):
    import numpy as np
    rng = np.random.default_rng(seed)
    idx = rng.choice(x_np.shape[0], size=n, replace=False)
    x = x_np[idx].astype(np.float64)
    mu = rng.normal(size=(K, D)) * 5
    inv = np.repeat(np.eye(D)[None], K, 0) * 0.8
    logdet = np.full(K, -D * math.log(0.8))
    w = rng.dirichlet(np.full(K, 2.0))
    u = rng.random((n, 2))
    u[u == 0] = 1.0
    mu_lr = mu[:, None, :] + rng.normal(size=(K, 2, D))
    inv_lr = np.repeat(inv[:, None], 2, 1)
    ld_lr = np.repeat(logdet[:, None], 2, 1)
    lrw = np.full((K, 2), 0.5)
    return (x, mu, inv, logdet, w, u, mu_lr, inv_lr, ld_lr, lrw)


def cpu_baseline(K, D, n):
    """The FP64 C restatement of the per-point phases (label, sub-label and statistics phases) on a
    bounded sample of n points at the workload's K and D: timed on 1 thread, then on every host core
    (one process per core, each on its own n-point sample)."""
    import multiprocessing as mp
    import numpy as np
    rng = np.random.default_rng(0)
    xs = (rng.normal(size=(n, D)) * 5).astype(np.float32)
    t1 = _cpu_sample_worker(cpu_sample_payload(xs, n, 1, K, D))
    cores = os.cpu_count() or 1
    payloads = [cpu_sample_payload((rng.normal(size=(n, D)) * 5).astype(np.float32), n, 2 + i, K, D)
                for i in range(cores)]
    with mp.get_context("spawn").Pool(cores) as pool:
        pool.map(_cpu_sample_worker, [cpu_sample_payload(xs[:64], 64, 1, K, D)] * cores)   # workers warm
        t0 = time.perf_counter()
        pool.map(_cpu_sample_worker, payloads)
        tall = time.perf_counter() - t0
    return {"value": cores * n / tall, "unit": UNIT, "cores": cores, "kind": "port",
            "one_thread": {"value": n / t1, "cores": 1, "seconds": t1},
            "sample": f"{n} points x 1 iteration of the per-point phases (K={K}, D={D}) through the FP64 C "
                      f"restatement (oracle/dpmm_oracle.c) per process; {cores} processes on {cores} host "
                      f"cores: {tall:.1f} s; 1 thread: {t1:.1f} s"}


# ----------------------------------------------------------------------------- reference arm
def run_reference(args, rank, world):
    import numpy as np
    if rank != 0:
        return 0
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    cfg = c5_config(args)
    D, K = cfg["D"], cfg["K_true"]
    per = args.ref_points_per_core
    rng = np.random.default_rng(0)
    x_np = (rng.normal(size=(per * cores, D)) * 5).astype(np.float32)
    ctx = mp.get_context("spawn")
    payloads = [cpu_sample_payload(x_np[i * per:(i + 1) * per], per, i, K, D) for i in range(cores)]
    times = []
    with ctx.Pool(cores) as pool:
        for step in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            pool.map(_cpu_sample_worker, payloads)
            dt = time.perf_counter() - t0
            if step >= args.warmup:
                times.append(dt)
    n = per * cores
    tot = sum(times)
    value = n * len(times) / tot
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": "C5 Gaussian N=1e7 D=64 K=100 (bounded host sample per step)",
                       "points_per_step": n, "K": K, "D": D},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{n} points ({per} per process x {cores} processes) per step through "
                                       "the label, sub-label and statistics phases of the reference's "
                                       "per-point path, FP64 C restatement"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------- our arm
# Sampler configurations ("arms") timed on the same data, seed and iteration counts.  "mixed" is the
# product path; "plain" is the plain FP32 form the metric compares it with: the reference's algorithm
# (dense label phase over all K clusters, per-cluster statistics, every split / merge candidate
# evaluated exactly, parameters drawn on the host in FP64) with its per-point arithmetic in FP32 SIMT
# kernels.  The ablation arms switch the mixed path's changes on one at a time.
ARMS = {
    "plain": dict(mode="fp32", prune=False, host_draws=True, screen=False,
                  what="FP32 SIMT dense label phase, SIMT statistics, host FP64 parameter draws, every "
                       "split / merge candidate exact"),
    "plain+device_draws": dict(mode="fp32", prune=False, host_draws=False, screen=False,
                               what="plain + NIW parameter draws on the device"),
    "plain+device_draws+tensor_cores": dict(mode="tc", prune=False, host_draws=False, screen=False,
                                            what="+ split-BF16 tcgen05 label / sub-label contractions and "
                                                 "split-TF32 tcgen05 statistics (dense label phase)"),
    "plain+device_draws+tensor_cores+pruning": dict(mode="tc", prune=True, host_draws=False, screen=False,
                                                    what="+ pruned label phase (exact, 30-nat margin)"),
    "mixed": dict(mode="auto", prune=True, host_draws=False, screen=True,
                  what="+ learned split / merge screen (top 16 exact, full sweep every 10): the product path"),
}


def make_run_desc(cfg, args, arm, iterations, rank, local, keep):
    from dpmmsubclusters_gpu_b200 import capi
    import numpy as np
    a = ARMS[arm]
    rd = capi.dpmm_run_desc()
    mult = cfg.get("prior") == "multinomial"
    rd.prior_type = capi.PRIOR_MULTINOMIAL if mult else capi.PRIOR_GAUSSIAN
    rd.iterations = iterations
    rd.initial_clusters = args.initial_clusters
    rd.burnout = cfg.get("burnout", 15)
    rd.alpha = cfg["alpha"]
    rd.seed = 12345 + (0 if args.multi_gpu == "shard" else rank)   # shards of one run share the seed
    rd.loglik_mode = {"auto": capi.LL_AUTO, "fp32": capi.LL_FP32, "tc": capi.LL_TC_BF16X3}[a["mode"]]
    rd.rng_kind = capi.RNG_PHILOX
    rd.k_max = 256
    rd.device = local
    if mult:
        al = np.full(cfg["D"], cfg["prior_alpha"])
        keep.append(al)
        rd.mult_alpha = al.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    else:
        m = np.zeros(cfg["D"])
        psi = np.eye(cfg["D"])
        keep += [m, psi]
        rd.niw_k, rd.niw_v = cfg["kappa"], cfg["nu"]
        rd.niw_m = m.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        rd.niw_psi = psi.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    rd.host_param_draws = int(a["host_draws"])
    rd.label_prune_margin = 0.0 if a["prune"] else -1.0
    if a["screen"]:
        from dpmmsubclusters_gpu_b200.screen import load_params
        sp = load_params()
        keep.append(sp)
        rd.screen_mode = capi.SCREEN_ON
        rd.screen_params = sp.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    return rd


def run_arm(arm, args, cfg, x, z_np, rank, local, dist, L, clocks=False, shard=None):
    """Create a sampler of configuration `arm` on the device-resident points x, run the untimed burn-in
    and warm-up iterations, then time exactly args.steps iterations with CUDA events on the sampler's
    stream (barrier + device synchronisation on both sides, max over ranks).  Returns the arm's numbers,
    the NMI of the final labels against the generating labels and the per-kernel timers."""
    import numpy as np
    import torch
    from dpmmsubclusters_gpu_b200.capi import check
    N, D = cfg["N"], cfg["D"]
    keep = []
    rd = make_run_desc(cfg, args, arm, cfg["iterations"], rank, local, keep)
    h = ctypes.c_void_p()
    if shard is not None:
        # one shard of a data set of world x N points: statistics summed over the ranks (NCCL)
        from dpmmsubclusters_gpu_b200 import capi
        sh = capi.dpmm_shard()
        sh.rank, sh.world, sh.point_offset, sh.n_total = rank, args.gpus_world, rank * N, args.gpus_world * N
        sh.allreduce = shard.callback
        keep.append(sh)
        check(L.dpmm_sampler_create_sharded(ctypes.byref(rd), N, D, ctypes.c_void_p(x.data_ptr()), 1,
                                            ctypes.byref(sh), ctypes.byref(h)))
    else:
        check(L.dpmm_sampler_create(ctypes.byref(rd), N, D, ctypes.c_void_p(x.data_ptr()), 1, ctypes.byref(h)))
    ctx = L.dpmm_sampler_context(h)
    if args.fuse:
        check(L.dpmm_set_fused_sub_stats(ctx, 1))
    stream = torch.cuda.ExternalStream(L.dpmm_sampler_stream(h), device=f"cuda:{local}")
    t0 = time.perf_counter()
    check(L.dpmm_sampler_step(h, args.burnin + args.warmup))
    torch.cuda.synchronize()
    burn_s = time.perf_counter() - t0
    k_before = ctypes.c_int32()
    check(L.dpmm_sampler_num_clusters(h, ctypes.byref(k_before)))

    check(L.dpmm_phase_times(ctx, 1, None, None))
    launches0 = L.dpmm_kernel_launch_count()
    ks = []
    with ClockSampler(local if clocks else -1) as clk:
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        if args.profile_region:
            torch.cuda.profiler.start()
        e0.record(stream)
        for _ in range(args.steps):
            check(L.dpmm_sampler_step(h, 1))
            kk = ctypes.c_int32()
            L.dpmm_sampler_num_clusters(h, ctypes.byref(kk))
            ks.append(kk.value)
        e1.record(stream)
        torch.cuda.synchronize()
        if args.profile_region:
            torch.cuda.profiler.stop()
        if dist:
            dist.barrier()
    elapsed_ms = e0.elapsed_time(e1)
    launches = L.dpmm_kernel_launch_count() - launches0
    ph_ms = (ctypes.c_double * 11)()
    ph_calls = (ctypes.c_int64 * 11)()
    check(L.dpmm_phase_times(ctx, 0, ph_ms, ph_calls))
    prune = (ctypes.c_double * 6)()
    check(L.dpmm_label_pruning_stats(ctx, prune))
    if dist:
        t = torch.tensor([elapsed_ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms = float(t.item())
    mi = ctypes.c_void_p()
    check(L.dpmm_sampler_model_info(h, ctypes.byref(mi)))
    lab = np.ctypeslib.as_array(L.dpmm_model_info_labels(mi), shape=(N,)).copy()
    scr = np.zeros(8, np.int64)
    check(L.dpmm_model_info_screen_stats(mi, scr.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
    L.dpmm_model_info_free(mi)
    check(L.dpmm_sampler_destroy(h))
    return {"arm": arm, "value": N * args.steps / (elapsed_ms / 1e3), "elapsed_ms": elapsed_ms,
            "ms_per_step": elapsed_ms / args.steps, "ks": ks, "k_before": k_before.value,
            "nmi": _nmi(lab[::10], z_np[::10]), "launches": int(launches), "ph_ms": list(ph_ms),
            "ph_calls": list(ph_calls), "prune": list(prune), "screen": scr, "burnin_s": burn_s,
            "clocks": clk.summary() if clocks else None}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--burnin", type=int, default=130)
    ap.add_argument("--initial-clusters", type=int, default=1,
                    help="clusters the sampler starts from (the reference's default is 1)")
    ap.add_argument("--n", type=int, default=10_000_000)
    ap.add_argument("--d", type=int, default=64)
    ap.add_argument("--k-true", type=int, default=100)
    ap.add_argument("--arm", default="mixed", choices=sorted(ARMS),
                    help="the configuration reported as `value` (default: the product path)")
    ap.add_argument("--compare", default="plain", choices=sorted(ARMS) + ["none"],
                    help="the arm timed beside it on the same data and iterations (vs_baseline = value / its value)")
    ap.add_argument("--multi-gpu", default="shard", choices=["shard", "replicas"],
                    help="with N > 1 ranks: shard one data set of N x n points by points over the ranks, summing "
                         "the per-cluster statistics with NCCL (default), or run N independent replicas")
    ap.add_argument("--ablation", action="store_true",
                    help="also time every intermediate arm (one change at a time) and report them")
    ap.add_argument("--fuse", action="store_true",
                    help="sub-labels and their statistics in one fused pass (k_sub_stats_tc) instead of two kernels")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--ref-points-per-core", type=int, default=600)
    ap.add_argument("--cpu-points", type=int, default=20000,
                    help="points of the CPU baseline sample (timed at 1 thread and at all threads)")
    ap.add_argument("--profile-region", action="store_true",
                    help="bracket the timed steps with cudaProfilerStart/Stop (for ncu --profile-from-start off)")
    ap.add_argument("--workload", default="c5", choices=["c5", "c3", "c4", "study"],
                    help="c4: 256 uneven data sets advanced together (BatchSampler) vs one at a time; study: "
                         "NMI and final cluster count over 10 sampler seeds, mixed vs plain FP32")
    ap.add_argument("--study-seeds", type=int, default=10)
    ap.add_argument("--study-shapes", default="c5r,c2", help="comma list of c5r (C5 at N=1e6) and c2")
    ap.add_argument("--c3-n", type=int, default=1_000_000, help="points of the multinomial workload")
    ap.add_argument("--c4-sets", type=int, default=256)
    ap.add_argument("--c4-seq-sets", type=int, default=32, help="data sets timed one at a time (a subset)")
    args = ap.parse_args()
    assert args.warmup >= 0 and args.steps >= 1

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "c4":
        return run_c4(args, rank, world, local)
    if args.workload == "study":
        return run_study(args, rank, local)

    import numpy as np
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    from dpmmsubclusters_gpu_b200.capi import lib
    L = lib()
    mult = args.workload == "c3"
    cfg = c3_config(args) if mult else c5_config(args)
    N, D = cfg["N"], cfg["D"]
    args.gpus_world = world
    sharded = world > 1 and args.multi_gpu == "shard"
    shard = None
    if sharded:
        from dpmmsubclusters_gpu_b200.shard import TorchDistributedExchange
        shard = TorchDistributedExchange(device=True)
    if mult:
        x, z = generate_c3_torch(cfg, 1003 + (0 if sharded else rank), f"cuda:{local}")
    elif sharded:
        x, z = generate_c5_torch(cfg, 1000 + 5, f"cuda:{local}", point_seed=7000 + rank)
    else:
        x, z = generate_c5_torch(cfg, 1000 + 5 + rank, f"cuda:{local}")
    z_np = z.cpu().numpy()
    torch.cuda.synchronize()

    main_arm = run_arm(args.arm, args, cfg, x, z_np, rank, local, dist, L, clocks=True, shard=shard)
    # the end-to-end call next, before the other arms and the CPU baseline (16 host processes) leave
    # the host's memory in another state for the upload's host-side copy
    e2e = run_e2e(args, cfg, rank, local, world, dist, L) if not args.no_e2e and not mult else None
    others = []
    if args.ablation:
        others = [a for a in ARMS if a != args.arm]
    elif args.compare != "none" and args.compare != args.arm:
        others = [args.compare]
    other_res = {a: run_arm(a, args, cfg, x, z_np, rank, local, dist, L, shard=shard) for a in others}

    r = main_arm
    value = world * r["value"]
    ph_ms, ph_calls, prune, ks = r["ph_ms"], r["ph_calls"], r["prune"], r["ks"]
    pk, pk_src = peaks()
    k_mean = float(np.mean(ks)) if ks else float(r["k_before"])
    tc = padded(D) in (32, 64) and ARMS[args.arm]["mode"] != "fp32"
    if mult:
        kernels = mult_kernel_rooflines(ph_ms, ph_calls, N, D, k_mean, pk, pk_src)
    else:
        kernels = kernel_rooflines(ph_ms, ph_calls, N, D, k_mean, prune[4], pk, pk_src, tc, tc and args.fuse)
    # the roofline of the kernel with the most device time in the timed region
    dominant = max(kernels, key=lambda k: kernels[k]["total_ms"]) if kernels else None
    roofline = dict(kernels[dominant], kernel=dominant) if dominant else None
    phases = ["labels", "sub_labels_stats", "stats", "split_hastings", "merge_hastings", "relabel", "params",
              "label_tc_kernel", "label_prune_scan_kernel", "label_prune_draw_kernel", "slot_stats_kernel"]

    def arm_summary(a):
        return {"what": ARMS[a["arm"]]["what"], "value": world * a["value"], "unit": UNIT,
                "ms_per_step": a["ms_per_step"], "nmi_vs_generating_labels": a["nmi"],
                "clusters_in_timed_steps": a["ks"], "gpu_launches": a["launches"],
                "phase_ms_per_step": {p: a["ph_ms"][i] / args.steps for i, p in enumerate(phases)
                                      if a["ph_calls"][i]}}

    cmp_arm = other_res.get(args.compare)
    vs = value / (world * cmp_arm["value"]) if cmp_arm else None
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": vs,
            "dtype": "f32+bf16x3" if ARMS[args.arm]["mode"] != "fp32" else "f32",
            "data": "synthetic (seeded draws of the configuration's generative model, generated on device)",
            "config": {"workload": ("C3 multinomial DPMM N=1e6 D=1000 50 true components (theta ~ Dir(0.1), "
                                    "weights Dir(1), lengths Poisson(200), counts BF16-exact); Dirichlet(1) prior; "
                                    "alpha=10" if mult else
                                    "C5 Gaussian DPMM N=1e7 D=64 100 true clusters (means N(0,25I), "
                                    "cov AA^T/D+0.5I, Dir(2) weights, f32); NIW k=1 m=0 nu=67 Psi=I; alpha=10"),
                       "N": N, "D": D, "arm": args.arm, "arm_what": ARMS[args.arm]["what"],
                       "multi_gpu": ("one data set of %d x N points sharded by points, statistics summed with "
                                     "NCCL (weak scaling)" % world if sharded else
                                     "independent replicas" if world > 1 else "one GPU"),
                       "initial_clusters": args.initial_clusters,
                       "initial_clusters_note": ("head start: the sampler starts from as many clusters as the "
                                                 "generating model has (the reference's default is 1)"
                                                 if args.initial_clusters > 1 else "the reference's default"),
                       "burnin_iterations": args.burnin,
                       "sub_labels_and_statistics": ("one fused pass (--fuse)" if args.fuse else
                                                     "two kernels (k_sub_labels_tc, k_slot_stats_tc)"),
                       "clusters_in_timed_steps": ks,
                       "l2": "inputs (N*D*4 = %.2f GB) larger than L2" % (N * D * 4 / 1e9),
                       "nmi_vs_generating_labels": r["nmi"],
                       "parameter_draws": "host" if ARMS[args.arm]["host_draws"] else "device",
                       "label_pruning": {"enabled": ARMS[args.arm]["prune"], "attempts": int(prune[0]),
                                         "pruned_phases": int(prune[1]),
                                         "kept_other_clusters_per_point": prune[2], "margin_nats": prune[3],
                                         "last_attempt_kept_per_point": prune[4],
                                         "last_attempt_chunks_over_capacity": int(prune[5])},
                       "screen": screen_summary("on" if ARMS[args.arm]["screen"] else "off", r["screen"]),
                       "vs_baseline": (f"value / the '{args.compare}' arm's value, both timed in this run on the "
                                       "same data, seed, burn-in and timed iterations" if cmp_arm else None)},
            "gpu_launches": r["launches"],
            "roofline": roofline,
            "kernel_rooflines": kernels,
            "phase_ms_per_step": {p: ph_ms[i] / args.steps for i, p in enumerate(phases) if ph_calls[i]},
            "clocks": r["clocks"]}
    if cmp_arm:
        line["compare"] = dict(arm_summary(cmp_arm), arm=args.compare,
                               nmi_delta=r["nmi"] - cmp_arm["nmi"], speedup=vs)
    if args.ablation:
        line["ablation"] = {a: arm_summary(v) for a, v in list(other_res.items()) + [(args.arm, r)]}
    line["clocks"].pop("samples", None)
    del x
    torch.cuda.empty_cache()

    if mult:
        line["metric"] = "sampler points*iters/sec at C3 (multinomial N=1e6 D=1000): mixed+learned vs plain FP32"
        line["dtype"] = "bf16 counts x bf16x3 log theta, f32 accumulate" if ARMS[args.arm]["mode"] != "fp32" else "f32"
    if rank == 0 and not args.no_cpu and not mult:
        line["cpu_baseline"] = cpu_baseline(cfg["K_true"], D, args.cpu_points)
    if e2e is not None:
        line["e2e"] = e2e
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_e2e(args, cfg, rank, local, world, dist, L):
    """The same metric through the public whole-sampler call (dpmm_dp_parallel) from HOST buffers:
    point upload, initialisation, burn-in + warm-up + timed iterations and the label download
    are all inside the timed region (wall clock, max over ranks)."""
    import numpy as np
    import torch
    from dpmmsubclusters_gpu_b200.capi import check
    x, _ = generate_c5_torch(cfg, 2000 + rank, f"cuda:{local}")
    xh = x.double().cpu().numpy()
    del x
    torch.cuda.empty_cache()
    iters = args.burnin + args.warmup + args.steps
    keep = []
    rd = make_run_desc(cfg, args, args.arm, iters, rank, local, keep)
    h2d0, d2h0 = ctypes.c_uint64(), ctypes.c_uint64()
    L.dpmm_transfer_bytes(ctypes.byref(h2d0), ctypes.byref(d2h0))
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    mi = ctypes.c_void_p()
    check(L.dpmm_dp_parallel(ctypes.byref(rd), xh.shape[0], xh.shape[1],
                             xh.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(mi)))
    labels = np.ctypeslib.as_array(L.dpmm_model_info_labels(mi), shape=(xh.shape[0],)).copy()
    L.dpmm_model_info_free(mi)
    dt = time.perf_counter() - t0
    if dist:
        t = torch.tensor([dt], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dt = float(t.item())
    h2d1, d2h1 = ctypes.c_uint64(), ctypes.c_uint64()
    L.dpmm_transfer_bytes(ctypes.byref(h2d1), ctypes.byref(d2h1))
    assert labels.min() >= 1
    return {"value": world * xh.shape[0] * iters / dt, "unit": UNIT,
            "h2d_bytes_per_step": int((h2d1.value - h2d0.value) / iters),
            "d2h_bytes_per_step": int((d2h1.value - d2h0.value) / iters),
            "iterations": iters, "wall_s": dt,
            "note": "dpmm_dp_parallel from host float64 points: upload, init, all iterations and label "
                    "download in the timed region"}


def c4_data(n_sets, seed):
    """Seeded synthetic data sets of the batched-uneven shape: N ~ logUniform[1e3, 2e5], D from
    {2, 8, 16, 64}, true K ~ Uniform{2..30}, means U(-10, 10)^D, covariances A A^T / D + 0.5 I."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_sets):
        N = int(round(math.exp(rng.uniform(math.log(1e3), math.log(2e5)))))
        D = int(rng.choice([2, 8, 16, 64]))
        K = int(rng.integers(2, 31))
        mus = rng.uniform(-10, 10, size=(K, D))
        z = rng.integers(0, K, size=N)
        x = np.empty((N, D))
        for c in range(K):
            idx = np.flatnonzero(z == c)
            A = rng.normal(size=(D, D))
            L = np.linalg.cholesky(A @ A.T / D + 0.5 * np.eye(D))
            x[idx] = mus[c] + rng.normal(size=(idx.size, D)) @ L.T
        out.append((x.astype(np.float32).astype(np.float64).T.copy(), z))
    return out


def generate_c2_torch(seed, device, N=1_000_000, D=32, K=20):
    """Seeded draws of the C2 shape: means U(-20, 20)^D, covariances A A^T / D + 0.5 I, Dirichlet(1) weights."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    torch.manual_seed(seed)
    w = torch.distributions.Dirichlet(torch.ones(K)).sample()
    mus = (torch.rand(K, D, device=device, generator=g) * 40 - 20)
    z = torch.multinomial(w.to(device), N, replacement=True, generator=g)
    x = torch.empty(N, D, device=device, dtype=torch.float32)
    for k in range(K):
        idx = torch.nonzero(z == k).flatten()
        A = torch.randn(D, D, device=device, generator=g, dtype=torch.float64)
        L = torch.linalg.cholesky(A @ A.T / D + 0.5 * torch.eye(D, device=device, dtype=torch.float64)).float()
        x[idx] = torch.randn(idx.numel(), D, device=device, generator=g) @ L.T + mus[k]
    return x.contiguous(), z


def run_study(args, rank, local):
    """End-to-end quality of the product path against the plain FP32 form: for each shape, one seeded
    synthetic data set and sampler seeds 0 .. S-1, both arms run the full iteration count from one
    initial cluster; reported per seed: NMI against the generating labels, final cluster count and
    seconds; and the means, spreads and the largest |NMI difference| over the seeds."""
    import numpy as np
    import torch
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    from dpmmsubclusters_gpu_b200.capi import check, lib
    L = lib()
    shapes = {
        "c5r": dict(desc="C5 shape at N=1e6: D=64, 100 true clusters, means N(0,25I), cov AA^T/D+0.5I, Dir(2) "
                         "weights; NIW k=1 m=0 nu=67 Psi=I; alpha=10; 150 iterations, burnout 15",
                    iters=150, burnout=15, alpha=10.0),
        "c2": dict(desc="C2 shape: N=1e6, D=32, 20 true clusters, means U(-20,20)^D, cov AA^T/D+0.5I, Dir(1) "
                        "weights; NIW k=1 m=0 nu=35 Psi=I; alpha=10; 200 iterations, burnout 20",
                   iters=200, burnout=20, alpha=10.0),
    }
    out = {"metric": "end-to-end NMI and final cluster count over sampler seeds: mixed+learned vs plain FP32",
           "unit": "NMI", "data": "synthetic (seeded draws of each shape's generative model, on device)",
           "impl": "ours", "shapes": {}}
    for name in args.study_shapes.split(","):
        sh = shapes[name]
        if name == "c5r":
            cfg = dict(N=1_000_000, D=64, K_true=100, alpha=10.0, nu=67.0, kappa=1.0, iterations=sh["iters"],
                       mean_sd=5.0, dirichlet=2.0)
            x, z = generate_c5_torch(cfg, 1105, f"cuda:{local}")
        else:
            cfg = dict(N=1_000_000, D=32, K_true=20, alpha=10.0, nu=35.0, kappa=1.0, iterations=sh["iters"])
            x, z = generate_c2_torch(1102, f"cuda:{local}")
        z_np = z.cpu().numpy()
        res = {}
        for arm in ("mixed", "plain"):
            # one untimed short run first: the process's first sampler teardown carries a one-time cost
            # of the driver (about 0.9 s on the B200) that is no part of a run
            keep = []
            a = argparse.Namespace(initial_clusters=1, multi_gpu="replicas")
            rd = make_run_desc(cfg, a, arm, 5, 0, local, keep)
            h = ctypes.c_void_p()
            check(L.dpmm_sampler_create(ctypes.byref(rd), cfg["N"], cfg["D"], ctypes.c_void_p(x.data_ptr()), 1,
                                        ctypes.byref(h)))
            check(L.dpmm_sampler_step(h, 5))
            check(L.dpmm_sampler_destroy(h))
            rows = []
            for seed in range(args.study_seeds):
                keep = []
                a = argparse.Namespace(initial_clusters=1, multi_gpu="replicas")
                rd = make_run_desc(cfg, a, arm, sh["iters"], 0, local, keep)
                rd.seed = seed + 1          # seed 0 would mean "time based"
                rd.burnout = sh["burnout"]
                rd.alpha = sh["alpha"]
                h = ctypes.c_void_p()
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                check(L.dpmm_sampler_create(ctypes.byref(rd), cfg["N"], cfg["D"], ctypes.c_void_p(x.data_ptr()), 1,
                                            ctypes.byref(h)))
                check(L.dpmm_sampler_step(h, sh["iters"]))
                kk = ctypes.c_int32()
                check(L.dpmm_sampler_num_clusters(h, ctypes.byref(kk)))
                mi = ctypes.c_void_p()
                check(L.dpmm_sampler_model_info(h, ctypes.byref(mi)))
                lab = np.ctypeslib.as_array(L.dpmm_model_info_labels(mi), shape=(cfg["N"],)).copy()
                L.dpmm_model_info_free(mi)
                check(L.dpmm_sampler_destroy(h))
                torch.cuda.synchronize()
                dt = time.perf_counter() - t0
                rows.append({"seed": seed + 1, "nmi": _nmi(lab, z_np), "final_k": kk.value, "seconds": dt})
            nm = np.array([r["nmi"] for r in rows])
            ks = np.array([r["final_k"] for r in rows])
            res[arm] = {"runs": rows, "nmi_mean": float(nm.mean()), "nmi_std": float(nm.std()),
                        "final_k_mean": float(ks.mean()), "final_k_std": float(ks.std()),
                        "final_k_values": sorted(int(k) for k in ks),
                        "seconds_mean": float(np.mean([r["seconds"] for r in rows]))}
        dn = [abs(a["nmi"] - b["nmi"]) for a, b in zip(res["mixed"]["runs"], res["plain"]["runs"])]
        out["shapes"][name] = {"workload": sh["desc"], "true_clusters": cfg["K_true"], "arms": res,
                               "nmi_mean_difference": res["mixed"]["nmi_mean"] - res["plain"]["nmi_mean"],
                               "max_abs_nmi_difference_same_seed": float(max(dn)),
                               "speedup_mean_seconds": res["plain"]["seconds_mean"] / res["mixed"]["seconds_mean"]}
        del x
        torch.cuda.empty_cache()
    print(json.dumps(out), flush=True)
    return 0


def run_c4(args, rank, world, local):
    """Batched uneven data sets: all data sets advanced together by BatchSampler (one label launch per
    padded dimension per iteration, CUDA-graph replayed) vs a subset of the same data sets run one at a
    time through dp_parallel; throughput = sum of N x iterations / wall time of the sampler loop."""
    import numpy as np
    import torch
    from dpmmsubclusters_gpu_b200 import BatchSampler, capi, niw_hyperparams, prior_type
    from dpmmsubclusters_gpu_b200.api import dp_parallel_sampling_class
    torch.cuda.set_device(local)
    iters = 100
    data = c4_data(args.c4_sets, 1004 + rank)
    hyp = [niw_hyperparams(1.0, np.zeros(x.shape[0]), x.shape[0] + 3.0, np.eye(x.shape[0])) for x, _ in data]
    npts = np.array([x.shape[1] for x, _ in data], dtype=np.float64)
    b = BatchSampler([x for x, _ in data], hyp, 5.0, iters=iters, init_clusters=1, burnout=15, k_max=64,
                     device=local)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b.step(iters)
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - t0
    info = b.info()
    nmis = [_nmi(b.model_info(i).labels, z) for i, (_, z) in enumerate(data)]
    b.close()
    m = min(args.c4_seq_sets, len(data))
    t0 = time.perf_counter()
    for i in range(m):
        x = data[i][0]
        s = dp_parallel_sampling_class(x.shape[1], x, 1 + i, prior_type.Gaussian, loglik_mode=capi.LL_FP32,
                                       k_max=64, device=local)
        s.dp_parallel(hyp[i], 5.0, iters=iters, init_clusters=1, verbose=False, burnout=15)
    torch.cuda.synchronize()
    t_seq = time.perf_counter() - t0
    line = {"metric": "batched uneven data sets: points*iters/sec (all data sets advanced together)",
            "value": float(npts.sum() * iters / t_batch), "unit": UNIT, "n_gpus": world, "steps": iters,
            "warmup": 0, "ms_per_step": t_batch / iters * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded, host)",
            "config": {"workload": "C4: %d data sets, N ~ logU[1e3, 2e5], D in {2, 8, 16, 64}, K* ~ U{2..30}, "
                                   "NIW k=1 m=0 nu=D+3 Psi=I, alpha=5, %d iterations" % (len(data), iters),
                       "total_points": int(npts.sum()), "batch_info": info,
                       "nmi_mean": float(np.mean(nmis)), "nmi_min": float(np.min(nmis)),
                       "timing": "wall clock around the sampler loop (setup and data upload excluded)"},
            "one_at_a_time": {"data_sets": m, "value": float(npts[:m].sum() * iters / t_seq), "unit": UNIT,
                              "wall_s": t_seq},
            "batch_wall_s": t_batch}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def screen_summary(flag, st):
    """counters of the learned split/merge screen over the whole run (burn-in included)"""
    if flag != "on":
        return {"enabled": False}
    keys = ("split_candidates", "split_exact", "merge_candidates", "merge_exact", "sweeps", "sweep_accepts",
            "sweep_hits", "disabled_at")
    d = {k: int(v) for k, v in zip(keys, st)}
    d["enabled"] = True
    d["top"], d["sweep_every"], d["split_min_candidates"] = 16, 10, 256
    d["sweep_recall"] = d["sweep_hits"] / d["sweep_accepts"] if d["sweep_accepts"] else None
    return d


def _nmi(a, b):
    import numpy as np
    ua, ia = np.unique(a, return_inverse=True)
    ub, ib = np.unique(b, return_inverse=True)
    c = np.zeros((ua.size, ub.size))
    np.add.at(c, (ia, ib), 1)
    p = c / c.sum()
    pa, pb = p.sum(1), p.sum(0)
    h = lambda q: -np.sum(q[q > 0] * np.log(q[q > 0]))
    nz = p > 0
    mi = np.sum(p[nz] * np.log(p[nz] / np.outer(pa, pb)[nz]))
    return float(2 * mi / (h(pa) + h(pb)))


if __name__ == "__main__":
    sys.exit(main())

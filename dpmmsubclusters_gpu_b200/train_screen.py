"""Train the learned split/merge screen on the device and write its parameters.

    python -m dpmmsubclusters_gpu_b200.train_screen [--out DIR] [--quick]

Training data are the screen's own features with the exact FP64 log Hastings ratio of every split
candidate and every cluster pair, logged (screen_mode DPMM_SCREEN_LOG) by the plain sampler -- every
candidate evaluated exactly, as the reference does -- on seeded synthetic data of two shapes:

  gaussian  D = 2, 2 true clusters, means U(-100, 100)^D, covariances A A^T + I (A ~ N(0, 1)), equal
            weights, float64, N = 100,000; NIW(kappa 1, m 0, nu 5, Psi I), alpha 1
  counts    multinomial D = 1000, 50 components, theta ~ Dir(0.1), weights ~ Dir(1), lengths ~
            Poisson(200), Dirichlet(1) prior, alpha 10; N = 50,000 points per run (the shape's 1e6
            points are not needed for candidate statistics and would only slow the logging runs)

Runs start from several initial cluster counts so that splits and merges of every kind occur.  Runs
are split 80 / 20 into training and held-out sets; the network (dpmm_screen_train: the library's own
forward / backward / Adam kernels) regresses clamp(log ratio, -30, 10) / 10.  The held-out report
gives, per (run, iteration, kind) group, the recall@16 of candidates with log ratio > -1 under the
trained network, under the proxy feature alone, and under a random order.

Output: screen_params.f32 (raw FP32, DPMM_SCREEN_PARAMS values) and screen_params.json (report).
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import capi, screen
from .api import dp_parallel_sampling_class, multinomial_hyper, niw_hyperparams, prior_type

TOP = 16


def gaussian_shape(seed: int, n: int = 100_000, d: int = 2, k: int = 2):
    rng = np.random.default_rng(seed)
    mus = rng.uniform(-100, 100, size=(k, d))
    z = rng.integers(0, k, size=n)
    x = np.empty((n, d))
    for c in range(k):
        a = rng.normal(size=(d, d))
        idx = np.flatnonzero(z == c)
        x[idx] = rng.multivariate_normal(mus[c], a @ a.T + np.eye(d), size=idx.size)
    return x, z


def counts_shape(seed: int, n: int = 50_000, d: int = 1000, k: int = 50):
    rng = np.random.default_rng(seed)
    theta = rng.dirichlet(np.full(d, 0.1), size=k)
    w = rng.dirichlet(np.ones(k))
    z = rng.choice(k, size=n, p=w)
    lengths = rng.poisson(200, size=n)
    x = np.empty((n, d))
    for c in range(k):
        idx = np.flatnonzero(z == c)
        if idx.size:
            x[idx] = rng.multinomial(lengths[idx], theta[c])
    return x, z


def mixture_shape(seed: int, n: int, d: int, k: int, mean: str):
    """The C2 / C5 generative shapes (evaluation only): means U(-20, 20)^D (C2) or N(0, 25 I) (C5),
    covariances A A^T / D + 0.5 I, Dirichlet(1) (C2) or Dirichlet(2) (C5) weights."""
    rng = np.random.default_rng(seed)
    mus = rng.uniform(-20, 20, size=(k, d)) if mean == "uniform" else rng.normal(size=(k, d)) * 5.0
    w = rng.dirichlet(np.full(k, 1.0 if mean == "uniform" else 2.0))
    z = rng.choice(k, size=n, p=w)
    x = np.empty((n, d))
    for c in range(k):
        a = rng.normal(size=(d, d))
        idx = np.flatnonzero(z == c)
        x[idx] = rng.multivariate_normal(mus[c], a @ a.T / d + 0.5 * np.eye(d), size=idx.size)
    return x, z


def log_run(kind: str, seed: int, init_clusters: int, iters: int):
    if kind in ("c2", "c5"):
        x, _ = (mixture_shape(5000 + seed, 100_000, 32, 20, "uniform") if kind == "c2"
                else mixture_shape(6000 + seed, 100_000, 64, 100, "normal"))
        d = x.shape[1]
        hyper = niw_hyperparams(1.0, np.zeros(d), d + 3.0, np.eye(d))
        alpha, prior = 10.0, prior_type.Gaussian
    elif kind == "gaussian":
        x, _ = gaussian_shape(1000 + seed)
        d = x.shape[1]
        hyper = niw_hyperparams(1.0, np.zeros(d), 5.0, np.eye(d))
        alpha, prior = 1.0, prior_type.Gaussian
    else:
        x, _ = counts_shape(3000 + seed)
        d = x.shape[1]
        hyper = multinomial_hyper(np.ones(d))
        alpha, prior = 10.0, prior_type.Multinomial
    s = dp_parallel_sampling_class(x.shape[0], x.T, seed + 1, prior, screen_mode=capi.SCREEN_LOG)
    mi = s.dp_parallel(hyper, alpha, iters=iters, init_clusters=init_clusters, verbose=False, burnout=5)
    return mi.screen_log


def recall_at_top(groups, score, hr, top=TOP, thresh=-1.0):
    """Share of the attainable positives (log ratio > thresh) that the `top` best scores of their
    group hold: sum of hits / sum of min(top, positives) over groups with a positive."""
    hits = total = 0
    for g in groups:
        pos = g[hr[g] > thresh]
        if pos.size == 0:
            continue
        order = g[np.lexsort((g, -score[g]))][:top]
        hits += np.isin(pos, order).sum()
        total += min(top, pos.size)
    return (hits / total if total else float("nan")), int(total)


def ranking_report(groups, score, hr, thresh=-1.0):
    """How well a ranking finds the candidates worth an exact ratio (log ratio > thresh), per group
    (run, iteration, kind): recall within the top k for k = 1 .. 16, and the exact evaluations needed to
    reach every positive of a group (the rank of its last positive), summed over the groups."""
    out = {f"recall_at_{k}": recall_at_top(groups, score, hr, top=k, thresh=thresh)[0] for k in (1, 2, 4, 8, 16)}
    need = 0
    for g in groups:
        pos = hr[g] > thresh
        if not pos.any():
            continue
        order = np.lexsort((g, -score[g]))
        need += int(np.flatnonzero(pos[order]).max()) + 1
    out["evaluations_to_reach_every_positive"] = need
    out["candidates"] = int(sum(len(g) for g in groups if (hr[g] > thresh).any()))
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=screen.HERE)
    ap.add_argument("--quick", action="store_true", help="fewer runs (smoke test of the pipeline)")
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--dump", default=None, help="also write the logged rows to this .npz")
    args = ap.parse_args(argv)
    t0 = time.time()
    # training shapes (C1: D = 2 Gaussian; C3: D = 1000 counts), then evaluation-only shapes the network
    # never sees in training (C2: D = 32; C5: D = 64): does the ranking carry over?
    plan = [("gaussian", s, ic, 100) for s, ic in enumerate([1, 4, 8, 16, 24, 32, 6, 12, 20, 28, 2, 10, 14, 18, 26,
                                                              30, 36, 40, 3, 22])]
    plan += [("counts", s, ic, 60) for s, ic in enumerate([1, 10, 30, 60, 20, 5, 40, 80])]
    evals = [("c2", s, ic, 60) for s, ic in enumerate([1, 8, 30])] + [("c5", s, ic, 40) for s, ic in enumerate([1, 50, 150])]
    if args.quick:
        plan = [("gaussian", 0, 8, 30), ("gaussian", 1, 16, 30), ("counts", 0, 10, 15)]
        evals = [("c2", 0, 8, 20)]
    plan = plan + evals
    runs = []
    for i, (kind, seed, ic, iters) in enumerate(plan):
        lg = log_run(kind, seed, ic, iters)
        if lg is None:
            continue
        f, hr, kd, it = lg
        runs.append({"kind": kind, "seed": seed, "init": ic, "f": f, "hr": hr, "k": kd, "it": it, "run": i})
        print(f"[log] {kind} seed {seed} init {ic}: {hr.size} rows ({(kd == 1).sum()} merge)", flush=True)
    if args.dump:
        np.savez_compressed(args.dump, **{f"{k}_{i}": r[k] for i, r in enumerate(runs) for k in ("f", "hr", "k", "it")},
                            meta=np.array([[r["run"], r["seed"], r["init"], r["kind"] == "gaussian"] for r in runs]))
    rng = np.random.default_rng(args.seed)
    train_idx = [i for i, r in enumerate(runs) if r["kind"] in ("gaussian", "counts")]
    eval_idx = [i for i, r in enumerate(runs) if r["kind"] in ("c2", "c5")]
    held = set(rng.choice(train_idx, size=max(1, len(train_idx) // 5), replace=False).tolist())

    def stack(sel):
        rs = [runs[i] for i in sel]
        F = np.concatenate([r["f"] for r in rs])
        HR = np.concatenate([r["hr"] for r in rs])
        G = np.concatenate([r["run"] * 1_000_000 + r["it"] * 2 + r["k"] for r in rs])
        return F, HR, G

    Ftr, HRtr, _ = stack([i for i in train_idx if i not in held])
    Fte, HRte, Gte = stack(sorted(held))
    # rows far below acceptance carry one target value (-3); keep all rows near it and a share of the rest
    near = HRtr > -60
    keep = near | (rng.random(HRtr.size) < 0.25)
    Ftr, HRtr = Ftr[keep], HRtr[keep]
    p0 = screen.init_params(args.seed)
    params, losses = screen.train(Ftr, screen.target(HRtr), p0, epochs=args.epochs, batch=256, lr=2e-3,
                                  seed=args.seed)
    score = screen.forward(Fte, params)
    groups = [np.flatnonzero(Gte == g) for g in np.unique(Gte)]
    r_net, npos = recall_at_top(groups, score, HRte)
    r_proxy, _ = recall_at_top(groups, Fte[:, 2].astype(np.float64), HRte)
    r_rand, _ = recall_at_top(groups, rng.random(HRte.size), HRte)
    r_init, _ = recall_at_top(groups, screen.forward(Fte, p0), HRte)
    shape_g = {sh: [g for g in groups if (Fte[g[0], 1] > 0) == (sh == "gaussian")] for sh in ("gaussian", "counts")}
    per_shape = {sh: {"trained": recall_at_top(gs, score, HRte)[0],
                      "proxy_feature_only": recall_at_top(gs, Fte[:, 2].astype(np.float64), HRte)[0],
                      "attainable_positives": recall_at_top(gs, score, HRte)[1]} for sh, gs in shape_g.items()}
    # the rankings on the held-out runs of the training shapes and on the evaluation-only shapes
    comparison = {}
    for name, sel in [("held_out_C1_C3_shapes", sorted(held))] + [
            (f"unseen_{sh}_shape", [i for i in eval_idx if runs[i]["kind"] == sh]) for sh in ("c2", "c5")]:
        if not sel:
            continue
        F, HR, G = stack(sel)
        gs = [np.flatnonzero(G == g) for g in np.unique(G)]
        comparison[name] = {"trained": ranking_report(gs, screen.forward(F, params), HR),
                            "proxy_feature_only": ranking_report(gs, F[:, 2].astype(np.float64), HR),
                            "untrained_init": ranking_report(gs, screen.forward(F, p0), HR),
                            "random_order": ranking_report(gs, rng.random(HR.size), HR),
                            "rows": int(HR.size), "groups": len(gs)}
    os.makedirs(args.out, exist_ok=True)
    screen.save_params(params, os.path.join(args.out, "screen_params.f32"))
    report = {
        "runs": [{"shape": r["kind"], "seed": r["seed"], "initial_clusters": r["init"], "rows": int(r["hr"].size),
                  "held_out": i in held} for i, r in enumerate(runs)],
        "train_rows": int(HRtr.size), "held_out_rows": int(HRte.size), "epochs": args.epochs, "batch": 256,
        "lr": 2e-3, "epoch_loss": [float(v) for v in losses],
        "held_out_recall_at_16": {"trained": r_net, "proxy_feature_only": r_proxy, "untrained_init": r_init,
                                  "random_order": r_rand, "attainable_positives": npos,
                                  "positive": "log ratio > -1", "groups": len(groups), "per_shape": per_shape,
                                  "definition": "hits / sum over groups of min(16, positives); group = "
                                                "(run, iteration, kind)"},
        "ranking_comparison": comparison,
        "seconds": round(time.time() - t0, 1),
    }
    with open(os.path.join(args.out, "screen_params.json"), "w") as fh:
        json.dump(report, fh, indent=1)
    print(json.dumps(report["held_out_recall_at_16"]), flush=True)
    print(json.dumps(comparison), flush=True)
    print(f"[train] final loss {losses[-1]:.5f}, {report['seconds']} s", flush=True)


if __name__ == "__main__":
    main()

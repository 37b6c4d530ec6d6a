"""Time the reference's own GPU executable against this library on the same input (test infrastructure).

    python oracle/compare_reference_gpu.py [--n 1000000] [--d 32] [--k 20] [--iters 60] [--out DIR]

Writes a seeded synthetic data set of the C2 shape (means U(-20, 20)^D, covariances A A^T / D + 0.5 I,
Dirichlet(1) weights) as a float64 N x D .npy (the layout the reference's loader reads correctly) and a
params JSON (NIW kappa 1, m 0, nu D + 3, Psi I; alpha 10; burn-out period 15, so that clusters split
from the 16th iteration on), runs the reference executable built from its
sources by oracle/Makefile (oracle/_ref/dpmm_ref, sm_100a) with --model_path / --params_path /
--result_path, and this library's dp_parallel_from_file on the same two files, and prints one JSON line:
seconds per iteration (the reference's own iter_count; this library's iteration times), points x
iterations / s, the final cluster count and the NMI against the generating labels of each.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
REF_EXE = os.path.join(HERE, "_ref", "dpmm_ref")


def c2_data(n, d, k, seed):
    rng = np.random.default_rng(seed)
    w = rng.dirichlet(np.ones(k))
    mus = rng.uniform(-20, 20, size=(k, d))
    z = rng.choice(k, size=n, p=w)
    x = np.empty((n, d))
    for c in range(k):
        idx = np.flatnonzero(z == c)
        a = rng.normal(size=(d, d))
        L = np.linalg.cholesky(a @ a.T / d + 0.5 * np.eye(d))
        x[idx] = mus[c] + rng.normal(size=(idx.size, d)) @ L.T
    return x, z


def nmi(a, b):
    from sklearn.metrics import normalized_mutual_info_score
    return float(normalized_mutual_info_score(a, b))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--d", type=int, default=32)
    ap.add_argument("--k", type=int, default=20)
    ap.add_argument("--iters", type=int, default=60)
    ap.add_argument("--seed", type=int, default=1102)
    ap.add_argument("--out", default="/tmp/dpmm_compare")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    x, z = c2_data(args.n, args.d, args.k, args.seed)
    npy, pj, rj = (os.path.join(args.out, f) for f in ("x.npy", "params.json", "result.json"))
    np.save(npy, x)
    with open(pj, "w") as f:
        json.dump({"alpha": 10.0, "iterations": args.iters, "burnout_period": 15, "outlier_mod": 0.0,
                   "randomSeed": 7, "initial_clusters": 1,
                   "hyper_params": {"k": 1.0, "m": [0.0] * args.d, "v": args.d + 3.0,
                                    "psi": np.eye(args.d).tolist()}}, f)
    out = {"workload": f"C2 shape: N={args.n}, D={args.d}, {args.k} true clusters, float64 .npy, "
                       f"{args.iters} iterations from one cluster (burn-out 15), alpha 10, NIW(1, 0, D+3, I)"}
    if os.path.exists(REF_EXE):
        t0 = time.perf_counter()
        p = subprocess.run([REF_EXE, f"--model_path={npy}", f"--params_path={pj}", "--prior_type=Gaussian",
                            f"--result_path={rj}"], capture_output=True, text=True, timeout=3600)
        wall = time.perf_counter() - t0
        if p.returncode == 0:
            r = json.load(open(rj))
            it = np.array(r["iter_count"], dtype=np.float64)
            lab = np.array(r["labels"])
            out["reference_gpu_build"] = {"s_per_iteration": float(it.mean()),
                                          "points_iters_per_s": args.n / float(it.mean()),
                                          "final_clusters": int(len(np.unique(lab))), "nmi": nmi(lab, z),
                                          "process_wall_s": wall}
        else:
            out["reference_gpu_build"] = {"failed": (p.stdout + p.stderr)[-400:]}
    else:
        out["reference_gpu_build"] = {"failed": "oracle/_ref/dpmm_ref not built"}
    from dpmmsubclusters_gpu_b200 import dp_parallel_sampling_class, prior_type
    t0 = time.perf_counter()
    mi = dp_parallel_sampling_class(npy, pj, prior_type.Gaussian).dp_parallel_from_file()
    wall = time.perf_counter() - t0
    it = np.asarray(mi.iter_count, dtype=np.float64)
    out["this_library"] = {"s_per_iteration": float(it.mean()), "points_iters_per_s": args.n / float(it.mean()),
                           "final_clusters": int(len(np.unique(mi.labels))), "nmi": nmi(mi.labels, z),
                           "call_wall_s": wall}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()

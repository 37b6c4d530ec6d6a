"""Extract the reference's own golden vectors for the hot path into reference_goldens.json.

Reads the reference's GoogleTest sources as TEXT (they are not compiled or run) and
records, per test, the comma-initialised inputs (``name << a, b, ...;``) and the
expectations (``EXPECT_NEAR(value, expr, tol)`` / ``ASSERT_NEAR`` / ``EXPECT_EQ``).

    python tests/golden/make_golden.py [REFERENCE_DIR]

The default reference directory is the read-only mount used while building this
project; the output is committed so that tests never need the reference at run time.
Tests covered (paths relative to the reference's DPMMSubClusters/ directory):
  test/cudaKernel_gaussian_test.cpp     log_likelihood, log_likelihood_ignore_weight,
                                        log_likelihood_sigma_is_identity, alias count tests
  test/cudaKernel_multinomial_test.cpp  log_likelihood_labels
  test/local_clusters_actions_test.cpp  update_suff_stats_posterior, should_split_local,
                                        create_suff_stats_dict_worker
  test/niw_test.cpp                     CreateSufficientStatistics, CalcPosterior,
                                        LogMarginalLikelihood_Dim3, LogMarginalLikelihood_Dim50
  test/multinomial_prior_test.cpp       CreateSufficientStatistics, LogMarginalLikelihood,
                                        AggregateSuffStats
"""
from __future__ import annotations

import json
import os
import re
import sys

# the reference checkout: argv[1], else $DPMM_REFERENCE_DIR, else `reference/` beside this repository
DEFAULT_REF = os.environ.get("DPMM_REFERENCE_DIR") or os.path.join(
    os.path.dirname(os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))),
    "reference", "DPMMSubClusters")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_goldens.json")

WANTED = {
    "test/cudaKernel_gaussian_test.cpp": [
        "sample_log_cat_array_less_prob_for_one", "sample_log_cat_array_less_prob_for_two",
        "sample_log_cat_array_sub_cluster_less_prob_for_one_all_indices",
        "sample_log_cat_array_sub_cluster_less_prob_for_one_few_indices",
        "log_likelihood", "log_likelihood_ignore_weight", "log_likelihood_sigma_is_identity"],
    "test/cudaKernel_multinomial_test.cpp": ["log_likelihood_labels"],
    "test/local_clusters_actions_test.cpp": [
        "update_suff_stats_posterior", "should_split_local", "create_suff_stats_dict_worker"],
    "test/niw_test.cpp": ["CreateSufficientStatistics", "CalcPosterior", "LogMarginalLikelihood_Dim3",
                          "LogMarginalLikelihood_Dim50"],
    "test/multinomial_prior_test.cpp": ["CreateSufficientStatistics", "LogMarginalLikelihood",
                                        "AggregateSuffStats"],
}

NUM = r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?f?"


def _num(s: str) -> float:
    return float(s.rstrip("f"))


def test_bodies(src: str):
    """Yield (name, body) for each TEST(...) block by brace matching."""
    for m in re.finditer(r"TEST\(\s*\w+\s*,\s*(\w+)\s*\)\s*\{", src):
        i = m.end()
        depth = 1
        while depth and i < len(src):
            if src[i] == "{":
                depth += 1
            elif src[i] == "}":
                depth -= 1
            i += 1
        yield m.group(1), src[m.end():i - 1]


def parse_body(body: str):
    rec = {"inits": [], "scalars": {}, "expect": []}
    for m in re.finditer(r"([\w\->\.\(\)]+?)\s*<<\s*([^;]+);", body):
        vals = [v.strip() for v in m.group(2).split(",")]
        try:
            nums = [_num(v) for v in vals]
        except ValueError:
            continue
        rec["inits"].append({"name": m.group(1).strip(), "values": nums})
    for m in re.finditer(r"(?:double|int|float)\s+(\w+)\s*=\s*(" + NUM + r")\s*;", body):
        rec["scalars"][m.group(1)] = _num(m.group(2))
    for m in re.finditer(r"(EXPECT|ASSERT)_NEAR\(\s*(" + NUM + r")\s*,\s*(.+?)\s*,\s*(" + NUM + r")\s*\)\s*;", body):
        rec["expect"].append({"kind": "near", "value": _num(m.group(2)), "expr": m.group(3).strip(),
                              "tol": _num(m.group(4))})
    for m in re.finditer(r"(EXPECT|ASSERT)_EQ\(\s*(" + NUM + r")\s*,\s*([^)]+?)\s*\)", body):
        rec["expect"].append({"kind": "eq", "value": _num(m.group(2)), "expr": m.group(3).strip()})
    for m in re.finditer(r"make_shared<niw_hyperparams>\(\s*(" + NUM + r")\s*,\s*(\w+)\s*,\s*(\w+|" + NUM +
                         r")\s*,\s*(\w+)\s*\)", body):
        rec.setdefault("niw_ctor", []).append([m.group(1), m.group(2), m.group(3), m.group(4)])
    for m in re.finditer(r"niw_hyperparams\s+(\w+)\(\s*(" + NUM + r")\s*,\s*(\w+)\s*,\s*(" + NUM +
                         r")\s*,\s*(\w+)\s*\)", body):
        rec.setdefault("niw_objs", {})[m.group(1)] = [_num(m.group(2)), m.group(3), _num(m.group(4)), m.group(5)]
    for m in re.finditer(r"suff_statistics->N\s*=\s*(\d+)\s*;", body):
        rec.setdefault("suff_N", []).append(int(m.group(1)))
    for m in re.finditer(r"make_shared<(?:niw|multinomial)_sufficient_statistics>\(\s*(" + NUM + r")", body):
        rec.setdefault("ss_ctor_N", []).append(_num(m.group(1)))
    for m in re.finditer(r"std::vector<int>\s+(\w+)\s*=\s*\{([^}]*)\}", body):
        rec.setdefault("int_vectors", {})[m.group(1)] = [int(v) for v in m.group(2).split(",")]
    for m in re.finditer(r"alpha\.push_back\(\s*(" + NUM + r")\s*\)", body):
        rec.setdefault("alpha_push", []).append(_num(m.group(1)))
    for m in re.finditer(r"log_likelihood_array\w*\(i,\s*(\d)\)\s*=\s*(" + NUM + r")\s*;", body):
        rec.setdefault("loglik_fill", {})[m.group(1)] = _num(m.group(2))
    return rec


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else DEFAULT_REF
    out = {"source": "BGU-CS-VIL/DPMMSubClusters_GPU DPMMSubClusters/test (read as text)", "tests": {}}
    for rel, names in WANTED.items():
        with open(os.path.join(ref, rel)) as f:
            src = f.read()
        bodies = dict(test_bodies(src))
        for name in names:
            rec = parse_body(bodies[name])
            rec["file"] = rel
            out["tests"][f"{os.path.basename(rel)[:-4]}::{name}"] = rec
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", OUT, len(out["tests"]), "tests")


if __name__ == "__main__":
    main()

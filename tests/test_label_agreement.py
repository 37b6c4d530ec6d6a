"""Host part of the verbose-mode label agreement (dpmm_nmi_from_table): NMI = 2 I / (H(X) + H(Y)) as
dp_parallel_sampling.cpp:171-179 computes it, and the variation of information, from a contingency
table, against scikit-learn's arithmetic-mean NMI and a numpy restatement on the expanded labels."""
import numpy as np
import pytest
from sklearn.metrics import normalized_mutual_info_score

from dpmmsubclusters_gpu_b200.api import nmi_from_table
from dpmmsubclusters_gpu_b200.capi import DpmmError


def _expand(table):
    a, b = [], []
    for k in range(table.shape[0]):
        for g in range(table.shape[1]):
            a += [k] * int(table[k, g])
            b += [g] * int(table[k, g])
    return np.array(a), np.array(b)


def _vi(a, b):
    n = a.size
    _, ia = np.unique(a, return_inverse=True)
    _, ib = np.unique(b, return_inverse=True)
    joint = np.zeros((ia.max() + 1, ib.max() + 1))
    np.add.at(joint, (ia, ib), 1)
    p = joint / n
    pa, pb = p.sum(1), p.sum(0)
    h = lambda q: -np.sum(q[q > 0] * np.log(q[q > 0]))
    nz = p > 0
    mi = np.sum(p[nz] * np.log(p[nz] / np.outer(pa, pb)[nz]))
    return h(pa) + h(pb) - 2 * mi


@pytest.mark.parametrize("K,G,seed", [(3, 2, 0), (10, 7, 1), (40, 40, 2), (1, 5, 3)])
def test_table_scores_match_sklearn(K, G, seed):
    rng = np.random.default_rng(seed)
    table = rng.integers(0, 50, size=(K, G))
    table[rng.random(table.shape) < 0.3] = 0
    table[0, 0] += 1
    a, b = _expand(table)
    nmi, vi = nmi_from_table(table)
    assert abs(nmi - normalized_mutual_info_score(b, a)) <= 1e-12
    assert abs(vi - _vi(a, b)) <= 1e-10


def test_single_class_scores_one():
    assert nmi_from_table(np.array([[7]])) == (1.0, 0.0)


def test_empty_table_is_rejected():
    with pytest.raises(DpmmError):
        nmi_from_table(np.zeros((3, 3), np.int64))

"""The split-TF32 operands of the tensor-core statistics kernel (csrc/dpmm_tc.cu tf32_rna and the
hi / lo split of k_slot_stats_tc), restated with numpy bit operations: rounding to 10 explicit
mantissa bits by adding half of the dropped 13-bit field and clearing it is round-to-nearest with ties
away from zero, and c = hi + lo + e with |e| <= 2^-22 |c| (so the three products hi*hi + lo*hi +
hi*lo carry the Gram sums at FP32-level accuracy)."""
import numpy as np


def tf32_rna(v):
    b = np.asarray(v, np.float32).view(np.uint32)
    return ((b + np.uint32(0x1000)) & np.uint32(0xFFFFE000)).view(np.float32)


def test_rounding_is_nearest_ties_away():
    rng = np.random.default_rng(0)
    v = (rng.normal(size=200000) * np.exp(rng.uniform(-30, 30, size=200000))).astype(np.float32)
    r = tf32_rna(v).astype(np.float64)
    ulp = np.ldexp(1.0, np.frexp(np.abs(v).astype(np.float64))[1] - 11)   # 10 explicit bits
    err = np.abs(r - v.astype(np.float64))
    assert np.all(err <= ulp / 2 * (1 + 1e-12))
    # representable in 10 explicit bits: the low 13 bits are clear
    assert np.all((tf32_rna(v).view(np.uint32) & np.uint32(0x1FFF)) == 0)
    # ties (exactly half an ulp above a tf32 value) go away from zero
    base = tf32_rna(np.float32(1.5))
    tie = (base.view(np.uint32) + np.uint32(0x1000)).view(np.float32)
    assert tf32_rna(tie) > tie and tf32_rna(-tie) < -tie


def test_two_term_split_error_bound():
    rng = np.random.default_rng(1)
    c = (rng.normal(size=500000) * np.exp(rng.uniform(-20, 20, size=500000))).astype(np.float32)
    hi = tf32_rna(c)
    lo = tf32_rna((c - hi).astype(np.float32))
    e = np.abs(c.astype(np.float64) - hi.astype(np.float64) - lo.astype(np.float64))
    assert np.all(e <= 2.0 ** -22 * np.abs(c.astype(np.float64)))

"""Comparison metric of the reference's translate tests
(fv3core tests/savepoint/test_translate.py:26-76): relative difference
2|a-b|/(|a|+|b|), NaN equal to NaN, and values below ``near_zero`` in both
arrays treated as equal."""
import numpy as np


def compare_arr(computed, ref):
    computed = np.asarray(computed, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        denom = np.abs(computed) + np.abs(ref)
        out = np.where(denom > 0, 2.0 * np.abs(computed - ref) / np.where(denom > 0, denom, 1.0), 0.0)
    both_nan = np.isnan(computed) & np.isnan(ref)
    return np.where(both_nan, 0.0, out)


def max_rel_err(computed, ref, near_zero=1e-18):
    err = compare_arr(computed, ref)
    small = (np.abs(np.asarray(computed)) < near_zero) & (np.abs(np.asarray(ref)) < near_zero)
    err = np.where(small, 0.0, err)
    if np.any(np.isnan(err)):
        return float("inf")
    return float(err.max()) if err.size else 0.0


def parity_err(computed, ref, near_zero_frac=1e-6):
    """Relative error used for CUDA-vs-oracle parity: the translate-test
    metric 2|a-b|/(|a|+|b|), except that points where the reference value is
    smaller than ``near_zero_frac`` times the field's largest magnitude are
    measured against that magnitude floor instead (values crossing zero carry
    cancellation error of order the field's scale times machine epsilon,
    which a pointwise relative measure would amplify without bound).
    NaN must coincide with NaN."""
    a = np.asarray(computed, dtype=np.float64)
    b = np.asarray(ref, dtype=np.float64)
    nan_a, nan_b = np.isnan(a), np.isnan(b)
    if np.any(nan_a != nan_b):
        return float("inf")
    a = np.where(nan_a, 0.0, a)
    b = np.where(nan_b, 0.0, b)
    scale = float(np.max(np.abs(b))) if b.size else 0.0
    if scale == 0.0:
        return float(np.max(np.abs(a))) if a.size else 0.0
    floor = near_zero_frac * scale
    denom = np.maximum(0.5 * (np.abs(a) + np.abs(b)), floor)
    return float(np.max(np.abs(a - b) / denom))

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

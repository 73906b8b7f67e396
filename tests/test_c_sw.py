"""CGridShallowWaterDynamics (with d2a2c_vect): oracle vs the reference's
golden output; CUDA vs oracle."""
import os

import numpy as np
import pytest

import cases
import oracle_runs
from metrics import max_rel_err, parity_err

OUT = ["delp", "pt", "w", "uc", "vc", "ua", "va", "ut", "vt", "divgd", "omga", "delpc", "ptc"]
HERE = os.path.dirname(os.path.abspath(__file__))


def _compare_full(a, b):
    """Max relative error over the whole storage; NaN must match NaN."""
    nan_a, nan_b = np.isnan(a), np.isnan(b)
    if np.any(nan_a != nan_b):
        return float("inf")
    return max_rel_err(np.where(nan_a, 0, a), np.where(nan_b, 0, b))


def test_oracle_matches_reference_golden():
    d = np.load(os.path.join(HERE, "golden", "c_sw.npz"))
    n, nz, seed = int(d["arg_n"]), int(d["arg_nz"]), int(d["arg_seed"])
    out = oracle_runs.run_c_sw(cases.c_sw_case(n, nz, seed), n, nz)
    for k in OUT:
        assert _compare_full(out[k], d[k]) == 0.0, k


def _interior_mask(n, nz, h=3):
    """Points the CUDA path must reproduce: everything except the last
    (never-written) storage row/column, where both sides hold NaN/inputs."""
    m = n + 2 * h + 1
    return (slice(None), slice(0, m - 1), slice(0, m - 1), slice(0, nz))


@pytest.mark.gpu
@pytest.mark.parametrize("n,nz,seed", [(12, 6, 21), (24, 10, 4), (48, 5, 9), (12, 79, 6)])
def test_gpu_matches_oracle(n, nz, seed):
    import gpu_runs

    case = cases.c_sw_case(n, nz, seed)
    ref = oracle_runs.run_c_sw(case, n, nz)
    gpu = gpu_runs.run_c_sw(case, n, nz)
    sl = _interior_mask(n, nz)
    for k in OUT:
        err = parity_err(gpu[k][sl], ref[k][sl])
        assert err <= 1e-12, (k, err)

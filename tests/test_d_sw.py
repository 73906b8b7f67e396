"""DGridShallowWaterLagrangianDynamics: oracle vs the reference's golden
output; CUDA vs oracle."""
import os

import numpy as np
import pytest

import cases
import oracle_runs
from metrics import parity_err

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = ["delp", "pt", "u", "v", "w", "uc", "vc", "divgd", "mfx", "mfy", "cx", "cy", "crx", "cry",
       "xfx", "yfx", "q_con", "heat_source", "diss_est", "ptc"]


def _same(a, b):
    nan_a, nan_b = np.isnan(a), np.isnan(b)
    return bool(np.all(nan_a == nan_b) and np.all(np.where(nan_a, 0, a) == np.where(nan_b, 0, b)))


def test_oracle_matches_reference_golden():
    d = np.load(os.path.join(HERE, "golden", "d_sw.npz"))
    n, nz, seed = int(d["arg_n"]), int(d["arg_nz"]), int(d["arg_seed"])
    out = oracle_runs.run_d_sw(cases.d_sw_case(n, nz, seed), n, nz)
    for k in oracle_runs.DSW_ARGS:
        assert _same(out[k], d[k]), k


# staggering of each output: extra interface point in i and/or j
STAGGER = {
    "delp": (0, 0), "pt": (0, 0), "w": (0, 0), "q_con": (0, 0), "heat_source": (0, 0), "diss_est": (0, 0),
    "ptc": (0, 0), "u": (0, 1), "vc": (0, 1), "mfy": (0, 1), "cy": (0, 1), "yfx": (0, 1), "cry": (0, 1),
    "v": (1, 0), "uc": (1, 0), "mfx": (1, 0), "cx": (1, 0), "xfx": (1, 0), "crx": (1, 0), "divgd": (1, 1),
}


def _compute_region(name, n, nz, h=3):
    di, dj = STAGGER[name]
    return (slice(None), slice(h, h + n + di), slice(h, h + n + dj), slice(0, nz))


@pytest.mark.gpu
@pytest.mark.parametrize("n,nz,seed", [(12, 8, 31), (24, 12, 2), (48, 6, 8), (12, 79, 7)])
def test_gpu_matches_oracle(n, nz, seed):
    import gpu_runs

    case = cases.d_sw_case(n, nz, seed)
    ref = oracle_runs.run_d_sw(case, n, nz)
    gpu = gpu_runs.run_d_sw(case, n, nz)
    for k in OUT:
        sl = _compute_region(k, n, nz)
        err = parity_err(gpu[k][sl], ref[k][sl])
        assert err <= 1e-12, (k, err)


@pytest.mark.gpu
@pytest.mark.parametrize("nord", [0, 1])
def test_gpu_matches_oracle_other_nord(nord):
    """nord 1 takes the del-n chains with one pass after the first (nmax =
    1), nord 0 the single-pass chains; C48 so that the chains run both in
    the fused tiles and in the cube-corner tiles."""
    import gpu_runs

    n, nz, seed = 48, 6, 9
    case = cases.d_sw_case(n, nz, seed)
    ref = oracle_runs.run_d_sw(case, n, nz, overrides={"nord": nord})
    gpu = gpu_runs.run_d_sw(case, n, nz, overrides={"nord": nord})
    for k in OUT:
        sl = _compute_region(k, n, nz)
        err = parity_err(gpu[k][sl], ref[k][sl])
        assert err <= 1e-12, (k, err)

"""The mixed-precision build (FP32 fields and bulk arithmetic, FP64 column
solves) against the FP64 build on the same state: one AcousticDynamics call
with n_split = 6 (the acoustic part of one dynamics step of the baroclinic
configuration).  The target is a max relative error of 1e-4 in delp and pt;
the other prognostic fields are reported with looser bounds."""
import numpy as np
import pytest

import cases

H = 3


def _rel(a, b, n, nz, extra=(0, 0)):
    sl = (slice(None), slice(H, H + n + extra[0]), slice(H, H + n + extra[1]), slice(0, nz))
    a, b = a[sl], b[sl]
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-30)))


def _rms(a, b, n, nz):
    sl = (slice(None), slice(H, H + n), slice(H, H + n), slice(0, nz))
    return float(np.sqrt(np.mean((a[sl] - b[sl]) ** 2)) / np.sqrt(np.mean(b[sl] ** 2)))


@pytest.mark.gpu
@pytest.mark.parametrize("n,nz,seed", [(24, 79, 3), (48, 79, 8)])
def test_mixed_matches_fp64_after_one_step(n, nz, seed):
    import gpu_runs

    case = cases.acoustics_case(n, nz, seed, n_split=6)
    ref = gpu_runs.run_acoustics(case, n, nz, "f64")
    mix = gpu_runs.run_acoustics(case, n, nz, "f32")
    errs = {k: _rel(mix[k], ref[k], n, nz) for k in ("delp", "pt", "q_con", "delz")}
    rms = {k: _rms(mix[k], ref[k], n, nz) for k in ("u", "v", "w", "delp", "pt")}
    print("max rel", errs, "rms rel", rms)
    assert errs["delp"] <= 1e-4 and errs["pt"] <= 1e-4, errs
    assert errs["q_con"] <= 1e-3 and errs["delz"] <= 1e-3, errs
    assert rms["u"] <= 1e-3 and rms["v"] <= 1e-3 and rms["w"] <= 5e-2, rms

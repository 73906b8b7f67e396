"""The step preamble and epilogue of DynamicalCore.step_dynamics
(fv_dynamics.py:54-169): fv_setup and pt_adjust, set_omega with the omega
filter, the negative-tracer fixes (neg_adj3) and the cubed-to-latlon winds.
The oracle against a golden run of the reference's own functions (six tiles
in lock step with a threaded halo exchange), the CUDA path against the
oracle, phase by phase."""
import os

import numpy as np
import pytest

import cases
import oracle_runs
from metrics import max_rel_err, parity_err

HERE = os.path.dirname(os.path.abspath(__file__))
H = 3


def _golden():
    g = np.load(os.path.join(HERE, "golden", "fv_step.npz"))
    n, nz, seed = int(g["arg_n"]), int(g["arg_nz"]), int(g["arg_seed"])
    return g, n, nz, cases.fv_step_case(n, nz, seed)


def _fields(g):
    return [k for k in g.files if not k.startswith(("arg_", "meta_"))]


def test_oracle_matches_reference_golden():
    """Every storage point of every field each phase writes, bit for bit."""
    g, n, nz, case = _golden()
    out = oracle_runs.run_fv_step(case, n, nz)
    for k in _fields(g):
        assert np.array_equal(out[k], g[k], equal_nan=True), k


def test_golden_case_exercises_the_negative_fixes():
    """The fixture is not trivial: the fixes change most negative points of
    every species and the temperature."""
    g, n, nz, case = _golden()
    c = (slice(None), slice(H, H + n), slice(H, H + n), slice(0, nz))
    for name in cases.WATER_NAMES:
        assert np.count_nonzero(g["wrap_" + name][c] != case[name][c]) > 0.1 * case[name][c].size, name
    assert np.count_nonzero(g["wrap_pt"][c] != g["pre_pt"][c]) > 100


def test_fillq_conserves_column_mass():
    """fillq only moves water between levels: the column integral of q dp
    is kept where the column total is positive."""
    from oracle._util import Tile
    from oracle.fv_step import fillq

    n, nz = 12, 8
    t = Tile(n, nz)
    rng = np.random.default_rng(3)
    q = rng.uniform(-2e-4, 1e-3, (t.m, t.m, t.nk))
    dp = rng.uniform(100.0, 1000.0, (t.m, t.m, t.nk))
    c = (slice(H, H + n), slice(H, H + n), slice(0, nz))
    before = np.sum(q[c] * dp[c], axis=-1)
    fillq(t, q, dp)
    after = np.sum(q[c] * dp[c], axis=-1)
    assert np.allclose(after, before, rtol=1e-12, atol=1e-15)
    assert np.all(q[c] >= -1e-18)


def _compute(a, n, nz):
    return a[:, H:H + n, H:H + n, :nz]


@pytest.mark.gpu
@pytest.mark.parametrize("n,nz,seed", [(12, 8, 71), (24, 79, 72)])
def test_gpu_matches_oracle(n, nz, seed):
    """1e-12 on the compute domain of every field each phase writes, against
    the oracle with the kernels' exp/log; u and v also on their halos (the
    order-4 winds update them)."""
    import gpu_runs
    from oracle import _math

    case = cases.fv_step_case(n, nz, seed)
    with _math.device_math():
        ref = oracle_runs.run_fv_step(case, n, nz)
    gpu = gpu_runs.run_fv_step(case, n, nz)
    bad = {}
    for k in ref:
        a, b = (gpu[k], ref[k]) if k in ("wrap_u", "wrap_v") else (_compute(gpu[k], n, nz), _compute(ref[k], n, nz))
        e = parity_err(a[..., :nz], b[..., :nz])
        if not e <= 1e-12:
            bad[k] = e
    assert not bad, bad


@pytest.mark.gpu
def test_gpu_matches_reference_golden():
    """Against the reference's own output (numpy's exp/log), both metrics:
    every field within 1e-12 (pkz carries one exp and one log, not
    amplified)."""
    import gpu_runs

    g, n, nz, case = _golden()
    gpu = gpu_runs.run_fv_step(case, n, nz)
    bad = {}
    for k in _fields(g):
        a, b = _compute(gpu[k], n, nz), _compute(g[k], n, nz)
        e = (parity_err(a, b), max_rel_err(a, b))
        if not (e[0] <= 1e-12 and e[1] <= 1e-12):
            bad[k] = e
    assert not bad, bad


@pytest.mark.gpu
def test_gpu_mixed_precision_step_stages():
    """The mixed-precision build on the golden case: every field finite and
    within 1e-5 of its range of the FP64 result (the A-grid winds within
    1e-5 of the wind speed: va is a small difference of large products)."""
    import gpu_runs

    g, n, nz, case = _golden()
    f32 = gpu_runs.run_fv_step(case, n, nz, "f32")
    wind = float(max(np.max(np.abs(_compute(g[k], n, nz))) for k in ("wrap_u", "wrap_v")))
    for k in _fields(g):
        a, b = _compute(f32[k], n, nz), _compute(g[k], n, nz)
        assert np.all(np.isfinite(a)), k
        scale = wind if k in ("wrap_ua", "wrap_va") else (float(np.max(np.abs(b))) or 1.0)
        assert np.max(np.abs(a - b)) <= 1e-5 * scale, (k, float(np.max(np.abs(a - b))), scale)

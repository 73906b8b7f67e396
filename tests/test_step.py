"""DynamicalCore.step_dynamics (fv_dynamics.py:395-557): one dynamics step
of the nonhydrostatic core composed from the stages — preamble, acoustic
substeps, tracer advection, vertical remapping (no saturation adjustment),
omega filter, negative-tracer fixes, A-grid winds.  The oracle's step
against a golden run of the reference's own classes composed as
DynamicalCore._compute composes them; the CUDA DynamicalCore against the
oracle and the golden."""
import os

import numpy as np
import pytest

import cases
import oracle_runs
from metrics import max_rel_err, parity_err

HERE = os.path.dirname(os.path.abspath(__file__))
H = 3
# stored region of each field: extra points on (i, j, k)
STEP_OUT = {"u": (0, 1, 0), "v": (1, 0, 0), "w": (0, 0, 0), "delz": (0, 0, 0), "delp": (0, 0, 0), "pt": (0, 0, 0),
            "pe": (0, 0, 1), "pk": (0, 0, 1), "peln": (0, 0, 1), "pkz": (0, 0, 0), "q_con": (0, 0, 0),
            "cappa": (0, 0, 0), "omga": (0, 0, 0), "ua": (0, 0, 0), "va": (0, 0, 0)}
FIELDS = list(STEP_OUT) + list(cases.STEP_TRACERS) + ["ps"]
# Against the reference's numpy exp/log/pow (parity metric, compare_arr with
# near-zero 1e-18): about 30 times the floor that the two transcendental
# flavours give the oracle on the golden case (test_conditioning_of_the_step:
# u 1.6e-10, v 1.2e-10, w 1.8e-8, omga 8.2e-11, va 3.2e-9 (6.1e-9),
# qo3mr 1.3e-12 (4e-14); every other field below 3e-14), the acoustic
# substeps' amplification of last-place differences into the winds.
# With the saturation adjustment (step_satadj) the species that are small
# differences of terms carrying its saturation tables' exp / log are added
# (floors qliquid 1.1e-11, qrain 2.0e-12, q_con 3.4e-13, qsnow 5.0e-13,
# qice 3.2e-13, qcld 1.6e-13).
STEP_BOUNDS = {"u": (1e-8, 1e-8), "v": (1e-8, 1e-8), "w": (5e-7, 5e-7), "omga": (3e-9, 3e-9),
               "va": (1e-7, 2e-7), "qo3mr": (5e-11, 1e-12)}
BOUNDS = {"step": STEP_BOUNDS,
          "step_satadj": dict(STEP_BOUNDS, qliquid=(3e-10, 3e-10), qrain=(6e-11, 6e-11), q_con=(1e-11, 1e-11),
                              qsnow=(1e-11, 1e-11), qice=(1e-11, 1e-11), qcld=(1e-11, 1e-11))}
GOLDENS = tuple(BOUNDS)


def _golden(name="step"):
    g = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    n, nz, seed = int(g["arg_n"]), int(g["arg_nz"]), int(g["arg_seed"])
    return g, n, nz, cases.CASES[name](n=n, nz=nz, seed=seed)


def _region(a, name, n, nz):
    di, dj, dk = STEP_OUT.get(name, (0, 0, 0))
    sl = (slice(None), slice(H, H + n + di), slice(H, H + n + dj))
    return a[sl] if name == "ps" else a[sl + (slice(0, nz + dk),)]


@pytest.mark.parametrize("name", GOLDENS)
def test_oracle_matches_reference_golden(name):
    """Every stored point of every field, bit for bit (the second golden
    with the remapping's fast saturation adjustment)."""
    g, n, nz, case = _golden(name)
    out = oracle_runs.run_step(case, n, nz)
    for k in FIELDS:
        assert np.array_equal(_region(out[k], k, n, nz), g[k], equal_nan=True), k


@pytest.mark.parametrize("name", GOLDENS)
def test_conditioning_of_the_step(name):
    """The floors behind BOUNDS: the oracle with numpy's exp/log/pow
    against the oracle with the kernels' own."""
    from oracle import _math

    g, n, nz, case = _golden(name)
    a = oracle_runs.run_step(case, n, nz)
    with _math.device_math():
        b = oracle_runs.run_step(case, n, nz)
    for k in FIELDS:
        x, y = _region(a[k], k, n, nz), _region(b[k], k, n, nz)
        bp, bc = BOUNDS[name].get(k, (1e-12, 1e-12))
        assert parity_err(x, y) <= bp / 10 and max_rel_err(x, y) <= bc / 10, (k, parity_err(x, y))


def test_golden_step_moves_every_field():
    """The fixture is not trivial: the step changes every prognostic field at
    nearly every point, and the remapping puts delp back on the Eulerian
    levels (ak + bk ps)."""
    g, n, nz, case = _golden()
    for k in ("u", "v", "w", "delz", "pt", "qvapor"):
        x, y = g[k], _region(case[k], k, n, nz)
        assert np.count_nonzero(x != y) > 0.8 * x.size, k
    ps = g["ps"][..., None]
    dp2 = (case["ak"][1:nz + 1] + case["bk"][1:nz + 1] * ps) - (case["ak"][:nz] + case["bk"][:nz] * ps)
    dp2[..., 0] = (case["ak"][1] + case["bk"][1] * ps[..., 0]) - case["ptop"]
    dp2[..., nz - 1] = ps[..., 0] - (case["ak"][nz - 1] + case["bk"][nz - 1] * ps[..., 0])
    assert np.allclose(g["delp"], dp2, rtol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("name", GOLDENS)
def test_gpu_step_matches_reference_golden(name):
    """The CUDA DynamicalCore against the reference's own output, both
    metrics, every stored point, within BOUNDS (1e-12 where not listed)."""
    import gpu_runs

    g, n, nz, case = _golden(name)
    gpu = gpu_runs.run_step(case, n, nz)
    bad = {}
    for k in FIELDS:
        a = _region(gpu[k], k, n, nz)
        e = (parity_err(a, g[k]), max_rel_err(a, g[k]))
        bp, bc = BOUNDS[name].get(k, (1e-12, 1e-12))
        if not (e[0] <= bp and e[1] <= bc):
            bad[k] = e
    assert not bad, bad


@pytest.mark.gpu
@pytest.mark.parametrize("n,nz,seed,n_split,sat", [(12, 12, 101, 2, False), (12, 79, 102, 6, False),
                                                   (12, 79, 104, 6, True)])
def test_gpu_step_matches_oracle(n, nz, seed, n_split, sat):
    """1e-12 on every field (parity metric) against the oracle with the
    kernels' exp/log/pow; at C12 L79 the step of the baroclinic namelist
    (dt_atmos 225 s, n_split 6), without and with the fast saturation
    adjustment."""
    import gpu_runs
    from oracle import _math

    case = cases.step_case(n, nz, seed, n_split, sat_adj=sat)
    with _math.device_math():
        ref = oracle_runs.run_step(case, n, nz)
    gpu = gpu_runs.run_step(case, n, nz)
    bad = {}
    for k in FIELDS:
        e = parity_err(_region(gpu[k], k, n, nz), _region(ref[k], k, n, nz))
        if not e <= 1e-12:
            bad[k] = e
    assert not bad, bad


@pytest.mark.gpu
def test_gpu_two_steps_match_oracle():
    """Two steps in a row (DynamicalCore's and the acoustic driver's
    temporaries carried from the first to the second, as in the
    reference): 1e-12 on every field against the oracle with the kernels'
    exp/log/pow, and every field finite on the compute domain."""
    import gpu_runs
    from oracle import _math

    g, n, nz, case = _golden()
    with _math.device_math():
        ref = oracle_runs.run_step(case, n, nz, steps=2)
    gpu = gpu_runs.run_step(case, n, nz, steps=2)
    bad = {}
    for k in FIELDS:
        a = _region(gpu[k], k, n, nz)
        e = parity_err(a, _region(ref[k], k, n, nz))
        if not (e <= 1e-12 and np.all(np.isfinite(a))):
            bad[k] = e
    assert not bad, bad


@pytest.mark.gpu
def test_gpu_mixed_precision_step():
    """The mixed-precision build through a whole step on the golden case:
    every field finite; mass, heat and pressure fields within 1e-4 of the
    FP64 result relative to their range, the winds within 1e-3 of the wind
    speed."""
    import gpu_runs

    g, n, nz, case = _golden()
    f64 = gpu_runs.run_step(case, n, nz)
    f32 = gpu_runs.run_step(case, n, nz, "f32")
    wind = float(max(np.max(np.abs(_region(f64[k], k, n, nz))) for k in ("u", "v")))
    bad = {}
    for k in FIELDS:
        a, b = _region(f32[k], k, n, nz), _region(f64[k], k, n, nz)
        if k in ("u", "v", "w", "ua", "va", "omga"):
            scale, bound = (wind if k != "omga" else float(np.max(np.abs(b)))), 1e-3
        else:
            scale, bound = float(np.max(np.abs(b))) or 1.0, 1e-4
        err = float(np.max(np.abs(a - b))) / scale
        if not (np.all(np.isfinite(a)) and err <= bound):
            bad[k] = err
    assert not bad, bad

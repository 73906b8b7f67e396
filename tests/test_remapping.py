"""LagrangianToEulerian (remapping.py:205-628), the vertical remapping of
DynamicalCore.step_dynamics, without the saturation adjustment.  The oracle
against golden runs of the reference's own classes (kord 9, the baroclinic
namelist, at L79; kord 10 and kord 8 for the profile's other limiters), the
CUDA path against the oracle and the goldens, and properties at larger
sizes."""
import os

import numpy as np
import pytest

import cases
import oracle_runs
from metrics import max_rel_err, parity_err

HERE = os.path.dirname(os.path.abspath(__file__))
H = 3
GOLDENS = ("remap", "remap_kord10", "remap_kord8", "remap_satadj")
OUT = cases.REMAP_TRACERS + ("pt", "delp", "delz", "peln", "u", "v", "w", "ua", "va", "cappa", "q_con", "pkz",
                             "pk", "pe", "ps")


def _out(g):
    """The fields a golden stores (the cloud fraction with the saturation
    adjustment)."""
    return OUT + (("qcld",) if "qcld" in g.files else ())


def _golden(name):
    g = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    n, nz, seed = int(g["arg_n"]), int(g["arg_nz"]), int(g["arg_seed"])
    return g, n, nz, cases.CASES[name](n=n, nz=nz, seed=seed)


def _box(a, n):
    """The stored box of a golden: storage [3, 3 + n + 1) in i and j."""
    return a[:, H:H + n + 1, H:H + n + 1]


@pytest.mark.parametrize("name", GOLDENS)
def test_oracle_matches_reference_golden(name):
    """Every point of the compute domain and the D-grid winds' extra row,
    every level, bit for bit."""
    g, n, nz, case = _golden(name)
    out = oracle_runs.run_remap(case, n, nz)
    for k in _out(g):
        assert np.array_equal(_box(out[k], n), g[k], equal_nan=True), k


def test_golden_case_exercises_the_remap():
    """The fixture is not trivial: target layers that span more than two
    source layers (the reference's while loop), negative tracer values that
    fillz removes, and every remapped field changed."""
    g, n, nz, case = _golden("remap")
    c = (slice(None), slice(H, H + n), slice(H, H + n))
    pe1 = case["pe"][c]
    ps = pe1[..., nz]
    pe2 = case["ak"][None, None, None, :] + case["bk"] * ps[..., None]
    span = np.zeros(pe1.shape[:3] + (nz,), int)
    for k in range(nz):
        span[..., k] = ((pe1[..., 1:nz] > pe2[..., k:k + 1]) & (pe1[..., 1:nz] < pe2[..., k + 1:k + 2])).sum(-1)
    assert (span >= 2).sum() > 100
    for name in cases.REMAP_TRACERS:
        assert (case[name][c][..., :nz] < 0).sum() > 0
        assert (g[name][:, :n, :n, :nz] < 0).sum() == 0, name
    for k in ("pt", "u", "v", "w", "delz"):
        assert np.count_nonzero(g[k][:, :n, :n, :nz] != case[k][c][..., :nz]) > 0.8 * n * n * nz * 6, k


def test_remap_is_conservative():
    """Without the filler, the tracer remap keeps each column's integral of
    q dp: sum_k q2 dp2 = sum_k q1 dp1 (the profile integrates to the layer
    means and the target layers tile the same pressure range)."""
    from oracle import remapping as R
    from oracle._util import Tile

    n, nz = 4, 30
    case = cases.remap_case(n, nz, 91)
    t = Tile(n, nz)
    box = (H, H + n, H, H + n)
    for tt in range(2):
        q = np.abs(case["qvapor"][tt]).copy()
        pe1 = case["pe"][tt]
        ps = pe1[..., nz]
        pe2 = case["ak"][None, None, :] + case["bk"][None, None, :] * ps[..., None]
        pe2[..., 0] = case["ptop"]
        pe2[..., nz] = ps
        c = (slice(H, H + n), slice(H, H + n))
        before = np.sum(q[c][..., :nz] * np.diff(pe1[c], axis=-1), axis=-1)
        R.map_single(q, pe1, pe2, box, 9, 0)
        after = np.sum(q[c][..., :nz] * np.diff(pe2[c], axis=-1), axis=-1)
        assert np.allclose(after, before, rtol=1e-12), np.max(np.abs(after / before - 1))
    del t


def test_dropin_rejects_what_the_reference_rejects():
    """kord_tm >= 0 and hydrostatic, as the reference; the saturation
    adjustment, which is not built."""
    import types

    from fv3core_b200.config import RemappingConfig, SatAdjustConfig
    from fv3core_b200.stencils.remapping import LagrangianToEulerian

    sf = types.SimpleNamespace(grid_indexing=types.SimpleNamespace(context=None, domain=(12, 12, 79)))
    sat = SatAdjustConfig(**cases.SAT_ADJUST_CONFIG)
    base = dict(cases.REMAP_CONFIG)
    with pytest.raises(NotImplementedError, match="kord_tm"):
        LagrangianToEulerian(sf, RemappingConfig(sat_adjust=sat, **dict(base, kord_tm=9)), None, 8, np.ones(79))
    with pytest.raises(NotImplementedError, match="Hydrostatic"):
        hsat = SatAdjustConfig(**dict(cases.SAT_ADJUST_CONFIG, hydrostatic=True))
        LagrangianToEulerian(sf, RemappingConfig(sat_adjust=hsat, **base), None, 8, np.ones(79))
    with pytest.raises(AssertionError, match="kord"):
        LagrangianToEulerian(sf, RemappingConfig(sat_adjust=sat, **dict(base, kord_tr=11)), None, 8, np.ones(79))


def _cmp(a, b, n, nz, extra=0):
    """The remapped region: compute domain (plus the winds' extra row)."""
    s = (slice(None), slice(H, H + n + extra), slice(H, H + n + extra))
    return a[s], b[s]


# Points where the kord-10 limiter switches (ext5 / ext6 are discontinuous
# in the profile) after a last-place difference of the moist pt
# conversion's exp / log between numpy and the kernels' own functions, and,
# with the saturation adjustment, single points where a species is a small
# difference of terms carrying the saturation tables' exp / log (qliquid
# 1.0e-12, qsnow 4.4e-12 between the two sets of functions): the oracle
# shows the same points with either set of functions
# (test_kord10_switch_comes_from_the_transcendentals), and the GPU matches
# the oracle bit for bit with the kernels' functions (test_gpu_matches_oracle).
SWITCHED = {"remap_kord10": {"pt": 1e-5, "pkz": 1e-5}, "remap_satadj": {"qliquid": 1e-11, "qsnow": 5e-11}}


def test_kord10_switch_comes_from_the_transcendentals():
    """The oracle with numpy's exp / log against the oracle with the
    kernels' own: identical to 1e-12 except at two kord-10 points where the
    limiter switches (2.7e-6 in pt) and single points of two species with
    the saturation adjustment, none for kord 9 and 8."""
    from oracle import _math

    for name in GOLDENS:
        g, n, nz, case = _golden(name)
        a = oracle_runs.run_remap(case, n, nz)
        with _math.device_math():
            b = oracle_runs.run_remap(case, n, nz)
        for k in _out(g):
            x, y = _box(a[k], n)[..., :nz], _box(b[k], n)[..., :nz]
            d = np.abs(x - y) / np.maximum(np.abs(y), 1e-300)
            bound = SWITCHED.get(name, {}).get(k, 1e-12)
            assert np.nanmax(d) <= bound, (name, k, float(np.nanmax(d)))
            assert np.count_nonzero(d > 1e-12) <= (4 if k in SWITCHED.get(name, {}) else 0), (name, k)


@pytest.mark.gpu
@pytest.mark.parametrize("name", GOLDENS)
def test_gpu_matches_reference_golden(name):
    """The CUDA remap against the reference's own output (numpy's exp/log),
    both metrics, on every stored point: 1e-12, except the kord-10 limiter
    switch points of SWITCHED (at most four points above 1e-12)."""
    import gpu_runs

    g, n, nz, case = _golden(name)
    gpu = gpu_runs.run_remap(case, n, nz)
    bad = {}
    for k in _out(g):
        a, b = _box(gpu[k], n), g[k]
        bound = SWITCHED.get(name, {}).get(k, 1e-12)
        e = (parity_err(a, b), max_rel_err(a, b))
        above = int(np.count_nonzero(np.abs(a - b) > 1e-12 * np.maximum(np.abs(b), 1e-300)))
        if not (e[0] <= bound and e[1] <= bound) or (bound > 1e-12 and above > 4):
            bad[k] = e + (above,)
    assert not bad, bad


@pytest.mark.gpu
@pytest.mark.parametrize("n,nz,seed,kord,sat", [(4, 79, 81, (-9, 9, 9, 9), False), (24, 79, 92, (-9, 9, 9, 9), False),
                                                (12, 63, 93, (-10, 10, 10, 10), False),
                                                (12, 40, 94, (-8, 8, 8, 8), False),
                                                (12, 79, 95, (-9, 9, 9, 9), True)])
def test_gpu_matches_oracle(n, nz, seed, kord, sat):
    """Bit for bit against the oracle running the kernels' exp/log, on the
    remapped region of every field (the last case with the fast saturation
    adjustment)."""
    import gpu_runs
    from oracle import _math

    case = cases.remap_case(n, nz, seed, kord=kord, sat_adj=sat)
    with _math.device_math():
        ref = oracle_runs.run_remap(case, n, nz)
    gpu = gpu_runs.run_remap(case, n, nz)
    bad = {}
    for k in OUT + ("qcld",):
        a, b = _cmp(gpu[k], ref[k], n, nz, extra=1)
        if not np.array_equal(a, b, equal_nan=True):
            d = np.abs(a - b)
            bad[k] = (int(np.count_nonzero(~(d == 0) & ~(np.isnan(a) & np.isnan(b)))), float(np.nanmax(d)))
    assert not bad, bad


@pytest.mark.gpu
def test_gpu_mixed_precision_remap():
    """The mixed-precision build (FP32 fields, the remap itself in FP64): every
    field finite and within 1e-5 of its range of the FP64 result on the
    kord-9 golden case."""
    import gpu_runs

    g, n, nz, case = _golden("remap")
    f64 = gpu_runs.run_remap(case, n, nz)
    f32 = gpu_runs.run_remap(case, n, nz, "f32")
    bad = {}
    for k in OUT:
        a, b = _box(f32[k], n), _box(f64[k], n)
        a, b = a[..., :nz], b[..., :nz]
        if k == "ps":
            a, b = _box(f32[k], n), _box(f64[k], n)
        scale = float(np.max(np.abs(b))) or 1.0
        err = float(np.max(np.abs(a - b))) / scale
        if not (np.all(np.isfinite(a)) and err <= 1e-5):
            bad[k] = err
    assert not bad, bad

"""Why the mixed-precision build misses 1e-4 in pt on the noisy benchmark
state: the PPM limiters' smoothness switch, not FP32 arithmetic.

The FP64 oracle is run from a noisy state and from the same state with
every field rounded to FP32 (the input of a mixed-precision run), once with
the smoothness switch of the PPM fluxes (3|b0| < |bl - br|, xppm.py:48-61)
as the reference takes it and once with the switch held at one branch
(mask = 1 everywhere, the unlimited flux).  With the switch, a rounding-size
change of the input flips the branch at some points and moves pt there by
forty times the rounding; with the switch held, the response stays at the
rounding itself.  (The mixed build's error equals this FP64 response,
``bench.py``'s ``mixed_error_vs_fp64``.)  A diagnostic of the oracle, which
this test patches on the CPU; nothing of the product changes."""
import numpy as np

import cases
import oracle_runs

N, NZ, NSPLIT, H = 24, 16, 6, 3


def _response(case, case32):
    a = oracle_runs.run_acoustics(case, N, NZ)
    b = oracle_runs.run_acoustics(case32, N, NZ)
    out = {}
    for name in ("delp", "pt", "delz"):
        x = a[name][:, H:H + N, H:H + N, :NZ]
        y = b[name][:, H:H + N, H:H + N, :NZ]
        with np.errstate(all="ignore"):
            rel = np.nan_to_num(np.abs(x - y) / np.abs(x))
        out[name] = (float(rel.max()), float(np.percentile(rel, 99.9)))
    return out


def test_limiter_switch_amplifies_fp32_rounding(monkeypatch):
    import oracle.ppm as ppm

    case = cases.acoustics_case(N, NZ, seed=5, n_split=NSPLIT)
    case32 = {k: (v.astype(np.float32).astype(np.float64)
                  if isinstance(v, np.ndarray) and v.dtype == np.float64 and v.ndim >= 3 else v)
              for k, v in case.items()}
    with_switch = _response(case, case32)
    monkeypatch.setattr(ppm, "advection_mask", lambda bl, b0, br, axis, mord=6: np.ones_like(b0))
    held = _response(case, case32)
    # the switch takes pt and delz to 2.5e-6 (measured) ...
    assert with_switch["pt"][0] > 1e-6 and with_switch["delz"][0] > 1e-6, with_switch
    # ... held at one branch, the response is the rounding (6e-8 pt, 2.4e-7 delz)
    assert held["pt"][0] < 2e-7 and held["delz"][0] < 1e-6 and held["delp"][0] < 1e-7, held
    # away from the flipped points the two agree: the 99.9th percentiles are
    # the rounding in both
    for name in ("delp", "pt", "delz"):
        assert with_switch[name][1] < 1e-6 and abs(with_switch[name][1] - held[name][1]) < 1e-7, name

"""AcousticDynamics (the whole acoustic substep loop): oracle vs the
reference's golden output (six tiles stepped together with a threaded halo
exchange); CUDA vs oracle."""
import os

import numpy as np
import pytest

import cases
import oracle_runs
from metrics import parity_err

HERE = os.path.dirname(os.path.abspath(__file__))
H = 3


def _same(a, b):
    nan_a, nan_b = np.isnan(a), np.isnan(b)
    return bool(np.all(nan_a == nan_b) and np.all(np.where(nan_a, 0, a) == np.where(nan_b, 0, b)))


def test_oracle_matches_reference_golden():
    g = np.load(os.path.join(HERE, "golden", "acoustics.npz"))
    n, nz, seed = int(g["arg_n"]), int(g["arg_nz"]), int(g["arg_seed"])
    out = oracle_runs.run_acoustics(cases.acoustics_case(n, nz, seed), n, nz)
    for k in g.files:
        if k.startswith(("arg_", "meta_")) or k not in out:
            continue
        assert _same(out[k], g[k]), k


# extra interface point (i, j) and number of levels (npz + dk) of each field
LAYOUT = {
    "u": (0, 1, 0), "v": (1, 0, 0), "w": (0, 0, 0), "delz": (0, 0, 0), "delp": (0, 0, 0), "pt": (0, 0, 0),
    "pe": (0, 0, 1), "pk": (0, 0, 1), "peln": (0, 0, 1), "pkz": (0, 0, 0), "q_con": (0, 0, 0),
    "diss_estd": (0, 0, 0), "omga": (0, 0, 0), "ua": (0, 0, 0), "va": (0, 0, 0), "uc": (1, 0, 0),
    "vc": (0, 1, 0), "mfxd": (1, 0, 0), "mfyd": (0, 1, 0), "cxd": (1, 0, 0), "cyd": (0, 1, 0),
    "tmp_zh": (0, 0, 1), "tmp_gz": (0, 0, 1), "tmp_pkc": (0, 0, 1), "tmp_pk3": (0, 0, 1),
    "tmp_heat_source": (0, 0, 0), "tmp_divgd": (1, 1, 0),
}
PROGNOSTIC = ("u", "v", "w", "delp", "pt", "delz", "q_con")


def _compute(name, n, nz):
    di, dj, dk = LAYOUT[name]
    return (slice(None), slice(H, H + n + di), slice(H, H + n + dj), slice(0, nz + dk))


@pytest.mark.gpu
@pytest.mark.parametrize("n,nz,seed,n_split", [(12, 8, 41, 2), (24, 16, 5, 3), (48, 12, 9, 1)])
def test_gpu_matches_oracle(n, nz, seed, n_split):
    import gpu_runs

    case = cases.acoustics_case(n, nz, seed, n_split=n_split)
    ref = oracle_runs.run_acoustics(case, n, nz)
    gpu = gpu_runs.run_acoustics(case, n, nz)
    errs = {k: parity_err(gpu[k][_compute(k, n, nz)], ref[k][_compute(k, n, nz)]) for k in LAYOUT}
    bad = {k: e for k, e in errs.items() if not e <= 1e-12}
    assert not bad, bad


@pytest.mark.gpu
def test_gpu_full_storage_matches_oracle():
    """Every point of every field, halos included, on the golden case."""
    import gpu_runs

    n, nz = 12, 8
    case = cases.acoustics_case(n, nz, 41)
    ref = oracle_runs.run_acoustics(case, n, nz)
    gpu = gpu_runs.run_acoustics(case, n, nz)
    bad = {}
    for k in gpu:
        e = parity_err(gpu[k], ref[k])
        if not e <= 1e-12:
            bad[k] = e
    assert not bad, bad

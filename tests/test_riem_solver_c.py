"""RiemannSolverC: oracle vs the reference's golden output, CUDA vs oracle."""
import numpy as np
import pytest

import cases
from metrics import max_rel_err, parity_err

GOLDEN = "tests/golden/riem_solver_c.npz"
TOL_GOLDEN = 1e-14  # oracle restates the reference bit for bit in FP64
TOL_GPU = 1e-12


def _run_oracle(case, n, nz):
    from oracle.riem_solver_c import riem_solver_c

    for t in range(6):
        riem_solver_c(
            case["dt2"], case["cappa"][t], case["ptop"], case["hs"][t], case["ws"][t], case["ptc"][t],
            case["q_con"][t], case["delpc"][t], case["gz"][t], case["pef"][t], case["w3"][t], case["p_fac"], n, nz,
        )
    return case


def _region(n, nz, h=3):
    return (slice(None), slice(h - 1, h + n + 1), slice(h - 1, h + n + 1), slice(0, nz + 1))


def test_oracle_matches_reference_golden():
    import os

    d = np.load(os.path.join(cases.__file__.rsplit("/", 1)[0], "riem_solver_c.npz"))
    n, nz, seed = int(d["arg_n"]), int(d["arg_nz"]), int(d["arg_seed"])
    c = _run_oracle(cases.riem_solver_c_case(n, nz, seed), n, nz)
    sl = _region(n, nz)
    for name in ("pef", "gz"):
        assert max_rel_err(c[name][sl], d[name]) <= TOL_GOLDEN, name


def _run_gpu(case, n, nz):
    import torch

    from fv3core_b200.stencil import StencilConfig, StencilFactory
    from fv3core_b200.stencils.riem_solver_c import RiemannSolverC
    from fv3core_b200.storage import GridIndexing, to_device, to_host

    gi = GridIndexing((n, n, nz), 3)
    sf = StencilFactory(StencilConfig(), gi)
    rs = RiemannSolverC(sf, p_fac=case["p_fac"])
    dev = {k: to_device(v) for k, v in case.items() if isinstance(v, np.ndarray)}
    rs(case["dt2"], dev["cappa"], case["ptop"], dev["hs"], dev["ws"], dev["ptc"], dev["q_con"], dev["delpc"],
       dev["gz"], dev["pef"], dev["w3"])
    torch.cuda.synchronize()
    return {k: to_host(dev[k]) for k in ("pef", "gz")}


@pytest.mark.gpu
@pytest.mark.parametrize("n,nz,seed", [(12, 16, 11), (12, 79, 3), (48, 79, 5), (20, 2, 7)])
def test_gpu_matches_oracle(n, nz, seed):
    from oracle import _math

    case = cases.riem_solver_c_case(n, nz, seed)
    gpu = _run_gpu({k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in case.items()}, n, nz)
    with _math.device_math():
        ref = _run_oracle(case, n, nz)
    sl = _region(n, nz)
    for name in ("pef", "gz"):
        err = parity_err(gpu[name][sl], ref[name][sl])
        assert err <= TOL_GPU, (name, err)


@pytest.mark.gpu
def test_gpu_matches_reference_golden():
    import os

    d = np.load(os.path.join(cases.__file__.rsplit("/", 1)[0], "riem_solver_c.npz"))
    n, nz, seed = int(d["arg_n"]), int(d["arg_nz"]), int(d["arg_seed"])
    gpu = _run_gpu(cases.riem_solver_c_case(n, nz, seed), n, nz)
    sl = _region(n, nz)
    for name in ("pef", "gz"):
        assert parity_err(gpu[name][sl], d[name]) <= TOL_GPU, name

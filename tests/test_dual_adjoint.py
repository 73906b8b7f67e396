"""The dual-number adjoint scheme (fv3core_b200/csrc/dual.h), built for the
host: p_grad_c's increments differentiated with duals give the gradients of
the hand-written adjoint (fv3core_b200/csrc/pgrad_adjoint.h), which torch
autograd checks in tests/test_pgrad_adjoint.py."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from test_pgrad_adjoint import DT2, H, _metrics, kernel_layout, pgc_case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path_factory, name):
    so = str(tmp_path_factory.mktemp(name) / f"{name}.so")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-o", so,
                           os.path.join(ROOT, "tests", "native", f"{name}.cpp")])
    return ctypes.CDLL(so)


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@pytest.mark.parametrize("n,nz,seed", [(12, 8, 3), (7, 4, 4)])
def test_dual_adjoint_matches_hand_written(tmp_path_factory, n, nz, seed):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    dual = _build(tmp_path_factory, "dual_adjoint_host")
    hand = _build(tmp_path_factory, "pgrad_adjoint_host")
    case = {k: kernel_layout(v) for k, v in pgc_case(n, nz, seed).items()}
    rng = np.random.default_rng(seed)
    gu, gv = rng.standard_normal(case["uc"].shape), rng.standard_normal(case["uc"].shape)
    rdxc, rdyc = _metrics(n)
    results = []
    for lib, name in ((dual, "pgc_dual_adjoint_host"), (hand, "pgc_adjoint_host")):
        out = [np.zeros_like(gu) for _ in range(3)]
        getattr(lib, name)(ctypes.c_int(n), ctypes.c_int(H), ctypes.c_int(nz), ctypes.c_double(DT2), _ptr(rdxc),
                           _ptr(rdyc), _ptr(case["delpc"]), _ptr(case["pkc"]), _ptr(case["gz"]), _ptr(gu), _ptr(gv),
                           *[_ptr(o) for o in out])
        results.append(out)
    for a, b in zip(*results):
        assert np.max(np.abs(a - b)) <= 1e-13 * np.max(np.abs(b))


@pytest.mark.parametrize("thin", [False, True])
def test_dual_scheme_on_update_dz_c(tmp_path_factory, thin):
    # a branchy stage (upwind choices, corner copies): the dual scatter of
    # the advected heights' cotangents equals the hand-written one
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    import cases
    from test_updatedzc_adjoint import DT2 as UDT, uzc_case

    from test_updatedzc_adjoint import kernel_layout as kl

    dual = _build(tmp_path_factory, "dual_adjoint_host")
    hand = _build(tmp_path_factory, "updatedzc_adjoint_host")
    n, nz = 12, 5
    case = uzc_case(n, nz, 7, thin)
    k = {name: kl(case[name]) for name in ("ut", "vt", "gz")}
    area = kl(np.asarray(cases.grid_for(n).area))
    rng = np.random.default_rng(2)
    g_gz_out, g_ws = rng.standard_normal(k["gz"].shape), rng.standard_normal(kl(case["ws"]).shape)
    hand_out = {name: np.zeros_like(k["gz"]) for name in ("gz", "ut", "vt", "hnew", "g_new")}
    hand.uzc_adjoint_host.restype = None
    hand.uzc_adjoint_host(ctypes.c_int(n), ctypes.c_int(H), ctypes.c_int(nz), ctypes.c_double(UDT),
                          _ptr(case["dp_ref"]), _ptr(area), _ptr(k["ut"]), _ptr(k["vt"]), _ptr(k["gz"]),
                          _ptr(g_gz_out), _ptr(g_ws), *[_ptr(hand_out[x]) for x in ("gz", "ut", "vt", "hnew",
                                                                                      "g_new")])
    mine = {name: np.zeros_like(k["gz"]) for name in ("gz", "ut", "vt")}
    box = np.zeros(k["gz"].shape, bool)
    box[:, :, H - 1:H + n + 1, H - 1:H + n + 1] = True
    mine["gz"][~box] = g_gz_out[~box]  # the pass-through outside the updated box
    dual.uzc_dual_scatter_host.restype = None
    dual.uzc_dual_scatter_host(ctypes.c_int(n), ctypes.c_int(H), ctypes.c_int(nz), _ptr(case["dp_ref"]), _ptr(area),
                               _ptr(k["ut"]), _ptr(k["vt"]), _ptr(k["gz"]), _ptr(hand_out["g_new"]),
                               *[_ptr(mine[x]) for x in ("gz", "ut", "vt")])
    for name in ("gz", "ut", "vt"):
        b = hand_out[name]
        assert np.max(np.abs(mine[name] - b)) <= 1e-12 * np.max(np.abs(b)), name


def test_dual_transcendentals_match_finite_differences(tmp_path_factory):
    """dexp, dlog and dpow are the library's fmath functions with their
    derivatives: a nonlinear column function's dual value equals the plain
    fmath evaluation bit for bit, and its derivative agrees with central
    differences of that evaluation (step 1e-6 relative, bound 1e-7)."""
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    lib = _build(tmp_path_factory, "dual_adjoint_host")
    x = np.random.default_rng(5).uniform(0.05, 40.0, 64)
    n = x.size
    value, deriv, plain = np.empty(n), np.empty(n), np.empty(n)
    lib.dual_transcendental_host(ctypes.c_int(n), _ptr(x), _ptr(value), _ptr(deriv))
    lib.plain_transcendental_host(ctypes.c_int(n), _ptr(x), _ptr(plain))
    np.testing.assert_array_equal(value, plain)
    h = 1e-6 * x
    fp, fm = np.empty(n), np.empty(n)
    xp, xm = x + h, x - h
    lib.plain_transcendental_host(ctypes.c_int(n), _ptr(xp), _ptr(fp))
    lib.plain_transcendental_host(ctypes.c_int(n), _ptr(xm), _ptr(fm))
    fd = (fp - fm) / (xp - xm)
    assert np.max(np.abs(fd - deriv) / np.abs(deriv)) < 1e-7

"""The adjoint of compute_pkz_tempadjust (temperature_adjust.py:8-44)
(fv3core_b200/csrc/tempadjust_adjoint.h) built for the host, against torch
autograd of a PyTorch-ops restatement that matches the oracle."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest
import torch

import cases
from fv3core_b200 import constants as C

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
H = 3
DTF = 0.5


def _case(n, nz, seed):
    st = cases.base_state(n, nz, seed)
    rng = np.random.default_rng(seed)
    heat = C.CV_AIR * st["delp"] * 0.5 * rng.standard_normal(st["delp"].shape)
    return {"delp": st["delp"], "delz": st["delz"], "cappa": st["cappa"], "heat": heat, "pt": st["pt"]}


def _limits(nk_heat):
    return np.array([0.1 if k == 0 else (0.5 if k == 1 else 1.0) for k in range(nk_heat)]) * DTF


def tempadjust_torch(dp, dz, pt, heat, cappa, lim):
    c = cappa / (1.0 - cappa)
    p = (C.RDG * dp / dz * pt) ** c
    dtmp = heat / (C.CV_AIR * dp)
    delt = torch.where(lim < dtmp.abs(), torch.where(dtmp > 0, lim, -lim), dtmp)
    return pt + delt / p, p


def _points(f, n, nk_heat):
    B = (slice(None), slice(H, H + n), slice(H, H + n), slice(0, nk_heat))
    lim = np.broadcast_to(_limits(nk_heat), next(iter(f.values()))[B].shape)
    return {k: np.ascontiguousarray(v[B]).ravel() for k, v in f.items()}, np.ascontiguousarray(lim).ravel()


def test_restatement_matches_oracle():
    from oracle._util import Tile
    from oracle.dyn_core import pkz_tempadjust

    n, nz, nk_heat = 12, 6, 4
    f = _case(n, nz, 2)
    pt, pkz = f["pt"].copy(), np.zeros_like(f["pt"])
    for t in range(6):
        pkz_tempadjust(Tile(n, nz), f["delp"][t], f["delz"][t], f["cappa"][t], f["heat"][t], pt[t], pkz[t], DTF,
                       nk_heat)
    pts, lim = _points(f, n, nk_heat)
    T = {k: torch.from_numpy(v) for k, v in pts.items()}
    new_pt, new_pkz = tempadjust_torch(T["delp"], T["delz"], T["pt"], T["heat"], T["cappa"], torch.from_numpy(lim))
    want_pt, _ = _points({"x": pt}, n, nk_heat)
    want_pkz, _ = _points({"x": pkz}, n, nk_heat)
    np.testing.assert_allclose(new_pt.numpy(), want_pt["x"], rtol=1e-14)
    np.testing.assert_allclose(new_pkz.numpy(), want_pkz["x"], rtol=1e-13)
    dtmp = pts["heat"] / (C.CV_AIR * pts["delp"])
    assert (np.abs(dtmp) > lim).any() and (np.abs(dtmp) < lim).any()  # both branches


@pytest.fixture(scope="module")
def host_lib(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    so = str(tmp_path_factory.mktemp("ta") / "tempadjust_adjoint.so")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-fPIC", "-shared", "-o", so,
                           os.path.join(ROOT, "tests", "native", "tempadjust_adjoint_host.cpp")])
    lib = ctypes.CDLL(so)
    lib.tempadjust_adjoint_host.restype = None
    return lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def test_host_adjoint_matches_torch_autograd(host_lib):
    n, nz, nk_heat = 12, 6, 4
    pts, lim = _points(_case(n, nz, 3), n, nk_heat)
    rng = np.random.default_rng(1)
    gt, gk = rng.standard_normal(lim.shape), rng.standard_normal(lim.shape)
    T = {k: torch.from_numpy(v.copy()).requires_grad_(k != "cappa") for k, v in pts.items()}
    new_pt, new_pkz = tempadjust_torch(T["delp"], T["delz"], T["pt"], T["heat"], T["cappa"], torch.from_numpy(lim))
    ((new_pt * torch.from_numpy(gt)).sum() + (new_pkz * torch.from_numpy(gk)).sum()).backward()
    out = {k: np.zeros(lim.shape) for k in ("delp", "delz", "pt", "heat")}
    host_lib.tempadjust_adjoint_host(
        ctypes.c_int(lim.size), _ptr(pts["delp"]), _ptr(pts["delz"]), _ptr(pts["pt"]), _ptr(pts["heat"]),
        _ptr(pts["cappa"]), _ptr(lim), ctypes.c_double(C.RDG), ctypes.c_double(C.CV_AIR), _ptr(gt), _ptr(gk),
        _ptr(out["delp"]), _ptr(out["delz"]), _ptr(out["pt"]), _ptr(out["heat"]))
    for k in out:
        b = T[k].grad.numpy()
        np.testing.assert_allclose(out[k], b, rtol=1e-10, atol=1e-12 * np.max(np.abs(b)), err_msg=k)

"""The adjoints of edge_pe (pe_halo.py:6-33) and PK3Halo (pk3_halo.py:36-68)
(fv3core_b200/csrc/pressure_adjoint.h) built for the host, against torch
autograd of PyTorch-ops restatements that match the oracle."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest
import torch

import cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
H = 3
AKAP = 0.2857142857142857


def kernel_layout(a):
    return np.ascontiguousarray(a.transpose(0, 3, 2, 1))


def ring(n, width):
    m = n + 2 * H + 1
    r = np.zeros((m, m), bool)
    r[H - width:H + n + width, H - width:H + n + width] = True
    r[H:H + n, H:H + n] = False
    return torch.from_numpy(r)


def edge_pe_torch(pe, delp, ptop, n):
    nk = pe.shape[1]
    col = torch.cat([torch.zeros_like(delp[:, :1]), torch.cumsum(delp[:, :nk - 1], dim=1)], dim=1) + ptop
    return torch.where(ring(n, 1), col, pe)


def pk3_halo_torch(pk3, delp, ptop, akap, n):
    nk = pk3.shape[1]
    col = (torch.cumsum(delp[:, :nk - 1], dim=1) + ptop) ** akap
    return torch.cat([pk3[:, :1], torch.where(ring(n, 2), col, pk3[:, 1:])], dim=1)


def _case(n, nz, seed):
    st = cases.base_state(n, nz, seed)
    rng = np.random.default_rng(seed)
    return st["delp"] * (1 + 1e-2 * rng.standard_normal(st["delp"].shape)), float(st["ptop"]), rng


def test_restatements_match_oracle():
    from oracle._util import Tile
    from oracle.dyn_core import edge_pe, pk3_halo

    n, nz = 12, 6
    delp, ptop, rng = _case(n, nz, 3)
    pe = rng.standard_normal(delp.shape)
    pk3 = rng.standard_normal(delp.shape)
    ref_pe, ref_pk3 = pe.copy(), pk3.copy()
    t = Tile(n, nz)
    for tile in range(6):
        edge_pe(t, ref_pe[tile], delp[tile], ptop)
        pk3_halo(t, ref_pk3[tile], delp[tile], ptop, AKAP, np.zeros((t.m, t.m)))
    kd = torch.from_numpy(kernel_layout(delp))
    mine_pe = edge_pe_torch(torch.from_numpy(kernel_layout(pe)), kd, ptop, n).numpy()
    mine_pk3 = pk3_halo_torch(torch.from_numpy(kernel_layout(pk3)), kd, ptop, AKAP, n).numpy()
    np.testing.assert_allclose(mine_pe, kernel_layout(ref_pe), rtol=1e-14, atol=0)
    np.testing.assert_allclose(mine_pk3, kernel_layout(ref_pk3), rtol=1e-13, atol=0)


@pytest.fixture(scope="module")
def host_lib(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    so = str(tmp_path_factory.mktemp("pa") / "pressure_adjoint.so")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-o", so,
                           os.path.join(ROOT, "tests", "native", "pressure_adjoint_host.cpp")])
    lib = ctypes.CDLL(so)
    lib.edge_pe_adjoint_host.restype = None
    lib.pk3_halo_adjoint_host.restype = None
    return lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@pytest.mark.parametrize("n,nz,seed", [(12, 6, 4), (7, 9, 5)])
def test_host_adjoints_match_torch_autograd(host_lib, n, nz, seed):
    delp, ptop, rng = _case(n, nz, seed)
    kd = kernel_layout(delp)
    shp = kd.shape
    for name in ("edge_pe", "pk3"):
        x = torch.from_numpy(rng.standard_normal(shp)).requires_grad_(True)
        d = torch.from_numpy(kd.copy()).requires_grad_(True)
        cot = rng.standard_normal(shp)
        y = edge_pe_torch(x, d, ptop, n) if name == "edge_pe" else pk3_halo_torch(x, d, ptop, AKAP, n)
        (y * torch.from_numpy(cot)).sum().backward()
        g = cot.copy()
        g_delp = np.zeros(shp)
        if name == "edge_pe":
            host_lib.edge_pe_adjoint_host(ctypes.c_int(n), ctypes.c_int(H), ctypes.c_int(nz), _ptr(g), _ptr(g_delp))
        else:
            host_lib.pk3_halo_adjoint_host(ctypes.c_int(n), ctypes.c_int(H), ctypes.c_int(nz), ctypes.c_double(ptop),
                                           ctypes.c_double(AKAP), _ptr(kd), _ptr(g), _ptr(g_delp))
        np.testing.assert_array_equal(g, x.grad.numpy())
        err = np.max(np.abs(g_delp - d.grad.numpy())) / np.max(np.abs(d.grad.numpy()))
        assert err <= 1e-13, (name, err)

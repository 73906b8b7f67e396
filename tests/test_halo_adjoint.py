"""The transposes of the halo updates (fv3core_b200/csrc/halo_adjoint.h),
compiled for the host, against the forward gathers of the package's tables
(fv3core_b200/halo_map.py, which the geometric halo tests check) by the
dot-product identity <H x, y> = <x, H^T y>, exact for these copies."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from fv3core_b200 import halo_map as hm

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
H = 3
NZ = 3


@pytest.fixture(scope="module")
def host_halo(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    so = str(tmp_path_factory.mktemp("halo_adj") / "halo_adjoint.so")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-fPIC", "-shared", "-o", so,
                           os.path.join(ROOT, "tests", "native", "halo_adjoint_host.cpp")])
    lib = ctypes.CDLL(so)
    for f in (lib.halo_scalar_adjoint_host, lib.halo_vector_adjoint_host, lib.interface_sync_adjoint_host):
        f.restype = None
    return lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _fields(n, count, seed):
    m = n + 2 * H + 1
    rng = np.random.default_rng(seed)
    return [rng.standard_normal((6, NZ + 1, m, m)) for _ in range(count)]


def _ints(*v):
    return [ctypes.c_int(x) for x in v]


def _dot(a, b):
    return sum(float((x * y).sum()) for x, y in zip(a, b))


@pytest.mark.parametrize("n", [12, 7])
@pytest.mark.parametrize("stagger,n_halo", [(1, 3), (1, 2), (0, 3)])
def test_scalar_transpose(host_halo, n, stagger, n_halo):
    x, y = _fields(n, 2, n + stagger + n_halo)
    hx = x.copy()
    for t, i, j, st, si, sj in hm.scalar_table(n, H, stagger, stagger, n_halo):
        hx[t, :, j, i] = x[st, :, sj, si]
    hty = y.copy()
    host_halo.halo_scalar_adjoint_host(*_ints(n, H, NZ), _ptr(hty), *_ints(stagger, n_halo, NZ + 1))
    assert abs(_dot([hx], [y]) - _dot([x], [hty])) <= 1e-12 * np.abs(hx * y).sum()


@pytest.mark.parametrize("n", [12, 7])
@pytest.mark.parametrize("grid,xs,ys", [(0, (1, 0), (0, 1)), (1, (0, 1), (1, 0))])
def test_vector_transpose(host_halo, n, grid, xs, ys):
    x = _fields(n, 2, n + grid)
    y = _fields(n, 2, n + grid + 10)
    hx = [f.copy() for f in x]
    for comp, table in enumerate(hm.vector_tables(n, H, xs, ys, H)):
        for t, i, j, st, si, sj, sc, sg in table:
            hx[comp][t, :, j, i] = sg * x[sc][st, :, sj, si]
    hty = [f.copy() for f in y]
    host_halo.halo_vector_adjoint_host(*_ints(n, H, NZ), _ptr(hty[0]), _ptr(hty[1]), *_ints(grid, NZ + 1))
    scale = sum(np.abs(a * b).sum() for a, b in zip(hx, y))
    assert abs(_dot(hx, y) - _dot(x, hty)) <= 1e-12 * scale


@pytest.mark.parametrize("n", [12, 7])
def test_interface_sync_transpose(host_halo, n):
    x = _fields(n, 2, n + 20)
    y = _fields(n, 2, n + 30)
    hx = [f.copy() for f in x]
    for dt, dc, di, dj, st, sc, si, sj, sg in hm.interface_sync_tables(n, H):
        hx[dc][dt, :, dj, di] = sg * x[sc][st, :, sj, si]
    hty = [f.copy() for f in y]
    host_halo.interface_sync_adjoint_host(*_ints(n, H, NZ), _ptr(hty[0]), _ptr(hty[1]), ctypes.c_int(NZ + 1))
    scale = sum(np.abs(a * b).sum() for a, b in zip(hx, y))
    assert abs(_dot(hx, y) - _dot(x, hty)) <= 1e-12 * scale

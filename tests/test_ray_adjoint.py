"""The adjoint of RayleighDamping (fv3core_b200/csrc/ray_adjoint.h), built
for the host, against the oracle's forward (ray_fast.py) by the dot-product
identity: the damping is linear in the winds."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

import cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
H = 3


def kernel_layout(a):
    return np.ascontiguousarray(a.transpose(0, 3, 2, 1))


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@pytest.fixture(scope="module")
def host_ray(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    so = str(tmp_path_factory.mktemp("ray") / "ray_adjoint.so")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-fPIC", "-shared", "-o", so,
                           os.path.join(ROOT, "tests", "native", "ray_adjoint_host.cpp")])
    lib = ctypes.CDLL(so)
    lib.ray_adjoint_host.restype = None
    return lib


@pytest.mark.parametrize("n,nz,seed,extra", [(12, 10, 1, 1), (7, 16, 2, 2), (12, 10, 3, 5)])
def test_transpose_dot_product_identity(host_ray, n, nz, seed, extra):
    from oracle._util import Tile
    from oracle.dyn_core import ray_fast

    st = cases.base_state(n, nz, seed)
    ak, bk = np.asarray(st["ak"]), np.asarray(st["bk"])
    dp = ak[1:] - ak[:-1] + (bk[1:] - bk[:-1]) * 1.0e5
    pfull = np.asarray(st["pfull"], dtype=np.float64)[:nz].copy()
    # damp the top extra + 1 levels (one damped level alone, given back to
    # itself, would be the identity)
    rf_cutoff = float(pfull[extra]) * 1.01
    dt, ptop, tau = 37.5, float(st["ptop"]), 10.0
    rng = np.random.default_rng(seed)
    shp = st["delp"].shape
    x = [rng.standard_normal(shp) for _ in range(3)]
    y = [rng.standard_normal(shp) for _ in range(3)]
    rx = [a.copy() for a in x]
    for t in range(6):
        ray_fast(Tile(n, nz), rx[0][t], rx[1][t], rx[2][t], dp, pfull, dt, ptop, rf_cutoff, tau)
    assert not np.array_equal(rx[0], x[0])  # the damping acted
    ky = [kernel_layout(a) for a in y]
    host_ray.ray_adjoint_host(ctypes.c_int(n), ctypes.c_int(H), ctypes.c_int(nz), _ptr(dp), _ptr(pfull),
                              ctypes.c_double(dt), ctypes.c_double(ptop), ctypes.c_double(rf_cutoff),
                              ctypes.c_double(tau), *[_ptr(a) for a in ky])
    rty = [a.transpose(0, 3, 2, 1) for a in ky]
    lhs = sum(float((a * b).sum()) for a, b in zip(rx, y))
    rhs = sum(float((a * b).sum()) for a, b in zip(x, rty))
    scale = sum(float(np.abs(a * b).sum()) for a, b in zip(rx, y))
    assert abs(lhs - rhs) <= 1e-13 * scale

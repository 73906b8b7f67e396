"""The transpose of HyperdiffusionDamping (fv3core_b200/csrc/del2cubed_adjoint.h)
built for the host: its pass functions reproduce the oracle's filter
(del2cubed.py), and the transpose satisfies the dot-product identity."""
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
    return np.ascontiguousarray(a.transpose(0, 3, 2, 1) if a.ndim == 4 else a.transpose(0, 2, 1))


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@pytest.fixture(scope="module")
def host_d2c(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    so = str(tmp_path_factory.mktemp("d2c") / "del2cubed_adjoint.so")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-o", so,
                           os.path.join(ROOT, "tests", "native", "del2cubed_adjoint_host.cpp")])
    lib = ctypes.CDLL(so)
    lib.del2cubed_forward_host.restype = None
    lib.del2cubed_adjoint_host.restype = None
    return lib


def _metrics(n):
    g = cases.grid_for(n)
    return [kernel_layout(np.asarray(getattr(g, k))) for k in ("del6_u", "del6_v", "rarea")]


def _args(n, nz, cd, nmax, metrics):
    return [ctypes.c_int(n), ctypes.c_int(H), ctypes.c_int(nz), ctypes.c_double(cd), ctypes.c_int(nmax)] + [
        _ptr(m) for m in metrics]


@pytest.mark.parametrize("n,nz,nmax", [(12, 3, 3), (13, 2, 2), (12, 2, 1)])
def test_forward_matches_oracle(host_d2c, n, nz, nmax):
    from oracle._util import Tile
    from oracle.dyn_core import del2cubed

    rng = np.random.default_rng(n + nmax)
    m = n + 2 * H + 1
    q = rng.standard_normal((6, m, m, nz + 1))
    cd = 0.2 * float(cases.grid_for(n).da_min)
    ref = q.copy()
    T = Tile(n, nz)
    for t in range(6):
        scr = {k: np.full((T.m, T.m, T.nk), np.nan) for k in ("q", "fx", "fy")}
        del2cubed(T, cases.metric_namespace(n, t), ref[t], cd, nmax, scr)
    mine = kernel_layout(q)
    host_d2c.del2cubed_forward_host(*_args(n, nz, cd, nmax, _metrics(n)), _ptr(mine))
    want = kernel_layout(ref)
    np.testing.assert_allclose(mine[:, :nz], want[:, :nz], rtol=0, atol=1e-12 * np.max(np.abs(want)))


@pytest.mark.parametrize("n,nz,nmax", [(12, 2, 3), (7, 2, 3), (12, 1, 2)])
def test_transpose_dot_product_identity(host_d2c, n, nz, nmax):
    rng = np.random.default_rng(n * nmax)
    m = n + 2 * H + 1
    x = rng.standard_normal((6, nz + 1, m, m))
    y = rng.standard_normal((6, nz + 1, m, m))
    y[:, nz] = 0.0  # the filter leaves level npz alone
    x[:, nz] = 0.0
    cd = 0.2 * float(cases.grid_for(n).da_min)
    metrics = _metrics(n)
    ax = x.copy()
    host_d2c.del2cubed_forward_host(*_args(n, nz, cd, nmax, metrics), _ptr(ax))
    aty = y.copy()
    host_d2c.del2cubed_adjoint_host(*_args(n, nz, cd, nmax, metrics), _ptr(aty))
    lhs, rhs = float((ax * y).sum()), float((x * aty).sum())
    assert abs(lhs - rhs) <= 1e-12 * float(np.abs(ax * y).sum())

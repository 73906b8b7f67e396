"""The transpose of DelnFluxNoSG (fv3core_b200/csrc/deln_adjoint.h),
compiled for the host, against the oracle's forward (oracle/fvtp2d.py
delnflux_nosg, which restates delnflux.py:1156-1207 and is pinned to the
reference through the d_sw golden) by the dot-product identity
<A q, g> = <q, A^T g>, on levels with and without the higher-order passes
and through the cube-corner copies."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

import cases
from oracle._util import Tile
from oracle.fvtp2d import DelnScratch, delnflux_nosg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no host compiler")
    so = str(tmp_path_factory.mktemp("deln_adj") / "deln_adjoint_host.so")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-o", so,
                           os.path.join(ROOT, "tests", "native", "deln_adjoint_host.cpp")])
    return ctypes.CDLL(so)


def _ptr(a):
    return np.ascontiguousarray(a).ctypes.data_as(ctypes.c_void_p)


@pytest.mark.parametrize("n,nz,nord,mass_weighted", [(12, 6, (0.0, 0.0, 2.0, 2.0), False),
                                                     (12, 5, (1.0, 1.0, 1.0, 1.0), False),
                                                     (16, 5, (0.0, 2.0, 2.0, 2.0), True)])
def test_transpose_satisfies_the_dot_product_identity(lib, n, nz, nord, mass_weighted):
    h = 3
    t = Tile(n, nz, h)
    g = cases.metric_namespace(n, 0)
    m = t.m
    rng = np.random.default_rng(n + nz)
    q = rng.standard_normal((m, m, nz))
    # the scheme's own coefficients (calc_damp, delnflux.py:24-26): one area
    # per pass, so every pass contributes at the same scale
    damp = np.array([(0.06 * g.da_min) ** (nord[min(k, 3)] + 1) for k in range(nz)])
    scr = DelnScratch((m, m, nz + 1))
    fx2, fy2 = np.full((m, m, nz), np.nan), np.full((m, m, nz), np.nan)
    d2 = np.full((m, m, nz), np.nan)
    delnflux_nosg(t, g, q, fx2, fy2, damp, d2, np.asarray(nord), mass=q if mass_weighted else None, nk=nz)
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    gx = np.zeros((m, m, nz))
    gy = np.zeros((m, m, nz))
    gx[s:e + 2, js:je + 1] = rng.standard_normal((n + 2 - 0, n + 1 - 0, nz))[: e + 2 - s, : je + 1 - js]
    gy[s:e + 1, js:je + 2] = rng.standard_normal((n + 1, n + 2, nz))[: e + 1 - s, : je + 2 - js]
    lhs = (np.sum(fx2[s:e + 2, js:je + 1] * gx[s:e + 2, js:je + 1], axis=(0, 1))
           + np.sum(fy2[s:e + 1, js:je + 2] * gy[s:e + 1, js:je + 2], axis=(0, 1)))  # per level
    assert np.all(np.isfinite(lhs))
    gq = np.zeros((m, m, nz))
    nmax = int(max(nord))
    lib.deln_nosg_adjoint_host(n, h, nz, nmax, _ptr(np.asarray(nord, dtype=np.float64)), _ptr(damp),
                               int(mass_weighted), _ptr(np.asarray(g.del6_u)), _ptr(np.asarray(g.del6_v)),
                               _ptr(np.asarray(g.rarea)), _ptr(gx), _ptr(gy), _ptr(gq))
    rhs = np.sum(q * gq, axis=(0, 1))
    scale = (np.sum(np.abs(fx2[s:e + 2, js:je + 1] * gx[s:e + 2, js:je + 1]), axis=(0, 1))
             + np.sum(np.abs(fy2[s:e + 1, js:je + 2] * gy[s:e + 1, js:je + 2]), axis=(0, 1)))
    assert np.all(np.abs(lhs - rhs) <= 1e-12 * scale), (lhs, rhs)
    # a wrong pass count breaks it on the levels that iterate
    if nmax > 1:
        gq1 = np.zeros((m, m, nz))
        lib.deln_nosg_adjoint_host(n, h, nz, nmax - 1, _ptr(np.asarray(nord, dtype=np.float64)), _ptr(damp),
                                   int(mass_weighted), _ptr(np.asarray(g.del6_u)), _ptr(np.asarray(g.del6_v)),
                                   _ptr(np.asarray(g.rarea)), _ptr(gx), _ptr(gy), _ptr(gq1))
        assert np.any(np.abs(lhs - np.sum(q * gq1, axis=(0, 1))) > 1e-6 * scale)

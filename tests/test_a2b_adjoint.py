"""The transpose of a2b_ord4 (fv3core_b200/csrc/a2b_adjoint.h) built for
the host: its point functions reproduce the oracle's interpolation
(a2b_ord4.py), and the transpose satisfies the dot-product identity
<A x, y> = <x, A^T y> to rounding."""
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
    """[6, i, j, k] -> [6, k, j, i] (2-D: [6, i, j] -> [6, j, i])."""
    return np.ascontiguousarray(a.transpose(0, 3, 2, 1) if a.ndim == 4 else a.transpose(0, 2, 1))


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@pytest.fixture(scope="module")
def host_a2b(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    so = str(tmp_path_factory.mktemp("a2b") / "a2b_adjoint.so")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-o", so,
                           os.path.join(ROOT, "tests", "native", "a2b_adjoint_host.cpp")])
    lib = ctypes.CDLL(so)
    lib.a2b_forward_host.restype = None
    lib.a2b_adjoint_host.restype = None
    return lib


class HostGrid:
    """The grid terms of a2b_ord4 in the kernel layout, kept alive for ctypes."""

    def __init__(self, n):
        g = cases.grid_for(n)
        self.dxa = kernel_layout(np.asarray(g.dxa))
        self.dya = kernel_layout(np.asarray(g.dya))
        self.edges = [np.ascontiguousarray(np.asarray(getattr(g, k), dtype=np.float64))
                      for k in ("edge_w", "edge_e", "edge_s", "edge_n")]
        self.extrap = np.ascontiguousarray(np.asarray(g.a2b_extrap, dtype=np.float64))

    def args(self):
        return [_ptr(self.dxa), _ptr(self.dya)] + [_ptr(e) for e in self.edges] + [_ptr(self.extrap)]


def _dims(n, nz, k0, k1):
    return [ctypes.c_int(v) for v in (n, H, nz, k0, k1)]


def a2b_forward(lib, grid, n, nz, k0, k1, q):
    """q, the result: kernel layout; the result is zero outside the B-grid box."""
    out = np.zeros_like(q)
    lib.a2b_forward_host(*_dims(n, nz, k0, k1), *grid.args(), _ptr(q), _ptr(out))
    return out


def a2b_transpose(lib, grid, n, nz, k0, k1, g):
    out = np.zeros_like(g)
    lib.a2b_adjoint_host(*_dims(n, nz, k0, k1), *grid.args(), _ptr(np.ascontiguousarray(g)), _ptr(out))
    return out


def _box(n, k0, k1):
    return (slice(None), slice(k0, k1), slice(H, H + n + 1), slice(H, H + n + 1))


@pytest.mark.parametrize("n,nz,k0,k1", [(12, 6, 0, 7), (16, 4, 1, 5)])
def test_forward_matches_oracle(host_a2b, n, nz, k0, k1):
    from oracle._util import Tile
    from oracle.a2b_ord4 import A2BScratch, a2b_ord4

    st = cases.base_state(n, nz, 2)
    q = st["pt"] * (1 + 1e-2 * np.random.default_rng(1).standard_normal(st["pt"].shape))
    t = Tile(n, nz)
    ref = np.zeros_like(q)
    for tile in range(6):
        a2b_ord4(t, cases.metric_namespace(n, tile), q[tile], ref[tile], k0, k1, A2BScratch(q[tile].shape))
    mine = a2b_forward(host_a2b, HostGrid(n), n, nz, k0, k1, kernel_layout(q))
    box = _box(n, k0, k1)
    want = kernel_layout(ref)[box]
    assert np.max(np.abs(mine[box] - want)) <= 1e-12 * np.max(np.abs(want))


@pytest.mark.parametrize("n,nz,seed", [(12, 3, 0), (13, 2, 1), (16, 2, 2)])
def test_transpose_dot_product_identity(host_a2b, n, nz, seed):
    rng = np.random.default_rng(seed)
    grid = HostGrid(n)
    m = n + 2 * H + 1
    x = rng.standard_normal((6, nz + 1, m, m))
    y = np.zeros_like(x)
    box = _box(n, 0, nz + 1)
    y[box] = rng.standard_normal(y[box].shape)
    ax = a2b_forward(host_a2b, grid, n, nz, 0, nz + 1, x)
    aty = a2b_transpose(host_a2b, grid, n, nz, 0, nz + 1, y)
    lhs, rhs = float((ax * y).sum()), float((x * aty).sum())
    assert abs(lhs - rhs) <= 1e-12 * (np.abs(ax * y).sum())
    # the transpose touches only what the interpolation reads
    reach = np.zeros(x.shape, bool)
    reach[:, :, H - 2:H + n + 3, H - 2:H + n + 3] = True
    assert not aty[~reach].any()


# ---------------------------------------------------------------- nh_p_grad


def nhp_case(n, nz, seed):
    st = cases.base_state(n, nz, seed)
    rng = np.random.default_rng(seed + 9)
    shp = st["delp"].shape
    f = {"u": st["u"].copy(), "v": st["v"].copy(), "pp": 10.0 * rng.standard_normal(shp),
         "gz": cases.heights(st, nz) * 9.80665, "pk3": st["pk"] * (1 + 1e-5 * rng.standard_normal(shp)),
         "delp": st["delp"].copy()}
    return f, float(st["ptop"])


OUTPUTS = ("u", "v", "pp", "pk3", "gz")


def oracle_nh_p_grad(f, n, nz, dt, ptop):
    """The oracle's stage on copies of f (oracle layout): the new fields."""
    from oracle._util import Tile
    from oracle.a2b_ord4 import A2BScratch
    from oracle.dyn_core import nh_p_grad

    from fv3core_b200 import constants as C

    out = {k: np.array(v, copy=True) for k, v in f.items()}
    T = Tile(n, nz)
    shape = (T.m, T.m, T.nk)
    for t in range(6):
        scr = {"wk": np.full(shape, np.nan), "wk1": np.full(shape, np.nan), "a2b_k1": A2BScratch(shape),
               "a2b_kbuffer": A2BScratch(shape), "a2b_kstandard": A2BScratch(shape)}
        nh_p_grad(T, cases.metric_namespace(n, t), scr, out["u"][t], out["v"][t], out["pp"][t], out["gz"][t],
                  out["pk3"][t], out["delp"][t], dt, ptop, C.KAPPA)
    return out


@pytest.mark.parametrize("n,nz,seed", [(12, 4, 3), (13, 3, 4)])
def test_host_nh_p_grad_adjoint_matches_oracle_finite_differences(host_a2b, n, nz, seed):
    from fv3core_b200 import constants as C

    f, ptop = nhp_case(n, nz, seed)
    dt = 37.5
    rng = np.random.default_rng(seed)
    cot = {k: rng.standard_normal(f[k].shape) for k in OUTPUTS}
    cot["gz"] *= 1e-3
    grid = HostGrid(n)
    g = cases.grid_for(n)
    rdx, rdy = kernel_layout(np.asarray(g.rdx)), kernel_layout(np.asarray(g.rdy))
    kf = {k: kernel_layout(v) for k, v in f.items()}
    kc = {k: kernel_layout(v) for k, v in cot.items()}
    grads = {k: np.zeros_like(kf["u"]) for k in ("u", "v", "pp", "pk3", "gz", "delp")}
    host_a2b.nhp_adjoint_host.restype = None
    host_a2b.nhp_adjoint_host(
        ctypes.c_int(n), ctypes.c_int(H), ctypes.c_int(nz), ctypes.c_double(dt), ctypes.c_double(ptop ** C.KAPPA),
        *grid.args(), _ptr(rdx), _ptr(rdy), _ptr(kf["pp"]), _ptr(kf["pk3"]), _ptr(kf["gz"]), _ptr(kf["delp"]),
        *[_ptr(kc[k]) for k in OUTPUTS], *[_ptr(grads[k]) for k in ("u", "v", "pp", "pk3", "gz", "delp")])
    grads = {k: v.transpose(0, 3, 2, 1) for k, v in grads.items()}  # back to the oracle layout

    def loss(x):
        out = oracle_nh_p_grad(x, n, nz, dt, ptop)
        return sum(float((out[k] * cot[k]).sum()) for k in OUTPUTS)

    for trial in range(3):
        dirs = {k: rng.standard_normal(v.shape) * (np.abs(v) + (10.0 if k == "pp" else 0.0)) for k, v in f.items()}
        eps = 1e-6
        lp = loss({k: f[k] + eps * dirs[k] for k in f})
        lm = loss({k: f[k] - eps * dirs[k] for k in f})
        fd = (lp - lm) / (2 * eps)
        ad = sum(float((grads[k] * dirs[k]).sum()) for k in f)
        assert abs(fd - ad) <= 1e-7 * abs(ad), (trial, fd, ad)

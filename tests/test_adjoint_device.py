"""Device builds of the adjoints whose headers are checked on the host
(tests/test_a2b_adjoint.py, test_halo_adjoint.py, test_pressure_adjoint.py,
test_ray_adjoint.py, test_del2cubed_adjoint.py, test_tempadjust_adjoint.py):
the gradients through their torch.autograd Functions on the GPU against the
host builds of the same headers."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
H = 3
N, NZ = 12, 6


def kernel_layout(a):
    return np.ascontiguousarray(a.transpose(0, 3, 2, 1) if a.ndim == 4 else a.transpose(0, 2, 1))


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _host(tmp_path_factory, name):
    so = str(tmp_path_factory.mktemp(name) / f"{name}.so")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-fPIC", "-shared", "-o", so,
                           os.path.join(ROOT, "tests", "native", f"{name}.cpp")])
    return ctypes.CDLL(so)


@pytest.fixture(scope="module")
def grid():
    import gpu_runs

    return gpu_runs.device_grid(N, NZ)


def _dev(a, grad=True):
    import torch

    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return t.requires_grad_(grad)


def _close(a, b, tol=1e-12):
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else a
    scale = max(float(np.max(np.abs(b))), 1e-300)
    assert float(np.max(np.abs(a - b))) <= tol * scale


def _random(shape, seed):
    return np.random.default_rng(seed).standard_normal(shape)


def test_halo_calls(grid, tmp_path_factory):
    from fv3core_b200.adjoint import halo_update_scalar, halo_update_vector, synchronize_vector_interfaces

    lib = _host(tmp_path_factory, "halo_adjoint_host")
    for f in (lib.halo_scalar_adjoint_host, lib.halo_vector_adjoint_host, lib.interface_sync_adjoint_host):
        f.restype = None
    gd, sf = grid
    m = N + 2 * H + 1
    shp = (6, NZ + 1, m, m)
    ints = [ctypes.c_int(v) for v in (N, H, NZ)]
    for stagger, n_halo in ((1, 3), (0, 3), (1, 2)):
        x, w = _dev(_random(shp, 1)), _random(shp, 2)
        (halo_update_scalar(x, sf, stagger, n_halo) * _dev(w, False)).sum().backward()
        want = w.copy()
        lib.halo_scalar_adjoint_host(*ints, _ptr(want), ctypes.c_int(stagger), ctypes.c_int(n_halo),
                                     ctypes.c_int(NZ + 1))
        _close(x.grad, want)
    for grid_kind in (0, 1):
        x, y = _dev(_random(shp, 3)), _dev(_random(shp, 4))
        wx, wy = _random(shp, 5), _random(shp, 6)
        ox, oy = halo_update_vector(x, y, sf, grid_kind)
        ((ox * _dev(wx, False)).sum() + (oy * _dev(wy, False)).sum()).backward()
        lib.halo_vector_adjoint_host(*ints, _ptr(wx), _ptr(wy), ctypes.c_int(grid_kind), ctypes.c_int(NZ + 1))
        _close(x.grad, wx)
        _close(y.grad, wy)
    u, v = _dev(_random(shp, 7)), _dev(_random(shp, 8))
    wu, wv = _random(shp, 9), _random(shp, 10)
    ou, ov = synchronize_vector_interfaces(u, v, sf)
    ((ou * _dev(wu, False)).sum() + (ov * _dev(wv, False)).sum()).backward()
    lib.interface_sync_adjoint_host(*ints, _ptr(wu), _ptr(wv), ctypes.c_int(NZ + 1))
    _close(u.grad, wu)
    _close(v.grad, wv)


def _state():
    return cases.base_state(N, NZ, 5)


def test_edge_pe_and_pk3_halo(grid, tmp_path_factory):
    from fv3core_b200 import constants as C
    from fv3core_b200.adjoint import edge_pe, pk3_halo

    lib = _host(tmp_path_factory, "pressure_adjoint_host")
    lib.edge_pe_adjoint_host.restype = None
    lib.pk3_halo_adjoint_host.restype = None
    gd, sf = grid
    st = _state()
    delp = kernel_layout(st["delp"])
    ptop = float(st["ptop"])
    ints = [ctypes.c_int(v) for v in (N, H, NZ)]
    pe, d = _dev(_random(delp.shape, 1)), _dev(delp)
    w = _random(delp.shape, 2)
    (edge_pe(pe, d, sf, ptop) * _dev(w, False)).sum().backward()
    g_delp = np.zeros_like(w)
    lib.edge_pe_adjoint_host(*ints, _ptr(w), _ptr(g_delp))
    _close(pe.grad, w)
    _close(d.grad, g_delp)
    pk3, d = _dev(_random(delp.shape, 3)), _dev(delp)
    w = _random(delp.shape, 4)
    (pk3_halo(pk3, d, sf, ptop, C.KAPPA) * _dev(w, False)).sum().backward()
    g_delp = np.zeros_like(w)
    lib.pk3_halo_adjoint_host(*ints, ctypes.c_double(ptop), ctypes.c_double(C.KAPPA), _ptr(delp), _ptr(w),
                              _ptr(g_delp))
    _close(pk3.grad, w)
    _close(d.grad, g_delp)


def test_ray_fast(grid, tmp_path_factory):
    from fv3core_b200.adjoint import ray_fast

    lib = _host(tmp_path_factory, "ray_adjoint_host")
    lib.ray_adjoint_host.restype = None
    gd, sf = grid
    st = _state()
    ak, bk = np.asarray(st["ak"]), np.asarray(st["bk"])
    dp = ak[1:] - ak[:-1] + (bk[1:] - bk[:-1]) * 1.0e5
    pfull = np.asarray(st["pfull"], dtype=np.float64)[:NZ].copy()
    rf_cutoff, dt, ptop, tau = float(pfull[2]) * 1.01, 37.5, float(st["ptop"]), 10.0
    shp = kernel_layout(st["delp"]).shape
    x = [_dev(_random(shp, s)) for s in (1, 2, 3)]
    w = [_random(shp, s) for s in (4, 5, 6)]
    out = ray_fast(*x, dp, pfull, sf, dt, ptop, rf_cutoff, tau)
    sum((o * _dev(wi, False)).sum() for o, wi in zip(out, w)).backward()
    lib.ray_adjoint_host(ctypes.c_int(N), ctypes.c_int(H), ctypes.c_int(NZ), _ptr(dp), _ptr(pfull),
                         ctypes.c_double(dt), ctypes.c_double(ptop), ctypes.c_double(rf_cutoff), ctypes.c_double(tau),
                         *[_ptr(wi) for wi in w])
    for xi, wi in zip(x, w):
        _close(xi.grad, wi)


def test_del2cubed(grid, tmp_path_factory):
    from fv3core_b200.adjoint import del2cubed

    lib = _host(tmp_path_factory, "del2cubed_adjoint_host")
    lib.del2cubed_adjoint_host.restype = None
    gd, sf = grid
    g = cases.grid_for(N)
    metrics = [kernel_layout(np.asarray(getattr(g, k))) for k in ("del6_u", "del6_v", "rarea")]
    cd = 0.2 * float(g.da_min)
    m = N + 2 * H + 1
    q, w = _dev(_random((6, NZ + 1, m, m), 1)), _random((6, NZ + 1, m, m), 2)
    (del2cubed(q, sf, cd, 3) * _dev(w, False)).sum().backward()
    lib.del2cubed_adjoint_host(ctypes.c_int(N), ctypes.c_int(H), ctypes.c_int(NZ), ctypes.c_double(cd),
                               ctypes.c_int(3), *[_ptr(a) for a in metrics], _ptr(w))
    _close(q.grad, w)


def test_pkz_tempadjust(grid, tmp_path_factory):
    from fv3core_b200 import constants as C
    from fv3core_b200.adjoint import pkz_tempadjust

    lib = _host(tmp_path_factory, "tempadjust_adjoint_host")
    lib.tempadjust_adjoint_host.restype = None
    gd, sf = grid
    st = _state()
    nk_heat, dtf = 4, 0.5
    k = {n: kernel_layout(st[n]) for n in ("delp", "delz", "cappa", "pt")}
    k["heat"] = C.CV_AIR * k["delp"] * 0.5 * _random(k["delp"].shape, 1)
    x = {n: _dev(k[n], n != "cappa") for n in ("delp", "delz", "cappa", "heat", "pt")}
    pkz = _dev(_random(k["pt"].shape, 2))
    gt, gk = _random(k["pt"].shape, 3), _random(k["pt"].shape, 4)
    new_pt, new_pkz = pkz_tempadjust(x["delp"], x["delz"], x["cappa"], x["heat"], x["pt"], pkz, sf, dtf, nk_heat)
    ((new_pt * _dev(gt, False)).sum() + (new_pkz * _dev(gk, False)).sum()).backward()
    box = (slice(None), slice(0, nk_heat), slice(H, H + N), slice(H, H + N))
    lim = np.broadcast_to(np.array([0.1, 0.5] + [1.0] * (nk_heat - 2))[None, :, None, None] * dtf,
                          k["pt"][box].shape)
    pts = {n: np.ascontiguousarray(k[n][box]).ravel() for n in ("delp", "delz", "pt", "heat", "cappa")}
    out = {n: np.zeros(pts["pt"].shape) for n in ("delp", "delz", "pt", "heat")}
    lib.tempadjust_adjoint_host(
        ctypes.c_int(pts["pt"].size), _ptr(pts["delp"]), _ptr(pts["delz"]), _ptr(pts["pt"]), _ptr(pts["heat"]),
        _ptr(pts["cappa"]), _ptr(np.ascontiguousarray(lim).ravel()), ctypes.c_double(C.RDG),
        ctypes.c_double(C.CV_AIR), _ptr(np.ascontiguousarray(gt[box]).ravel()),
        _ptr(np.ascontiguousarray(gk[box]).ravel()), *[_ptr(out[n]) for n in ("delp", "delz", "pt", "heat")])
    for n in ("delp", "delz", "pt", "heat"):
        got = x[n].grad.detach().cpu().numpy()
        _close(got[box].ravel(), out[n])
        outside = np.ones(got.shape, bool)
        outside[box] = False
        want_outside = gt[outside] if n == "pt" else 0.0
        assert np.array_equal(got[outside], np.broadcast_to(want_outside, got[outside].shape))
    g_pkz = pkz.grad.detach().cpu().numpy()
    assert not g_pkz[box].any()


def test_nh_p_grad(grid, tmp_path_factory):
    from fv3core_b200 import constants as C
    from fv3core_b200.adjoint import nh_p_grad

    lib = _host(tmp_path_factory, "a2b_adjoint_host")
    lib.nhp_adjoint_host.restype = None
    gd, sf = grid
    st = _state()
    g = cases.grid_for(N)
    rng = np.random.default_rng(6)
    f = {"u": st["u"], "v": st["v"], "pp": 10.0 * rng.standard_normal(st["delp"].shape),
         "gz": cases.heights(st, NZ) * 9.80665, "pk3": st["pk"], "delp": st["delp"]}
    kf = {n: kernel_layout(a) for n, a in f.items()}
    x = {n: _dev(a) for n, a in kf.items()}
    dt, ptop = 37.5, float(st["ptop"])
    outs = nh_p_grad(x["u"], x["v"], x["pp"], x["gz"], x["pk3"], x["delp"], sf, dt, ptop, C.KAPPA)
    names = ("u", "v", "pp", "gz", "pk3")
    cot = {n: _random(kf["u"].shape, 10 + i) for i, n in enumerate(names)}
    sum((o * _dev(cot[n], False)).sum() for o, n in zip(outs, names)).backward()
    grads = {n: np.zeros_like(kf["u"]) for n in ("u", "v", "pp", "pk3", "gz", "delp")}
    edges = [np.ascontiguousarray(np.asarray(getattr(g, k), dtype=np.float64))
             for k in ("edge_w", "edge_e", "edge_s", "edge_n")]
    extrap = np.ascontiguousarray(np.asarray(g.a2b_extrap, dtype=np.float64))
    dxa, dya = kernel_layout(np.asarray(g.dxa)), kernel_layout(np.asarray(g.dya))
    rdx, rdy = kernel_layout(np.asarray(g.rdx)), kernel_layout(np.asarray(g.rdy))
    lib.nhp_adjoint_host(
        ctypes.c_int(N), ctypes.c_int(H), ctypes.c_int(NZ), ctypes.c_double(dt), ctypes.c_double(ptop ** C.KAPPA),
        _ptr(dxa), _ptr(dya), *[_ptr(e) for e in edges], _ptr(extrap), _ptr(rdx), _ptr(rdy), _ptr(kf["pp"]),
        _ptr(kf["pk3"]), _ptr(kf["gz"]), _ptr(kf["delp"]), *[_ptr(cot[n]) for n in ("u", "v", "pp", "pk3", "gz")],
        *[_ptr(grads[n]) for n in ("u", "v", "pp", "pk3", "gz", "delp")])
    for n in grads:
        _close(x[n].grad, grads[n], tol=1e-11)

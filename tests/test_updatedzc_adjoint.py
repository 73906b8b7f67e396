"""The hand-written adjoint of UpdateGeopotentialHeightOnCGrid
(updatedzc.py:123-163): fv3core_b200/csrc/updatedzc_adjoint.h built for the
host and compared with torch autograd of a PyTorch-ops restatement (itself
equal to the oracle), then the device build behind
fv3core_b200.adjoint.update_dz_c on the GPU, alone and chained with
RiemannSolverC and p_grad_c as the acoustic loop chains them."""
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
DT2 = 18.75
DZ_MIN = 2.0


def dp_ref_of(st, nz):
    ak, bk = np.asarray(st["ak"]), np.asarray(st["bk"])
    dp = np.zeros(nz + 1)
    dp[:nz] = ak[1:] - ak[:-1] + (bk[1:] - bk[:-1]) * 1.0e5
    return dp


def uzc_case(n, nz, seed, thin=False):
    """Seeded inputs in the oracle's [6, i, j, k] order.  thin: some layers
    thinner than DZ_MIN, so that the floor acts."""
    st = cases.base_state(n, nz, seed)
    rng = np.random.default_rng(seed + 5)
    g = cases.grid_for(n)
    gz = cases.heights(st, nz)
    if thin:
        pick = rng.random(gz.shape[:3] + (nz,)) < 0.2
        for k in range(nz - 1, -1, -1):
            gz[..., k] = np.where(pick[..., k], gz[..., k + 1] + 1.0, gz[..., k])
    area = np.asarray(g.area)[:, :, :, None]
    return {
        "dp_ref": dp_ref_of(st, nz),
        "zs": st["phis"] * (1.0 / 9.80665),
        "ut": 0.02 * area * rng.standard_normal(gz.shape),
        "vt": 0.02 * area * rng.standard_normal(gz.shape),
        "gz": gz,
        "ws": 0.01 * rng.standard_normal(gz.shape[:3]),
    }


def kernel_layout(a):
    """[6, i, j, k] -> [6, k, j, i] (2-D: [6, i, j] -> [6, j, i])."""
    return np.ascontiguousarray(a.transpose(0, 3, 2, 1) if a.ndim == 4 else a.transpose(0, 2, 1))


def corner_maps(n, nz):
    """Flat source index of every (i, j) under the two-cell corner fills of
    the x and y sweeps (the oracle's rules applied to an index array)."""
    from oracle import corners
    from oracle._util import Tile

    t = Tile(n, nz)
    idx = np.arange(t.m * t.m, dtype=np.float64).reshape(t.m, t.m)
    mx = corners.fill_corners_2cells_x(t, idx).astype(np.int64).ravel()
    my = corners.fill_corners_2cells_y(t, idx).astype(np.int64).ravel()
    return torch.from_numpy(mx), torch.from_numpy(my)


def _p_weighted(a, dp0, nk):
    """p_weighted_average_top / _domain / _bottom (updatedzc.py:15-34)."""
    r = dp0[0] / (dp0[0] + dp0[1])
    cols = [a[..., 0] + (a[..., 0] - a[..., 1]) * r]
    for k in range(1, nk - 1):
        ir = 1.0 / (dp0[k - 1] + dp0[k])
        cols.append((dp0[k] * a[..., k - 1] + dp0[k - 1] * a[..., k]) * ir)
    k = nk - 1
    r = dp0[k - 1] / (dp0[k - 2] + dp0[k - 1])
    cols.append(a[..., k - 1] + (a[..., k - 1] - a[..., k - 2]) * r)
    return torch.stack(cols, dim=-1)


def update_dz_c_torch(f, area, dp0, n, nz, dt):
    """UpdateGeopotentialHeightOnCGrid on oracle-layout tensors [6, i, j, k]
    with differentiable torch ops: returns the new (gz, ws)."""
    s, e, nk = H, H + n - 1, nz + 1
    m = n + 2 * H + 1
    mx, my = corner_maps(n, nz)
    gz, ut, vt = f["gz"], f["ut"], f["vt"]
    gzf = gz.reshape(6, m * m, nk)
    gz_x = gzf[:, mx, :].reshape(6, m, m, nk)
    gz_y = gzf[:, my, :].reshape(6, m, m, nk)
    xfx, yfx = _p_weighted(ut, dp0, nk), _p_weighted(vt, dp0, nk)
    B, B1 = slice(s - 1, e + 2), slice(s, e + 3)
    I, Im = slice(s - 1, e + 3), slice(s - 2, e + 2)
    fx = xfx[:, I, B] * torch.where(xfx[:, I, B] > 0, gz_x[:, Im, B], gz_x[:, I, B])
    fy = yfx[:, B, I] * torch.where(yfx[:, B, I] > 0, gz_y[:, B, Im], gz_y[:, B, I])
    a = area[:, B, B, None]
    num = gz_y[:, B, B] * a + fx[:, :-1] - fx[:, 1:] + fy[:, :, :-1] - fy[:, :, 1:]
    den = a + xfx[:, B, B] - xfx[:, B1, B] + yfx[:, B, B] - yfx[:, B, B1]
    new = num / den
    below = new[..., nk - 1]
    outs = [None] * nk
    outs[nk - 1] = below
    ws_box = (f["zs"][:, B, B] - below) * (1.0 / dt)
    for k in range(nk - 2, -1, -1):
        v = new[..., k]
        kp1 = below + DZ_MIN
        below = torch.where(v > kp1, v, kp1)
        outs[k] = below
    gz_out = gz.clone()
    gz_out[:, B, B, :] = torch.stack(outs, dim=-1)
    ws_out = f["ws"].clone()
    ws_out[:, B, B] = ws_box
    return gz_out, ws_out


def _area(n):
    return torch.from_numpy(np.ascontiguousarray(np.asarray(cases.grid_for(n).area)))


@pytest.mark.parametrize("thin", [False, True])
def test_torch_restatement_matches_oracle(thin):
    from oracle._util import Tile
    from oracle.updatedz import update_dz_c

    n, nz = 12, 8
    case = uzc_case(n, nz, 4, thin)
    ref_gz, ref_ws = case["gz"].copy(), case["ws"].copy()
    for t in range(6):
        update_dz_c(Tile(n, nz), cases.metric_namespace(n, t), case["dp_ref"], case["zs"][t], case["ut"][t],
                    case["vt"][t], ref_gz[t], ref_ws[t], DT2)
    f = {k: torch.from_numpy(v.copy()) for k, v in case.items() if k != "dp_ref"}
    gz, ws = update_dz_c_torch(f, _area(n), case["dp_ref"], n, nz, DT2)
    assert np.max(np.abs(gz.numpy() - ref_gz)) <= 1e-12 * np.max(np.abs(ref_gz))
    assert np.max(np.abs(ws.numpy() - ref_ws)) <= 1e-12 * np.max(np.abs(ref_ws))
    if thin:  # the floor acted somewhere
        box = (slice(None), slice(H - 1, H + n + 1), slice(H - 1, H + n + 1))
        assert (np.diff(ref_gz[box], axis=-1) == -DZ_MIN).any()


@pytest.fixture(scope="module")
def host_adjoint(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    so = str(tmp_path_factory.mktemp("uzc") / "uzc_adjoint.so")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-o", so,
                           os.path.join(ROOT, "tests", "native", "updatedzc_adjoint_host.cpp")])
    lib = ctypes.CDLL(so)
    lib.uzc_forward_host.restype = None
    lib.uzc_adjoint_host.restype = None
    return lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _ints(n, nz):
    return ctypes.c_int(n), ctypes.c_int(H), ctypes.c_int(nz), ctypes.c_double(DT2)


@pytest.mark.parametrize("thin", [False, True])
def test_host_forward_matches_oracle(host_adjoint, thin):
    # the adjoint's recomputation of the forward is the stage's forward
    from oracle._util import Tile
    from oracle.updatedz import update_dz_c

    n, nz = 12, 8
    case = uzc_case(n, nz, 6, thin)
    ref_gz, ref_ws = case["gz"].copy(), case["ws"].copy()
    for t in range(6):
        update_dz_c(Tile(n, nz), cases.metric_namespace(n, t), case["dp_ref"], case["zs"][t], case["ut"][t],
                    case["vt"][t], ref_gz[t], ref_ws[t], DT2)
    k = {name: kernel_layout(case[name]) for name in ("zs", "ut", "vt", "gz")}
    area = kernel_layout(np.asarray(cases.grid_for(n).area))
    gz_out, ws_out = np.zeros_like(k["gz"]), np.zeros_like(k["zs"])
    host_adjoint.uzc_forward_host(*_ints(n, nz), _ptr(case["dp_ref"]), _ptr(area), _ptr(k["zs"]), _ptr(k["ut"]),
                                  _ptr(k["vt"]), _ptr(k["gz"]), _ptr(gz_out), _ptr(ws_out))
    box3 = (slice(None), slice(None), slice(H - 1, H + n + 1), slice(H - 1, H + n + 1))
    want_gz, want_ws = kernel_layout(ref_gz)[box3], kernel_layout(ref_ws)[box3[0:1] + box3[2:]]
    assert np.max(np.abs(gz_out[box3] - want_gz)) <= 1e-12 * np.max(np.abs(want_gz))
    assert np.max(np.abs(ws_out[box3[0:1] + box3[2:]] - want_ws)) <= 1e-12 * np.max(np.abs(want_ws))


def torch_grads(case, n, nz, g_gz, g_ws):
    """Gradients (oracle layout) of <g_gz, gz_new> + <g_ws, ws_new>."""
    f = {k: torch.from_numpy(v.copy()) for k, v in case.items() if k != "dp_ref"}
    for k in ("ut", "vt", "gz", "ws"):
        f[k].requires_grad_(True)
    gz, ws = update_dz_c_torch(f, _area(n), case["dp_ref"], n, nz, DT2)
    ((gz * torch.from_numpy(g_gz)).sum() + (ws * torch.from_numpy(g_ws)).sum()).backward()
    return {k: f[k].grad.numpy() for k in ("ut", "vt", "gz", "ws")}


@pytest.mark.parametrize("n,nz,seed,thin", [(12, 8, 6, False), (12, 8, 7, True), (16, 5, 8, True)])
def test_host_adjoint_matches_torch_autograd(host_adjoint, n, nz, seed, thin):
    case = uzc_case(n, nz, seed, thin)
    rng = np.random.default_rng(seed + 1)
    g_gz = rng.standard_normal(case["gz"].shape)
    g_ws = rng.standard_normal(case["ws"].shape)
    ref = torch_grads(case, n, nz, g_gz, g_ws)
    k = {name: kernel_layout(case[name]) for name in ("ut", "vt", "gz")}
    area = kernel_layout(np.asarray(cases.grid_for(n).area))
    out = {name: np.zeros_like(k["gz"]) for name in ("gz", "ut", "vt", "hnew", "g_new")}
    host_adjoint.uzc_adjoint_host(*_ints(n, nz), _ptr(case["dp_ref"]), _ptr(area), _ptr(k["ut"]), _ptr(k["vt"]),
                                  _ptr(k["gz"]), _ptr(kernel_layout(g_gz)), _ptr(kernel_layout(g_ws)),
                                  _ptr(out["gz"]), _ptr(out["ut"]), _ptr(out["vt"]), _ptr(out["hnew"]),
                                  _ptr(out["g_new"]))
    for name in ("gz", "ut", "vt"):
        b = kernel_layout(ref[name])
        err = np.max(np.abs(out[name] - b)) / np.max(np.abs(b))
        assert err <= 1e-12, (name, err)


# ---------------------------------------------------------------- GPU


@pytest.mark.gpu
@pytest.mark.parametrize("thin", [False, True])
def test_gpu_adjoint_matches_torch_autograd(thin):
    import gpu_runs

    from fv3core_b200.adjoint import update_dz_c
    from fv3core_b200.stencils.updatedzc import UpdateGeopotentialHeightOnCGrid
    from fv3core_b200.storage import to_device, to_host

    n, nz = 12, 8
    case = uzc_case(n, nz, 7, thin)
    gd, sf = gpu_runs.device_grid(n, nz)
    dev = {k: to_device(v) for k, v in case.items()}
    for k in ("ut", "vt", "gz", "ws"):
        dev[k].requires_grad_(True)
    gz, ws = update_dz_c(dev["dp_ref"], dev["zs"], dev["ut"], dev["vt"], dev["gz"], dev["ws"], sf, DT2)
    # the forward is the stage's own
    gz2, ws2 = dev["gz"].detach().clone(), dev["ws"].detach().clone()
    UpdateGeopotentialHeightOnCGrid(sf, gd.area)(dev["dp_ref"], dev["zs"], dev["ut"].detach(), dev["vt"].detach(),
                                                 gz2, ws2, DT2)
    assert torch.equal(gz, gz2) and torch.equal(ws, ws2)
    rng = np.random.default_rng(3)
    g_gz = rng.standard_normal(case["gz"].shape)
    g_ws = rng.standard_normal(case["ws"].shape)
    ((gz * to_device(g_gz)).sum() + (ws * to_device(g_ws)).sum()).backward()
    ref = torch_grads(case, n, nz, g_gz, g_ws)
    for k in ("ut", "vt", "gz", "ws"):
        a, b = to_host(dev[k].grad), ref[k]
        err = np.max(np.abs(a - b)) / np.max(np.abs(b))
        assert err <= 1e-11, (k, err)


@pytest.mark.gpu
def test_gpu_chain_update_dz_c_riemann_c_p_grad_c_matches_torch_autograd():
    # the C-grid vertical part of the acoustic loop (dyn_core.py): the
    # advected heights and surface w feed RiemannSolverC, whose pef and gz
    # feed p_grad_c; gradients of the new uc, vc reach ut, vt, gz, w3, delpc,
    # ptc, uc and vc through three hand-written adjoints
    import gpu_runs
    import torch_riem3
    from test_pgrad_adjoint import _metrics, p_grad_c_torch
    from test_riem_adjoint import riemc_case

    from fv3core_b200.adjoint import p_grad_c, riem_solver_c, update_dz_c
    from fv3core_b200.storage import to_device, to_host

    n, nz, seed = 12, 16, 11
    K = nz + 1
    case, cols, par = riemc_case(n, nz, seed)
    st = cases.base_state(n, nz, seed)
    rng = np.random.default_rng(31)
    shp = case["gz"].shape
    area = np.asarray(cases.grid_for(n).area)[:, :, :, None]
    case.update(ut=0.02 * area * rng.standard_normal(shp), vt=0.02 * area * rng.standard_normal(shp),
                uc=10 * rng.standard_normal(shp), vc=10 * rng.standard_normal(shp),
                dp_ref=dp_ref_of(st, nz), zs=st["phis"] * (1.0 / 9.80665))
    leaves = ("ut", "vt", "gz", "w3", "delpc", "ptc", "uc", "vc")
    gd, sf = gpu_runs.device_grid(n, nz)
    dev = {k: to_device(case[k]) for k in leaves + ("cappa", "q_con", "hs", "ws", "dp_ref", "zs")}
    for k in leaves:
        dev[k].requires_grad_(True)
    gz1, ws1 = update_dz_c(dev["dp_ref"], dev["zs"], dev["ut"], dev["vt"], dev["gz"], dev["ws"], sf, par["dt2"])
    pef, gz2 = riem_solver_c(dev["w3"], gz1, dev["delpc"], dev["ptc"], dev["cappa"], dev["hs"], ws1, dev["q_con"],
                             sf.grid_indexing, par["dt2"], par["ptop"], par["p_fac"])
    uc, vc = p_grad_c(dev["uc"], dev["vc"], dev["delpc"], pef, gz2, sf, par["dt2"])
    gu, gv = rng.standard_normal(uc.shape), rng.standard_normal(vc.shape)
    ((uc * torch.from_numpy(gu).cuda()).sum() + (vc * torch.from_numpy(gv).cuda()).sum()).backward()

    # the same chain in torch ops on the host, leaves in the oracle layout
    T = {k: torch.from_numpy(case[k].copy()).requires_grad_(True) for k in leaves}
    fixed = {k: torch.from_numpy(np.asarray(case[k], dtype=np.float64).copy()) for k in ("zs", "ws")}
    gz1_o, ws1_o = update_dz_c_torch({"gz": T["gz"], "ut": T["ut"], "vt": T["vt"], **fixed}, _area(n),
                                     case["dp_ref"], n, nz, par["dt2"])
    R = slice(H - 1, H + n + 1)

    def cols_of(t):  # oracle layout [6, i, j, k] -> [ncol, K]
        return t[:, R, R].reshape(6 * (n + 2) ** 2, -1)

    def kern(t):  # oracle layout -> kernel layout
        return t.permute(0, 3, 2, 1)

    fc = {k: torch.from_numpy(cols[k]) for k in ("cappa", "q_con", "hs")}
    pef_c, gz_c = torch_riem3.riemc_columns(cols_of(T["w3"]), cols_of(gz1_o), cols_of(T["delpc"]),
                                            cols_of(T["ptc"]), fc["cappa"], fc["q_con"], fc["hs"],
                                            ws1_o[:, R, R].reshape(-1), par["dt2"], par["ptop"], par["p_fac"])
    pef_o = torch.zeros_like(gz1_o)
    pef_o[:, R, R] = pef_c.reshape(6, n + 2, n + 2, K)
    gz2_o = gz1_o.clone()
    gz2_o[:, R, R] = gz_c.reshape(6, n + 2, n + 2, K)
    rdxc, rdyc = (torch.from_numpy(a) for a in _metrics(n))
    f = {"uc": kern(T["uc"]), "vc": kern(T["vc"]), "delpc": kern(T["delpc"]), "pkc": kern(pef_o),
         "gz": kern(gz2_o)}
    uc_t, vc_t = p_grad_c_torch(f, rdxc, rdyc, par["dt2"], n, nz)
    ((uc_t * torch.from_numpy(gu)).sum() + (vc_t * torch.from_numpy(gv)).sum()).backward()
    for k in leaves:
        a, b = to_host(dev[k].grad), T[k].grad.numpy()
        err = np.max(np.abs(a - b)) / np.max(np.abs(b))
        assert err <= 1e-10, (k, err)

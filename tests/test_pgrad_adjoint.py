"""The hand-written adjoint of p_grad_c_stencil (dyn_core.py:101-145):
fv3core_b200/csrc/pgrad_adjoint.h built for the host and compared with torch
autograd of a PyTorch-ops restatement (itself equal to the oracle), then the
device build behind fv3core_b200.adjoint.p_grad_c on the GPU."""
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


def pgc_case(n, nz, seed):
    """Seeded inputs in the oracle's [6, i, j, k] order."""
    st = cases.base_state(n, nz, seed)
    rng = np.random.default_rng(seed + 77)
    shp = st["delp"].shape
    return {
        "uc": 10 * rng.standard_normal(shp),
        "vc": 10 * rng.standard_normal(shp),
        "delpc": st["delp"] * (1 + 1e-3 * rng.standard_normal(shp)),
        "pkc": st["pe"] * (1 + 1e-4 * rng.standard_normal(shp)),
        "gz": cases.heights(st, nz) * 9.80665,
    }


def kernel_layout(a):
    """[6, i, j, k] -> [6, k, j, i] (2-D: [6, i, j] -> [6, j, i])."""
    return np.ascontiguousarray(a.transpose(0, 3, 2, 1) if a.ndim == 4 else a.transpose(0, 2, 1))


def p_grad_c_torch(f, rdxc, rdyc, dt2, n, nz):
    """p_grad_c on kernel-layout tensors with differentiable torch ops."""
    s, e = H, H + n - 1
    P, Pm, K, K1 = slice(s, e + 2), slice(s - 1, e + 1), slice(0, nz), slice(1, nz + 1)
    delpc, pkc, gz = f["delpc"], f["pkc"], f["gz"]

    def incr(rd, q):  # q: the neighbour's (j, i) slices
        p = (P, P)
        at = lambda a, kk, ji: a[(slice(None), kk) + ji]  # noqa: E731
        D = at(delpc, K, q) + at(delpc, K, p)
        A = (at(gz, K1, q) - at(gz, K, p)) * (at(pkc, K1, p) - at(pkc, K, q)) + \
            (at(gz, K, q) - at(gz, K1, p)) * (at(pkc, K1, q) - at(pkc, K, p))
        return dt2 * rd[:, None, P, P] / D * A

    uc, vc = f["uc"].clone(), f["vc"].clone()
    uc[:, K, P, P] = f["uc"][:, K, P, P] + incr(rdxc, (P, Pm))
    vc[:, K, P, P] = f["vc"][:, K, P, P] + incr(rdyc, (Pm, P))
    return uc, vc


def _metrics(n):
    g = cases.grid_for(n)
    return kernel_layout(np.asarray(g.rdxc)), kernel_layout(np.asarray(g.rdyc))


def test_torch_restatement_matches_oracle():
    from oracle._util import Tile
    from oracle.dyn_core import p_grad_c

    n, nz = 12, 8
    case = pgc_case(n, nz, 3)
    ref_uc, ref_vc = case["uc"].copy(), case["vc"].copy()
    for t in range(6):
        p_grad_c(Tile(n, nz), cases.metric_namespace(n, t), ref_uc[t], ref_vc[t], case["delpc"][t], case["pkc"][t],
                 case["gz"][t], DT2)
    f = {k: torch.from_numpy(kernel_layout(v)) for k, v in case.items()}
    rdxc, rdyc = (torch.from_numpy(a) for a in _metrics(n))
    uc, vc = p_grad_c_torch(f, rdxc, rdyc, DT2, n, nz)
    for a, b in ((uc, ref_uc), (vc, ref_vc)):
        b = kernel_layout(b)
        assert np.max(np.abs(a.numpy() - b)) <= 1e-13 * np.max(np.abs(b))


def torch_grads(case, n, nz, gu, gv):
    f = {k: torch.from_numpy(kernel_layout(v)).requires_grad_(True) for k, v in case.items()}
    rdxc, rdyc = (torch.from_numpy(a) for a in _metrics(n))
    uc, vc = p_grad_c_torch(f, rdxc, rdyc, DT2, n, nz)
    ((uc * torch.from_numpy(gu)).sum() + (vc * torch.from_numpy(gv)).sum()).backward()
    return {k: t.grad.numpy() for k, t in f.items()}


@pytest.fixture(scope="module")
def host_adjoint(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    so = str(tmp_path_factory.mktemp("pgc") / "pgc_adjoint.so")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-o", so,
                           os.path.join(ROOT, "tests", "native", "pgrad_adjoint_host.cpp")])
    return ctypes.CDLL(so)


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@pytest.mark.parametrize("n,nz,seed", [(12, 8, 3), (16, 5, 9)])
def test_host_adjoint_matches_torch_autograd(host_adjoint, n, nz, seed):
    case = pgc_case(n, nz, seed)
    rng = np.random.default_rng(seed)
    shp = kernel_layout(case["uc"]).shape
    gu, gv = rng.standard_normal(shp), rng.standard_normal(shp)
    ref = torch_grads(case, n, nz, gu, gv)
    np.testing.assert_array_equal(ref["uc"], gu)
    np.testing.assert_array_equal(ref["vc"], gv)
    f = {k: kernel_layout(v) for k, v in case.items()}
    rdxc, rdyc = _metrics(n)
    out = {k: np.zeros(shp) for k in ("delpc", "pkc", "gz")}
    host_adjoint.pgc_adjoint_host(
        ctypes.c_int(n), ctypes.c_int(H), ctypes.c_int(nz), ctypes.c_double(DT2), _ptr(rdxc), _ptr(rdyc),
        _ptr(f["delpc"]), _ptr(f["pkc"]), _ptr(f["gz"]), _ptr(gu), _ptr(gv), _ptr(out["delpc"]), _ptr(out["pkc"]),
        _ptr(out["gz"]))
    for k in out:
        b = ref[k]
        err = np.max(np.abs(out[k] - b)) / np.max(np.abs(b))
        assert err <= 1e-14, (k, err)
    # nothing outside the adjoint's box depends on the update
    outside = np.ones(shp, bool)
    outside[:, :, H - 1:H + n + 1, H - 1:H + n + 1] = False
    for k in out:
        assert not ref[k][outside].any()


# ---------------------------------------------------------------- GPU


@pytest.mark.gpu
def test_gpu_adjoint_matches_torch_autograd():
    import gpu_runs

    from fv3core_b200.adjoint import p_grad_c
    from fv3core_b200.stencils.p_grad_c import PGradC

    n, nz = 12, 8
    case = pgc_case(n, nz, 3)
    gd, sf = gpu_runs.device_grid(n, nz)
    dev = {k: torch.from_numpy(kernel_layout(v)).cuda().requires_grad_(True) for k, v in case.items()}
    uc, vc = p_grad_c(dev["uc"], dev["vc"], dev["delpc"], dev["pkc"], dev["gz"], sf, DT2)
    # the forward is the stage's own
    uc2, vc2 = dev["uc"].detach().clone(), dev["vc"].detach().clone()
    PGradC(sf)(gd.rdxc, gd.rdyc, uc2, vc2, dev["delpc"].detach(), dev["pkc"].detach(), dev["gz"].detach(), DT2)
    assert torch.equal(uc, uc2) and torch.equal(vc, vc2)
    rng = np.random.default_rng(5)
    gu, gv = rng.standard_normal(uc.shape), rng.standard_normal(vc.shape)
    ((uc * torch.from_numpy(gu).cuda()).sum() + (vc * torch.from_numpy(gv).cuda()).sum()).backward()
    ref = torch_grads(case, n, nz, gu, gv)
    for k in dev:
        a = dev[k].grad.cpu().numpy()
        b = ref[k]
        err = np.max(np.abs(a - b)) / np.max(np.abs(b))
        assert err <= 1e-12, (k, err)


@pytest.mark.gpu
def test_gpu_chain_riemann_c_then_p_grad_c_matches_torch_autograd():
    # RiemannSolverC's pef and gz feed p_grad_c as pkc and gz (dyn_core.py
    # acoustic loop): the two autograd Functions compose on the device
    import gpu_runs
    import torch_riem3
    from test_riem_adjoint import riemc_case

    from fv3core_b200.adjoint import p_grad_c, riem_solver_c
    from fv3core_b200.storage import to_device

    n, nz = 12, 16
    K = nz + 1
    case, cols, par = riemc_case(n, nz)
    rng = np.random.default_rng(21)
    shp = case["delpc"].shape
    case["uc"], case["vc"] = 10 * rng.standard_normal(shp), 10 * rng.standard_normal(shp)
    leaves = ("w3", "gz", "delpc", "ptc", "uc", "vc")
    gd, sf = gpu_runs.device_grid(n, nz)
    dev = {k: to_device(case[k]) for k in leaves + ("cappa", "q_con", "hs", "ws")}
    for k in leaves:
        dev[k].requires_grad_(True)
    pef, gz = riem_solver_c(dev["w3"], dev["gz"], dev["delpc"], dev["ptc"], dev["cappa"], dev["hs"], dev["ws"],
                            dev["q_con"], sf.grid_indexing, par["dt2"], par["ptop"], par["p_fac"])
    uc, vc = p_grad_c(dev["uc"], dev["vc"], dev["delpc"], pef, gz, sf, par["dt2"])
    gu, gv = rng.standard_normal(uc.shape), rng.standard_normal(vc.shape)
    ((uc * torch.from_numpy(gu).cuda()).sum() + (vc * torch.from_numpy(gv).cuda()).sum()).backward()

    # the same chain in torch ops on the host, with kernel-layout leaves
    T = {k: torch.from_numpy(kernel_layout(case[k])).requires_grad_(True) for k in leaves}
    R = slice(H - 1, H + n + 1)

    def cols_of(t):
        return t[:, :, R, R].permute(0, 3, 2, 1).reshape(6 * (n + 2) ** 2, -1)

    def full_of(c):
        return c.reshape(6, n + 2, n + 2, K).permute(0, 3, 2, 1)

    fixed = {k: torch.from_numpy(cols[k]) for k in ("cappa", "q_con", "hs", "ws")}
    pef_c, gz_c = torch_riem3.riemc_columns(cols_of(T["w3"]), cols_of(T["gz"]), cols_of(T["delpc"]),
                                            cols_of(T["ptc"]), fixed["cappa"], fixed["q_con"], fixed["hs"],
                                            fixed["ws"], par["dt2"], par["ptop"], par["p_fac"])
    pef_t = torch.zeros_like(T["gz"])
    pef_t[:, :, R, R] = full_of(pef_c)
    gz_t = T["gz"].clone()
    gz_t[:, :, R, R] = full_of(gz_c)
    rdxc, rdyc = (torch.from_numpy(a) for a in _metrics(n))
    f = {"uc": T["uc"], "vc": T["vc"], "delpc": T["delpc"], "pkc": pef_t, "gz": gz_t}
    uc_t, vc_t = p_grad_c_torch(f, rdxc, rdyc, par["dt2"], n, nz)
    ((uc_t * torch.from_numpy(gu)).sum() + (vc_t * torch.from_numpy(gv)).sum()).backward()
    for k in leaves:
        a, b = dev[k].grad.cpu().numpy(), T[k].grad.numpy()
        err = np.max(np.abs(a - b)) / np.max(np.abs(b))
        assert err <= 1e-10, (k, err)

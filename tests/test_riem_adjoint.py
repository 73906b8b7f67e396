"""The hand-written adjoint of RiemannSolver3's column solve
(fv3core_b200/csrc/riem_adjoint.h) against torch autograd of the PyTorch-ops
restatement (tests/torch_riem3.py), and that restatement's gradients against
central finite differences.  The header is compiled for the host here; the
GPU tests run the same code on the device through the C ABI."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest
import torch

import cases
import torch_riem3

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
H = 3


def riem3_case(n=12, nz=8, seed=5):
    """Compute-domain columns of a baroclinic state, as [ncol, K] arrays."""
    st = cases.base_state(n, nz, seed)
    rng = np.random.default_rng(seed + 77)
    shp = st["delp"].shape
    f = {"cappa": st["cappa"], "q_con": st["q_con"], "delp": st["delp"], "pt": st["pt"],
         "zh": cases.heights(st, nz) * (1.0 + 1e-4 * rng.standard_normal(shp)), "w": 0.1 * rng.standard_normal(shp)}
    cols = {k: np.ascontiguousarray(v[:, H:H + n, H:H + n, :].reshape(6 * n * n, -1)) for k, v in f.items()}
    cols["wsr"] = np.ascontiguousarray((0.01 * rng.standard_normal(shp[:3]))[:, H:H + n, H:H + n].reshape(-1))
    return cols, dict(dt=37.5, ptop=float(st["ptop"]), p_fac=0.05)


def torch_grads(cols, par, gw, gdz):
    T = {k: torch.from_numpy(v.copy()) for k, v in cols.items()}
    for k in ("w", "zh", "delp", "pt", "wsr"):
        T[k].requires_grad_(True)
    w_new, dz_new = torch_riem3.riem3_columns(T["w"], T["zh"], T["delp"], T["pt"], T["cappa"], T["q_con"], T["wsr"],
                                              par["dt"], par["ptop"], par["p_fac"])
    loss = (w_new * torch.from_numpy(gw)).sum() + (dz_new * torch.from_numpy(gdz)).sum()
    loss.backward()
    K = cols["zh"].shape[1]
    return {k: T[k].grad.numpy() for k in ("w", "zh", "delp", "pt", "wsr")}, K


@pytest.fixture(scope="module")
def host_adjoint(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no host compiler")
    so = str(tmp_path_factory.mktemp("adj") / "libriemadj.so")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-o", so,
                           os.path.join(ROOT, "tests", "native", "riem_adjoint_host.cpp")])
    return ctypes.CDLL(so)


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def test_host_adjoint_matches_torch_autograd(host_adjoint):
    cols, par = riem3_case()
    ncol, K = cols["zh"].shape
    rng = np.random.default_rng(11)
    gw = rng.standard_normal((ncol, K - 1))
    gdz = rng.standard_normal((ncol, K - 1)) * 1e-2
    ref, _ = torch_grads(cols, par, gw, gdz)
    gw_k = np.zeros((ncol, K)); gw_k[:, :K - 1] = gw
    gdz_k = np.zeros((ncol, K)); gdz_k[:, :K - 1] = gdz
    out = {k: np.zeros((ncol, K)) for k in ("w", "zh", "delp", "pt")}
    out["wsr"] = np.zeros(ncol)
    f = host_adjoint.riem3_adjoint_columns
    f.restype = None
    f(ctypes.c_int(ncol), ctypes.c_int(K), ctypes.c_double(par["dt"]), ctypes.c_double(par["ptop"]),
      ctypes.c_double(par["p_fac"]), _ptr(cols["wsr"]), _ptr(cols["w"]), _ptr(cols["zh"]), _ptr(cols["delp"]),
      _ptr(cols["pt"]), _ptr(cols["cappa"]), _ptr(cols["q_con"]), _ptr(gw_k), _ptr(gdz_k),
      _ptr(out["w"]), _ptr(out["zh"]), _ptr(out["delp"]), _ptr(out["pt"]), _ptr(out["wsr"]))
    for k, width in (("w", K - 1), ("zh", K), ("delp", K - 1), ("pt", K - 1), ("wsr", None)):
        a, b = (out[k], ref[k]) if width is None else (out[k][:, :width], ref[k][:, :width])
        err = np.max(np.abs(a - b)) / np.max(np.abs(b))
        assert err <= 1e-12, (k, err)


def riemc_case(n=12, nz=16, seed=11):
    """The RiemannSolverC case's columns (is-1..ie+1, js-1..je+1) as [ncol, K]."""
    case = cases.riem_solver_c_case(n, nz, seed)
    sl = (slice(None), slice(H - 1, H + n + 1), slice(H - 1, H + n + 1))
    cols = {k: np.ascontiguousarray(case[k][sl].reshape(6 * (n + 2) ** 2, -1))
            for k in ("w3", "gz", "delpc", "ptc", "cappa", "q_con")}
    cols["hs"] = np.ascontiguousarray(case["hs"][sl].reshape(-1))
    cols["ws"] = np.ascontiguousarray(case["ws"][sl].reshape(-1))
    return case, cols, dict(dt2=case["dt2"], ptop=float(case["ptop"]), p_fac=case["p_fac"])


def riemc_torch(cols, par, requires_grad=False):
    T = {k: torch.from_numpy(v.copy()) for k, v in cols.items()}
    if requires_grad:
        for k in ("w3", "gz", "delpc", "ptc", "ws"):
            T[k].requires_grad_(True)
    pef, gz = torch_riem3.riemc_columns(T["w3"], T["gz"], T["delpc"], T["ptc"], T["cappa"], T["q_con"], T["hs"],
                                        T["ws"], par["dt2"], par["ptop"], par["p_fac"])
    return T, pef, gz


def test_riemc_restatement_matches_oracle():
    from oracle.riem_solver_c import riem_solver_c

    n, nz = 12, 16
    case, cols, par = riemc_case(n, nz)
    ref = {k: (np.array(v, copy=True) if isinstance(v, np.ndarray) else v) for k, v in case.items()}
    for t in range(6):
        riem_solver_c(ref["dt2"], ref["cappa"][t], ref["ptop"], ref["hs"][t], ref["ws"][t], ref["ptc"][t],
                      ref["q_con"][t], ref["delpc"][t], ref["gz"][t], ref["pef"][t], ref["w3"][t], ref["p_fac"], n, nz)
    _, pef, gz = riemc_torch(cols, par)
    sl = (slice(None), slice(H - 1, H + n + 1), slice(H - 1, H + n + 1))
    for name, mine in (("pef", pef), ("gz", gz)):
        want = ref[name][sl].reshape(6 * (n + 2) ** 2, -1)
        err = np.max(np.abs(mine.detach().numpy() - want) / np.maximum(np.abs(want), 1e-30))
        assert err <= 1e-11, (name, err)


def test_host_riemc_adjoint_matches_torch_autograd(host_adjoint):
    _, cols, par = riemc_case()
    ncol, K = cols["gz"].shape
    rng = np.random.default_rng(12)
    gpef = rng.standard_normal((ncol, K)) * 1e-3
    ggz = rng.standard_normal((ncol, K))
    T, pef, gz = riemc_torch(cols, par, requires_grad=True)
    ((pef * torch.from_numpy(gpef)).sum() + (gz * torch.from_numpy(ggz)).sum()).backward()
    out = {k: np.zeros((ncol, K)) for k in ("w3", "gz", "delpc", "ptc")}
    out["ws"] = np.zeros(ncol)
    f = host_adjoint.riemc_adjoint_columns
    f.restype = None
    f(ctypes.c_int(ncol), ctypes.c_int(K), ctypes.c_double(par["dt2"]), ctypes.c_double(par["ptop"]),
      ctypes.c_double(par["p_fac"]), _ptr(cols["ws"]), _ptr(cols["w3"]), _ptr(cols["gz"]), _ptr(cols["delpc"]),
      _ptr(cols["ptc"]), _ptr(cols["cappa"]), _ptr(cols["q_con"]), _ptr(gpef), _ptr(ggz),
      _ptr(out["w3"]), _ptr(out["gz"]), _ptr(out["delpc"]), _ptr(out["ptc"]), _ptr(out["ws"]))
    for k, width in (("w3", K - 1), ("gz", K), ("delpc", K - 1), ("ptc", K - 1), ("ws", None)):
        b = T[k].grad.numpy()
        a, b = (out[k], b) if width is None else (out[k][:, :width], b[:, :width])
        err = np.max(np.abs(a - b)) / np.max(np.abs(b))
        assert err <= 1e-12, (k, err)


def test_torch_restatement_gradients_match_finite_differences():
    cols, par = riem3_case(n=4, nz=8, seed=9)
    ncol, K = cols["zh"].shape
    rng = np.random.default_rng(3)
    gw = rng.standard_normal((ncol, K - 1))
    gdz = rng.standard_normal((ncol, K - 1)) * 1e-2
    grads, _ = torch_grads(cols, par, gw, gdz)

    def loss(c):
        T = {k: torch.from_numpy(v) for k, v in c.items()}
        w_new, dz_new = torch_riem3.riem3_columns(T["w"], T["zh"], T["delp"], T["pt"], T["cappa"], T["q_con"],
                                                  T["wsr"], par["dt"], par["ptop"], par["p_fac"])
        return float((w_new.numpy() * gw).sum() + (dz_new.numpy() * gdz).sum())

    for trial in range(4):
        d = {k: rng.standard_normal(cols[k].shape) * np.abs(cols[k]) for k in ("w", "zh", "delp", "pt", "wsr")}
        eps = 1e-6
        cp = {k: v.copy() for k, v in cols.items()}
        cm = {k: v.copy() for k, v in cols.items()}
        for k in d:
            cp[k] = cols[k] + eps * d[k]
            cm[k] = cols[k] - eps * d[k]
        fd = (loss(cp) - loss(cm)) / (2 * eps)
        ad = sum(float((grads[k] * d[k]).sum()) for k in d)
        assert abs(fd - ad) <= 1e-5 * abs(ad), (trial, fd, ad)


# ---------------------------------------------------------------- GPU


def _device_case(n, nz, seed):
    """Full device fields of a RiemannSolver3 case and its [ncol, K] columns."""
    from fv3core_b200.storage import to_device

    st = cases.base_state(n, nz, seed)
    rng = np.random.default_rng(seed + 77)
    shp = st["delp"].shape
    f = {"cappa": st["cappa"], "q_con": st["q_con"], "delp": st["delp"], "pt": st["pt"],
         "zh": cases.heights(st, nz) * (1.0 + 1e-4 * rng.standard_normal(shp)), "w": 0.1 * rng.standard_normal(shp)}
    wsd = 0.01 * rng.standard_normal(shp[:3])
    zs = st["phis"] * (1.0 / 9.80665)
    dev = {k: to_device(v) for k, v in f.items()}
    dev["wsd"], dev["zs"] = to_device(wsd), to_device(zs)
    cols = {k: np.ascontiguousarray(v[:, H:H + n, H:H + n, :].reshape(6 * n * n, -1)) for k, v in f.items()}
    cols["wsr"] = np.ascontiguousarray(wsd[:, H:H + n, H:H + n].reshape(-1))
    return dev, cols, dict(dt=37.5, ptop=float(st["ptop"]), p_fac=0.05)


def _to_cols(t, n):
    from fv3core_b200.storage import to_host

    return to_host(t)[:, H:H + n, H:H + n, :].reshape(6 * n * n, -1)


@pytest.mark.gpu
@pytest.mark.parametrize("n,nz,seed", [(12, 8, 5), (24, 79, 6)])
def test_gpu_adjoint_matches_torch_autograd(n, nz, seed):
    from fv3core_b200.adjoint import riem_solver3
    from fv3core_b200.storage import GridIndexing

    dev, cols, par = _device_case(n, nz, seed)
    gi = GridIndexing((n, n, nz), H)
    for k in ("w", "zh", "delp", "pt", "wsd"):
        dev[k].requires_grad_(True)
    w_new, dz_new = riem_solver3(dev["w"], dev["zh"], dev["delp"], dev["pt"], dev["cappa"], dev["zs"], dev["wsd"],
                                 dev["q_con"], gi, par["dt"], par["ptop"], par["p_fac"])
    gen = torch.Generator(device="cuda").manual_seed(seed)
    gw = torch.randn(w_new.shape, dtype=w_new.dtype, device=w_new.device, generator=gen)
    gdz = 1e-2 * torch.randn(dz_new.shape, dtype=dz_new.dtype, device=dz_new.device, generator=gen)
    gdz[:, nz:] = 0.0
    ((w_new * gw).sum() + (dz_new * gdz).sum()).backward()
    K = nz + 1
    ref, _ = torch_grads(cols, par, _to_cols(gw, n)[:, :K - 1], _to_cols(gdz, n)[:, :K - 1])
    for k, width in (("w", K - 1), ("zh", K), ("delp", K - 1), ("pt", K - 1)):
        a = _to_cols(dev[k].grad, n)[:, :width]
        b = ref[k][:, :width]
        err = np.max(np.abs(a - b)) / np.max(np.abs(b))
        assert err <= 1e-10, (k, err)
    from fv3core_b200.storage import to_host

    g_wsd = to_host(dev["wsd"].grad)
    err = np.max(np.abs(g_wsd[:, H:H + n, H:H + n].reshape(-1) - ref["wsr"])) / np.max(np.abs(ref["wsr"]))
    assert err <= 1e-10, ("wsd", err)
    g_wsd[:, H:H + n, H:H + n] = 0.0
    assert not g_wsd.any()
    # outside the solved points w passes through
    gw_h, gwgrad_h = to_host(gw), to_host(dev["w"].grad)
    outside = np.ones(gw_h.shape, bool)
    outside[:, H:H + n, H:H + n, :nz] = False
    np.testing.assert_array_equal(gwgrad_h[outside], gw_h[outside])


@pytest.mark.gpu
def test_gpu_adjoint_matches_finite_differences_of_the_gpu_forward():
    from fv3core_b200.adjoint import riem_solver3
    from fv3core_b200.storage import GridIndexing

    n, nz = 12, 8
    dev, cols, par = _device_case(n, nz, 8)
    gi = GridIndexing((n, n, nz), H)
    gen = torch.Generator(device="cuda").manual_seed(4)
    gw = torch.randn(dev["w"].shape, dtype=torch.float64, device="cuda", generator=gen)
    gdz = 1e-2 * torch.randn(dev["w"].shape, dtype=torch.float64, device="cuda", generator=gen)

    def loss(w, zh, delp, pt):
        a, b = riem_solver3(w, zh, delp, pt, dev["cappa"], dev["zs"], dev["wsd"], dev["q_con"], gi, par["dt"],
                            par["ptop"], par["p_fac"])
        return (a * gw).sum() + (b * gdz).sum()

    x = {k: dev[k].clone().requires_grad_(True) for k in ("w", "zh", "delp", "pt")}
    loss(x["w"], x["zh"], x["delp"], x["pt"]).backward()
    for trial in range(4):
        d = {k: torch.randn(dev[k].shape, dtype=torch.float64, device="cuda", generator=gen) * dev[k].abs()
             for k in x}
        eps = 1e-6
        with torch.no_grad():
            lp = loss(*[dev[k] + eps * d[k] for k in ("w", "zh", "delp", "pt")])
            lm = loss(*[dev[k] - eps * d[k] for k in ("w", "zh", "delp", "pt")])
        fd = float((lp - lm) / (2 * eps))
        ad = sum(float((x[k].grad * d[k]).sum()) for k in x)
        assert abs(fd - ad) <= 1e-5 * abs(ad), (trial, fd, ad)


@pytest.mark.gpu
def test_gpu_riemc_adjoint_matches_torch_autograd():
    from fv3core_b200.adjoint import riem_solver_c
    from fv3core_b200.storage import GridIndexing, to_device, to_host

    n, nz = 12, 16
    case, cols, par = riemc_case(n, nz)
    gi = GridIndexing((n, n, nz), H)
    dev = {k: to_device(case[k]) for k in ("w3", "gz", "delpc", "ptc", "cappa", "q_con", "hs", "ws")}
    for k in ("w3", "gz", "delpc", "ptc", "ws"):
        dev[k].requires_grad_(True)
    pef, gz = riem_solver_c(dev["w3"], dev["gz"], dev["delpc"], dev["ptc"], dev["cappa"], dev["hs"], dev["ws"],
                            dev["q_con"], gi, par["dt2"], par["ptop"], par["p_fac"])
    gen = torch.Generator(device="cuda").manual_seed(2)
    gpef = 1e-3 * torch.randn(pef.shape, dtype=pef.dtype, device="cuda", generator=gen)
    ggz = torch.randn(gz.shape, dtype=gz.dtype, device="cuda", generator=gen)
    ((pef * gpef).sum() + (gz * ggz).sum()).backward()
    sl = (slice(None), slice(H - 1, H + n + 1), slice(H - 1, H + n + 1))

    def cols_of(t):
        return to_host(t)[sl].reshape(6 * (n + 2) ** 2, -1)

    T, pef_t, gz_t = riemc_torch(cols, par, requires_grad=True)
    ((pef_t * torch.from_numpy(cols_of(gpef))).sum() + (gz_t * torch.from_numpy(cols_of(ggz))).sum()).backward()
    K = nz + 1
    for k, width in (("w3", K - 1), ("gz", K), ("delpc", K - 1), ("ptc", K - 1)):
        a = cols_of(dev[k].grad)[:, :width]
        b = T[k].grad.numpy()[:, :width]
        err = np.max(np.abs(a - b)) / np.max(np.abs(b))
        assert err <= 1e-10, (k, err)
    g_ws = to_host(dev["ws"].grad)
    b = T["ws"].grad.numpy()
    err = np.max(np.abs(g_ws[sl].reshape(-1) - b)) / np.max(np.abs(b))
    assert err <= 1e-10, ("ws", err)

"""The acoustic-loop stages beside c_sw / d_sw / RiemannSolverC, one at a
time: CUDA through the package's classes vs the oracle on seeded inputs,
the oracle running the kernels' own exp/log/pow.  (The oracle of each stage
is pinned by the full-substep golden test.)"""
import numpy as np
import pytest

from oracle import _math

import cases
from metrics import parity_err

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _device_math():
    with _math.device_math():
        yield
H = 3
SIZES = [(12, 8, 3), (24, 16, 4), (12, 79, 5)]


def _state(n, nz, seed):
    st = cases.base_state(n, nz, seed)
    rng = np.random.default_rng(seed + 77)
    return st, rng


def _dp_ref(st, nz):
    ak, bk = np.asarray(st["ak"]), np.asarray(st["bk"])
    dp = np.zeros(nz + 1)
    dp[:nz] = ak[1:] - ak[:-1] + (bk[1:] - bk[:-1]) * 1.0e5
    return dp


def _check(gpu, ref, region=None, tol=1e-12):
    if region is not None:
        gpu, ref = gpu[region], ref[region]
    err = parity_err(gpu, ref)
    assert err <= tol, err


def _dev(a):
    from fv3core_b200.storage import to_device

    return to_device(a)


def _host(t):
    import torch

    from fv3core_b200.storage import to_host

    torch.cuda.synchronize()
    return to_host(t)


def _grid(n, nz):
    import gpu_runs

    return gpu_runs.device_grid(n, nz)


@pytest.mark.parametrize("n,nz,seed", SIZES)
def test_update_dz_c(n, nz, seed):
    from oracle._util import Tile
    from oracle.updatedz import update_dz_c

    from fv3core_b200.stencils.updatedzc import UpdateGeopotentialHeightOnCGrid

    st, rng = _state(n, nz, seed)
    g = cases.grid_for(n)
    dp = _dp_ref(st, nz)
    zs = st["phis"] * (1.0 / 9.80665)
    gz = cases.heights(st, nz)
    area = g.area[:, :, :, None]
    ut = 0.02 * area * rng.standard_normal(gz.shape)
    vt = 0.02 * area * rng.standard_normal(gz.shape)
    ws = np.zeros(zs.shape)
    dt2 = 18.75
    ref_gz, ref_ws = gz.copy(), ws.copy()
    for t in range(6):
        update_dz_c(Tile(n, nz), cases.metric_namespace(n, t), dp, zs[t], ut[t], vt[t], ref_gz[t], ref_ws[t], dt2)
    gd, sf = _grid(n, nz)
    d_gz, d_ws = _dev(gz), _dev(ws)
    UpdateGeopotentialHeightOnCGrid(sf, gd.area)(_dev(dp), _dev(zs), _dev(ut), _dev(vt), d_gz, d_ws, dt2)
    box = (slice(None), slice(H - 1, H + n + 1), slice(H - 1, H + n + 1))
    _check(_host(d_gz), ref_gz, box)
    _check(_host(d_ws), ref_ws, box)


@pytest.mark.parametrize("n,nz,seed", SIZES)
def test_update_dz_d(n, nz, seed):
    from oracle._util import Tile
    from oracle.d_sw import column_namelist
    from oracle.updatedz import UpdateDzDState, update_dz_d

    from fv3core_b200.config import baroclinic_dsw_config
    from fv3core_b200.stencils.d_sw import DGridShallowWaterLagrangianDynamics
    from fv3core_b200.stencils.updatedzd import UpdateHeightOnDGrid

    st, rng = _state(n, nz, seed)
    g = cases.grid_for(n)
    dp = _dp_ref(st, nz)
    zs = st["phis"] * (1.0 / 9.80665)
    zh = cases.heights(st, nz)
    shp = zh.shape
    area = g.area[:, :, :, None]
    crx, cry = 0.05 * rng.standard_normal(shp), 0.05 * rng.standard_normal(shp)
    xfx, yfx = 0.05 * area * rng.standard_normal(shp), 0.05 * area * rng.standard_normal(shp)
    wsd = np.zeros(zs.shape)
    dt = 37.5
    col = column_namelist(cases.DSW_CONFIG, nz)
    ref_zh, ref_wsd = zh.copy(), wsd.copy()
    for t in range(6):
        T = Tile(n, nz)
        with np.errstate(all="ignore"):
            update_dz_d(T, cases.metric_namespace(n, t), UpdateDzDState(T, dp, col), cases.DSW_CONFIG["hord_tm"],
                        zs[t], ref_zh[t], crx[t], cry[t], xfx[t], yfx[t], ref_wsd[t], dt)
    gd, sf = _grid(n, nz)
    DGridShallowWaterLagrangianDynamics(sf, gd, gd, None, False, False, baroclinic_dsw_config())
    up = UpdateHeightOnDGrid(sf, gd, gd, 0, cases.DSW_CONFIG["hord_tm"], dp, None)
    d_zh, d_wsd = _dev(zh), _dev(wsd)
    up(_dev(zs), d_zh, _dev(crx), _dev(cry), _dev(xfx), _dev(yfx), d_wsd, dt)
    box = (slice(None), slice(H, H + n), slice(H, H + n))
    _check(_host(d_zh), ref_zh, box)
    _check(_host(d_wsd), ref_wsd, box)


@pytest.mark.parametrize("n,nz,seed", SIZES)
@pytest.mark.parametrize("last_call", [False, True])
def test_riem_solver3(n, nz, seed, last_call):
    from oracle.riem_solver3 import riem_solver3

    from fv3core_b200.config import RiemannConfig
    from fv3core_b200.stencils.riem_solver3 import RiemannSolver3

    st, rng = _state(n, nz, seed)
    shp = st["delp"].shape
    zs = st["phis"] * (1.0 / 9.80665)
    f = {
        "cappa": st["cappa"], "delz": st["delz"].copy(), "q_con": st["q_con"], "delp": st["delp"], "pt": st["pt"],
        "zh": cases.heights(st, nz) * (1.0 + 1e-4 * rng.standard_normal(shp)), "pe": st["pe"].copy(),
        "ppe": np.zeros(shp), "pk3": np.zeros(shp), "pk": st["pk"].copy(), "peln": st["peln"].copy(),
        "w": 0.1 * rng.standard_normal(shp),
    }
    wsd = 0.01 * rng.standard_normal(shp[:3])
    dt, ptop, p_fac = 37.5, st["ptop"], 0.05
    ref = {k: np.array(v, copy=True) for k, v in f.items()}
    for t in range(6):
        riem_solver3(last_call, dt, ref["cappa"][t], ptop, zs[t], wsd[t], ref["delz"][t], ref["q_con"][t],
                     ref["delp"][t], ref["pt"][t], ref["zh"][t], ref["pe"][t], ref["ppe"][t], ref["pk3"][t],
                     ref["pk"][t], ref["peln"][t], ref["w"][t], p_fac, n, nz)
    gd, sf = _grid(n, nz)
    dev = {k: _dev(v) for k, v in f.items()}
    RiemannSolver3(sf, RiemannConfig(p_fac=p_fac, a_imp=1.0, use_logp=False, beta=0.0))(
        last_call, dt, dev["cappa"], ptop, _dev(zs), _dev(wsd), dev["delz"], dev["q_con"], dev["delp"], dev["pt"],
        dev["zh"], dev["pe"], dev["ppe"], dev["pk3"], dev["pk"], dev["peln"], dev["w"])
    box = (slice(None), slice(H, H + n), slice(H, H + n), slice(0, nz + 1))
    for k in ("delz", "zh", "pe", "ppe", "pk3", "pk", "peln", "w"):
        kb = box if k not in ("delz", "w") else box[:3] + (slice(0, nz),)
        _check(_host(dev[k]), ref[k], kb)


@pytest.mark.parametrize("n,nz,seed", SIZES)
def test_p_grad_c(n, nz, seed):
    from oracle._util import Tile
    from oracle.dyn_core import p_grad_c

    from fv3core_b200.stencils.p_grad_c import PGradC

    st, rng = _state(n, nz, seed)
    shp = st["delp"].shape
    uc, vc = 10 * rng.standard_normal(shp), 10 * rng.standard_normal(shp)
    delpc = st["delp"] * (1 + 1e-3 * rng.standard_normal(shp))
    pkc = st["pe"] * (1 + 1e-4 * rng.standard_normal(shp))
    gz = cases.heights(st, nz) * 9.80665
    dt2 = 18.75
    ref_uc, ref_vc = uc.copy(), vc.copy()
    for t in range(6):
        p_grad_c(Tile(n, nz), cases.metric_namespace(n, t), ref_uc[t], ref_vc[t], delpc[t], pkc[t], gz[t], dt2)
    gd, sf = _grid(n, nz)
    d_uc, d_vc = _dev(uc), _dev(vc)
    PGradC(sf)(gd.rdxc, gd.rdyc, d_uc, d_vc, _dev(delpc), _dev(pkc), _dev(gz), dt2)
    _check(_host(d_uc), ref_uc)
    _check(_host(d_vc), ref_vc)


@pytest.mark.parametrize("n,nz,seed", SIZES)
def test_nh_p_grad(n, nz, seed):
    from oracle._util import Tile
    from oracle.a2b_ord4 import A2BScratch
    from oracle.dyn_core import nh_p_grad

    from fv3core_b200 import constants as C
    from fv3core_b200.stencils.nh_p_grad import NonHydrostaticPressureGradient

    st, rng = _state(n, nz, seed)
    shp = st["delp"].shape
    f = {
        "u": st["u"].copy(), "v": st["v"].copy(), "pp": 10.0 * rng.standard_normal(shp),
        "gz": cases.heights(st, nz) * 9.80665, "pk3": st["pk"] * (1 + 1e-5 * rng.standard_normal(shp)),
        "delp": st["delp"].copy(),
    }
    dt, ptop = 37.5, st["ptop"]
    ref = {k: np.array(v, copy=True) for k, v in f.items()}
    T = Tile(n, nz)
    for t in range(6):
        scr = {"wk": np.full((T.m, T.m, T.nk), np.nan), "wk1": np.full((T.m, T.m, T.nk), np.nan),
               "a2b_k1": A2BScratch((T.m, T.m, T.nk)), "a2b_kbuffer": A2BScratch((T.m, T.m, T.nk)),
               "a2b_kstandard": A2BScratch((T.m, T.m, T.nk))}
        nh_p_grad(T, cases.metric_namespace(n, t), scr, ref["u"][t], ref["v"][t], ref["pp"][t], ref["gz"][t],
                  ref["pk3"][t], ref["delp"][t], dt, ptop, C.KAPPA)
    gd, sf = _grid(n, nz)
    dev = {k: _dev(v) for k, v in f.items()}
    NonHydrostaticPressureGradient(sf, gd, 0)(dev["u"], dev["v"], dev["pp"], dev["gz"], dev["pk3"], dev["delp"], dt,
                                              ptop, C.KAPPA)
    box = (slice(None), slice(H, H + n + 1), slice(H, H + n + 1), slice(0, nz))
    for k in ("u", "v", "pp", "gz", "pk3"):
        _check(_host(dev[k]), ref[k], box)


@pytest.mark.parametrize("n,nz,seed", SIZES)
def test_pe_and_pk3_halo(n, nz, seed):
    from oracle._util import Tile
    from oracle.dyn_core import edge_pe, pk3_halo

    from fv3core_b200 import constants as C
    from fv3core_b200.stencils.pe_halo import EdgePe
    from fv3core_b200.stencils.pk3_halo import PK3Halo

    st, rng = _state(n, nz, seed)
    shp = st["delp"].shape
    pe, pk3 = rng.standard_normal(shp), rng.standard_normal(shp)
    delp = st["delp"]
    ptop = st["ptop"]
    ref_pe, ref_pk3 = pe.copy(), pk3.copy()
    T = Tile(n, nz)
    for t in range(6):
        edge_pe(T, ref_pe[t], delp[t], ptop)
        pk3_halo(T, ref_pk3[t], delp[t], ptop, C.KAPPA, np.full((T.m, T.m), np.nan))
    gd, sf = _grid(n, nz)
    d_pe, d_pk3 = _dev(pe), _dev(pk3)
    EdgePe(sf)(d_pe, _dev(delp), ptop)
    PK3Halo(sf)(d_pk3, _dev(delp), ptop, C.KAPPA)
    _check(_host(d_pe), ref_pe)
    _check(_host(d_pk3), ref_pk3)


@pytest.mark.parametrize("n,nz,seed", SIZES)
def test_ray_fast(n, nz, seed):
    from oracle._util import Tile
    from oracle.dyn_core import ray_fast

    from fv3core_b200.stencils.ray_fast import RayleighDamping

    st, rng = _state(n, nz, seed)
    shp = st["delp"].shape
    u, v, w = st["u"].copy(), st["v"].copy(), 0.1 * rng.standard_normal(shp)
    dp = _dp_ref(st, nz)
    pfull = np.asarray(st["pfull"])
    dt, ptop, rf_cutoff, tau = 37.5, st["ptop"], 3000.0, 10.0
    assert pfull[0] < rf_cutoff
    ref = [u.copy(), v.copy(), w.copy()]
    for t in range(6):
        ray_fast(Tile(n, nz), ref[0][t], ref[1][t], ref[2][t], dp, pfull, dt, ptop, rf_cutoff, tau)
    gd, sf = _grid(n, nz)
    dev = [_dev(a) for a in (u, v, w)]
    RayleighDamping(sf, rf_cutoff, tau, False)(*dev, dp, pfull, dt, ptop, st["ks"])
    for d, r in zip(dev, ref):
        _check(_host(d), r)


@pytest.mark.parametrize("n,nz,seed", SIZES)
def test_del2cubed_and_tempadjust(n, nz, seed):
    from oracle._util import Tile
    from oracle.dyn_core import del2cubed, pkz_tempadjust

    from fv3core_b200.stencils.del2cubed import HyperdiffusionDamping
    from fv3core_b200.stencils.temperature_adjust import ComputePkzTempadjust

    st, rng = _state(n, nz, seed)
    shp = st["delp"].shape
    g = cases.grid_for(n)
    heat = 1e3 * rng.standard_normal(shp)
    cd = 0.2 * g.da_min
    T = Tile(n, nz)
    ref_heat = heat.copy()
    for t in range(6):
        scr = {k: np.full((T.m, T.m, T.nk), np.nan) for k in ("q", "fx", "fy")}
        del2cubed(T, cases.metric_namespace(n, t), ref_heat[t], cd, 3, scr)
    gd, sf = _grid(n, nz)
    d_heat = _dev(heat)
    HyperdiffusionDamping(sf, gd, gd.rarea, 3)(d_heat, cd)
    box = (slice(None), slice(None), slice(None), slice(0, nz))
    _check(_host(d_heat), ref_heat, box)
    # temperature adjustment from the filtered heat source
    pt, pkz = st["pt"].copy(), st["pkz"].copy()
    ref_pt, ref_pkz = pt.copy(), pkz.copy()
    dtf = abs(37.5 * 0.002)
    for t in range(6):
        pkz_tempadjust(T, st["delp"][t], st["delz"][t], st["cappa"][t], ref_heat[t], ref_pt[t], ref_pkz[t], dtf, nz)
    d_pt, d_pkz = _dev(pt), _dev(pkz)
    ComputePkzTempadjust(sf, nz)(_dev(st["delp"]), _dev(st["delz"]), _dev(st["cappa"]), _dev(ref_heat), d_pt, d_pkz,
                                dtf)
    _check(_host(d_pt), ref_pt)
    _check(_host(d_pkz), ref_pkz)


@pytest.mark.parametrize("n,nz,seed", SIZES)
def test_halo_updates(n, nz, seed):
    from oracle.halo import HaloExchange

    from fv3core_b200.halo import DeviceCubedSphereCommunicator, spec_for

    rng = np.random.default_rng(seed)
    m = n + 2 * H + 1
    shp = (6, m, m, nz + 1)
    fields = {k: rng.standard_normal(shp) for k in ("c", "c2", "b", "u", "v", "uc", "vc", "su", "sv")}
    ref = {k: v.copy() for k, v in fields.items()}
    hx = HaloExchange(n, H)
    hx.scalar(ref["c"], nk=nz)
    hx.scalar(ref["c2"], n_halo=2, nk=nz + 1)
    hx.scalar_corner(ref["b"], nk=nz)
    hx.vector_d(ref["u"], ref["v"], nk=nz)
    hx.vector_c(ref["uc"], ref["vc"], nk=nz)
    hx.sync_vector_interfaces(ref["su"], ref["sv"], nk=nz)
    gd, sf = _grid(n, nz)
    gi = gd.grid_indexing
    comm = DeviceCubedSphereCommunicator(gi)
    dev = {k: _dev(v) for k, v in fields.items()}
    comm.get_scalar_halo_updater([spec_for(gi, ("x", "y", "z"))]).update([dev["c"]])
    comm.get_scalar_halo_updater([spec_for(gi, ("x", "y", "z_interface"), n_halo=2)]).update([dev["c2"]])
    comm.get_scalar_halo_updater([spec_for(gi, ("x_interface", "y_interface", "z"))]).update([dev["b"]])
    comm.get_vector_halo_updater([spec_for(gi, ("x", "y_interface", "z"))],
                                 [spec_for(gi, ("x_interface", "y", "z"))]).update([dev["u"]], [dev["v"]])
    comm.get_vector_halo_updater([spec_for(gi, ("x_interface", "y", "z"))],
                                 [spec_for(gi, ("x", "y_interface", "z"))]).update([dev["uc"]], [dev["vc"]])
    comm.synchronize_vector_interfaces(dev["su"], dev["sv"])
    for k in fields:
        assert np.array_equal(_host(dev[k]), ref[k]), k

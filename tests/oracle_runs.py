"""Run oracle stages over all six tiles of a case (shared by tests)."""
import numpy as np

import cases
from fv3core_b200 import constants as C
from oracle._util import Tile


def run_c_sw(case, n, nz):
    from oracle.c_sw import c_sw

    names = ["delp", "pt", "u", "v", "w", "uc", "vc", "ua", "va", "ut", "vt", "divgd", "omga"]
    out = {k: np.array(case[k], copy=True) for k in names}
    out["delpc"] = np.zeros_like(out["delp"])
    out["ptc"] = np.zeros_like(out["delp"])
    g = cases.grid_for(n)
    for t in range(6):
        ns = cases.metric_namespace(n, t)
        arrs = {k: out[k][t] for k in names}
        with np.errstate(all="ignore"):
            delpc, ptc = c_sw(Tile(n, nz), ns, g.fC[t], *[arrs[k] for k in names], case["dt2"])
        out["delpc"][t] = delpc
        out["ptc"][t] = ptc
    return out


def run_riem_solver_c(case, n, nz):
    from oracle.riem_solver_c import riem_solver_c

    out = {k: (np.array(v, copy=True) if isinstance(v, np.ndarray) else v) for k, v in case.items()}
    for t in range(6):
        riem_solver_c(
            out["dt2"], out["cappa"][t], out["ptop"], out["hs"][t], out["ws"][t], out["ptc"][t],
            out["q_con"][t], out["delpc"][t], out["gz"][t], out["pef"][t], out["w3"][t], out["p_fac"], n, nz,
        )
    return out


DSW_ARGS = ["delpc", "delp", "ptc", "pt", "u", "v", "w", "uc", "vc", "ua", "va", "divgd", "mfx", "mfy",
            "cx", "cy", "crx", "cry", "xfx", "yfx", "q_con", "zh", "heat_source", "diss_est"]


def run_d_sw(case, n, nz, states=None, overrides=None):
    """``overrides``: namelist values replacing those of cases.DSW_CONFIG."""
    from oracle.d_sw import DSWState, d_sw

    config = {**cases.DSW_CONFIG, **(overrides or {})}
    out = {k: np.array(case[k], copy=True) for k in DSW_ARGS}
    g = cases.grid_for(n)
    for t in range(6):
        T = Tile(n, nz)
        ns = cases.metric_namespace(n, t)
        st = DSWState(T, ns, config) if states is None else states[t]
        arrs = {k: out[k][t] for k in DSW_ARGS}
        with np.errstate(all="ignore"):
            d_sw(T, ns, g.f0[t], st, config, *[arrs[k] for k in DSW_ARGS], case["dt"])
    return out


def run_acoustics(case, n, nz):
    """The oracle's AcousticDynamics over all six tiles; returns the state
    and the driver's temporaries (prefixed ``tmp_``)."""
    from oracle.dyn_core import AcousticDynamics

    g = cases.grid_for(n)
    cfg = {**cases.ACOUSTIC_CONFIG, **cases.RIEMANN_CONFIG, "n_split": int(case["n_split"]),
           "dsw": cases.DSW_CONFIG}
    metrics = [cases.metric_namespace(n, t) for t in range(6)]
    ad = AcousticDynamics(g, metrics, cfg, case["ak"], case["bk"], case["pfull"], case["phis"], nz)
    st = {k: (np.array(v, copy=True) if isinstance(v, np.ndarray) else v) for k, v in case.items()}
    with np.errstate(all="ignore"):
        ad(st)
    out = {k: st[k] for k in cases.ACOUSTIC_STATE}
    for name, arr in ad.tmp.items():
        out["tmp_" + name] = arr
    return out


def run_tracer_advection(case, n, nz):
    """The oracle's TracerAdvection (hord_tr = 8) over all six tiles; returns
    the tracers and the in-place updated dp1, mfxd, mfyd, cxd, cyd."""
    from oracle.tracer import TracerAdvection

    g = cases.grid_for(n)
    metrics = [cases.metric_namespace(n, t) for t in range(6)]
    ntr = case["tracers"].shape[0]
    adv = TracerAdvection(g, metrics, nz, ntr, hord=8)
    out = {k: np.array(case[k], copy=True) for k in ("tracers", "dp1", "mfxd", "mfyd", "cxd", "cyd")}
    with np.errstate(all="ignore"):
        adv([out["tracers"][q] for q in range(ntr)], out["dp1"], out["mfxd"], out["mfyd"], out["cxd"],
            out["cyd"], case["mdt"])
    return out


def run_fv_step(case, n, nz):
    """The oracle's step preamble, post_remap and wrapup (fv_dynamics.py
    54-169) over all six tiles; returns the state after each phase
    (prefixes pre_, post_, wrap_)."""
    from oracle import fv_step as F
    from oracle.dyn_core import del2cubed
    from oracle.halo import HaloExchange

    g = cases.grid_for(n)
    t = Tile(n, nz)
    st = {k: np.array(v, copy=True) for k, v in case.items()}
    halo = HaloExchange(n, 3)
    out = {}
    with np.errstate(all="ignore"):
        for tt in range(6):
            F.fv_setup(t, *[st[k][tt] for k in ("qvapor", "qliquid", "qrain", "qsnow", "qice", "qgraupel", "q_con",
                                                "cvm", "pkz", "pt", "cappa", "delp", "delz", "dp1")])
            F.pt_adjust(t, st["pkz"][tt], st["dp1"][tt], st["q_con"][tt], st["pt"][tt])
        out.update({f"pre_{k}": st[k].copy() for k in ("q_con", "cvm", "pkz", "pt", "cappa", "dp1")})
        for tt in range(6):
            F.set_omega(t, st["delp"][tt], st["delz"][tt], st["w"][tt], st["omga"][tt])
        # nf_omega = 1: omega halo update, then one del-2 pass with 0.18 da_min
        halo.scalar(st["omga"], nk=nz)
        for tt in range(6):
            ns = cases.metric_namespace(n, tt)
            scr = {name: np.full((t.m, t.m, t.nk), np.nan) for name in ("q", "fx", "fy")}
            del2cubed(t, ns, st["omga"][tt], 0.18 * g.da_min, 1, scr)
        out["post_omga"] = st["omga"].copy()
        for tt in range(6):
            F.adjust_negative_tracers(t, *[st[k][tt] for k in cases.WATER_NAMES], st["pt"][tt], st["delp"][tt],
                                      st["delz"][tt], st["peln"][tt])
        halo.vector_d(st["u"], st["v"], nk=nz)
        for tt in range(6):
            F.cubed_to_latlon_ord4(t, st["u"][tt], st["v"][tt], g.dx[tt], g.dy[tt], g.a11[tt], g.a12[tt],
                                   g.a21[tt], g.a22[tt], st["ua"][tt], st["va"][tt])
        out.update({f"wrap_{k}": st[k].copy() for k in cases.WATER_NAMES + ("pt", "u", "v", "ua", "va")})
    return out


def run_remap(case, n, nz):
    """The oracle's LagrangianToEulerian (remapping.py:416-628, no saturation
    adjustment) tile by tile; returns the remapped fields over the full
    storage."""
    from oracle import remapping as R

    t = Tile(n, nz)
    st = {k: np.array(v, copy=True) for k, v in case.items() if isinstance(v, np.ndarray)}
    out = {}
    cfg = cases.remap_config(case)
    g = cases.grid_for(n)
    with np.errstate(all="ignore"):
        for tt in range(6):
            tracers = {k: st[k][tt] for k in cases.REMAP_TRACERS}
            fields = {k: st[k][tt] for k in cases.REMAP_STATE}
            sa = None
            if cfg["do_sat_adj"]:
                sa = {"cfg": cases.SAT_ADJUST_CONFIG, "area": g.area[tt], "hs": st["phis"][tt], "dp1": st["dp1"][tt],
                      "qcld": st["qcld"][tt], "pfull": case["pfull"], "mdt": case["mdt"]}
            R.lagrangian_to_eulerian(t, tracers, fields, case["ak"], case["bk"], case["ptop"], C.KAPPA, C.ZVIR,
                                     True, sat_adjust=sa,
                                     **{k: v for k, v in cfg.items() if k != "do_sat_adj"})
    for k in cases.REMAP_TRACERS + cases.REMAP_STATE + ("qcld",):
        out[k] = st[k]
    return out


def run_step(case, n, nz, steps=1):
    """The oracle's DynamicalCore.step_dynamics for one k_split step
    (fv_dynamics.py:430-557): compute_preamble, dp1 = delp, AcousticDynamics,
    TracerAdvection of the eight tracers, LagrangianToEulerian, post_remap
    (set_omega, omega halo, del-2 filter) and wrapup (neg_adj3, halo,
    cubed-to-latlon); DynamicalCore's temporaries (cappa, dp1, cvm, wsd,
    te_2d, te0_2d) start at zero and, like the acoustic driver's, persist
    from one of ``steps`` steps to the next.  Returns the full storages."""
    from oracle.dyn_core import AcousticDynamics
    from oracle.halo import HaloExchange
    from oracle.tracer import TracerAdvection

    g = cases.grid_for(n)
    t = Tile(n, nz)
    m = t.m
    metrics = [cases.metric_namespace(n, tt) for tt in range(6)]
    st = {k: (np.array(v, copy=True) if isinstance(v, np.ndarray) else v) for k, v in case.items()}
    for name in ("te_2d", "te0_2d", "wsd"):
        st[name] = np.zeros((6, m, m))
    for name in ("cappa", "dp1", "cvm"):
        st[name] = np.zeros((6, m, m, nz + 1))
    bdt = float(case["dt_atmos"])
    st.update(mdt=bdt, n_map=1, akap=C.KAPPA)
    cfg = {**cases.ACOUSTIC_CONFIG, **cases.RIEMANN_CONFIG, "n_split": int(case["n_split"]),
           "dsw": cases.DSW_CONFIG}
    ad = AcousticDynamics(g, metrics, cfg, case["ak"], case["bk"], case["pfull"], case["phis"], nz)
    adv = TracerAdvection(g, metrics, nz, len(cases.REMAP_TRACERS), hord=8)
    halo = HaloExchange(n, 3)
    with np.errstate(all="ignore"):
        for _ in range(steps):
            _oracle_step(st, case, n, nz, t, g, metrics, ad, adv, halo, bdt)
    return st


def _oracle_step(st, case, n, nz, t, g, metrics, ad, adv, halo, bdt):
    from oracle import fv_step as F
    from oracle import remapping as R
    from oracle.dyn_core import del2cubed

    for tt in range(6):
        F.fv_setup(t, *[st[k][tt] for k in ("qvapor", "qliquid", "qrain", "qsnow", "qice", "qgraupel", "q_con",
                                            "cvm", "pkz", "pt", "cappa", "delp", "delz", "dp1")])
        F.pt_adjust(t, st["pkz"][tt], st["dp1"][tt], st["q_con"][tt], st["pt"][tt])
    st["dp1"][..., :nz] = st["delp"][..., :nz]
    ad(st)
    adv([st[q] for q in cases.REMAP_TRACERS], st["dp1"], st["mfxd"], st["mfyd"], st["cxd"], st["cyd"], bdt)
    for tt in range(6):
        sa = None
        if bool(case.get("do_sat_adj", False)):
            sa = {"cfg": cases.SAT_ADJUST_CONFIG, "area": g.area[tt], "hs": st["phis"][tt], "dp1": st["dp1"][tt],
                  "qcld": st["qcld"][tt], "pfull": case["pfull"], "mdt": bdt}
        R.lagrangian_to_eulerian(t, {k: st[k][tt] for k in cases.REMAP_TRACERS},
                                 {k: st[k][tt] for k in cases.REMAP_STATE}, case["ak"], case["bk"], case["ptop"],
                                 C.KAPPA, C.ZVIR, True, sat_adjust=sa,
                                 **{k: v for k, v in cases.REMAP_CONFIG.items() if k != "do_sat_adj"})
    for tt in range(6):
        F.set_omega(t, st["delp"][tt], st["delz"][tt], st["w"][tt], st["omga"][tt])
    halo.scalar(st["omga"], nk=nz)
    for tt in range(6):
        scr = {name: np.full((t.m, t.m, t.nk), np.nan) for name in ("q", "fx", "fy")}
        del2cubed(t, metrics[tt], st["omga"][tt], 0.18 * g.da_min, 1, scr)
    for tt in range(6):
        F.adjust_negative_tracers(t, *[st[k][tt] for k in cases.WATER_NAMES], st["pt"][tt], st["delp"][tt],
                                  st["delz"][tt], st["peln"][tt])
    halo.vector_d(st["u"], st["v"], nk=nz)
    for tt in range(6):
        F.cubed_to_latlon_ord4(t, st["u"][tt], st["v"][tt], g.dx[tt], g.dy[tt], g.a11[tt], g.a12[tt],
                               g.a21[tt], g.a22[tt], st["ua"][tt], st["va"][tt])

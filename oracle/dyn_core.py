"""Acoustic substep driver (reference ``fv3core/stencils/dyn_core.py``,
``AcousticDynamics.__call__`` 479-761) and the remaining stencils it calls:
p_grad_c, nh_p_grad, ray_fast, pe/pk3 halos, del2cubed, temperature adjust.

All six tiles are advanced together; the cubed-sphere halo exchange is
restated in ``halo.py``.
"""
import math

import numpy as np

from fv3core_b200 import constants as C

from . import _math
from . import corners
from ._util import Tile, at, c3, put, region, sh
from .a2b_ord4 import A2BScratch, a2b_ord4
from .c_sw import c_sw
from .d_sw import DSWState, d_sw
from .halo import HaloExchange
from .riem_solver3 import riem_solver3
from .riem_solver_c import riem_solver_c
from .updatedz import UpdateDzDState, update_dz_c, update_dz_d

HUGE_R = 1.0e40


def p_grad_c(t: Tile, g, uc, vc, delpc, pkc, gz, dt2):
    """p_grad_c_stencil (dyn_core.py:101-145), nonhydrostatic."""
    s, e, js, je, nz = t.isc, t.iec, t.jsc, t.jec, t.nz
    wk = delpc
    zk = lambda a: sh(a, 0, 0, 1)  # noqa: E731
    un = uc + dt2 * c3(g.rdxc) / (sh(wk, -1, 0) + wk) * (
        (sh(gz, -1, 0, 1) - gz) * (zk(pkc) - sh(pkc, -1, 0)) + (sh(gz, -1, 0) - zk(gz)) * (sh(pkc, -1, 0, 1) - pkc)
    )
    vn = vc + dt2 * c3(g.rdyc) / (sh(wk, 0, -1) + wk) * (
        (sh(gz, 0, -1, 1) - gz) * (zk(pkc) - sh(pkc, 0, -1)) + (sh(gz, 0, -1) - zk(gz)) * (sh(pkc, 0, -1, 1) - pkc)
    )
    put(uc, un, s, e + 2, js, je + 2, 0, nz)
    put(vc, vn, s, e + 2, js, je + 2, 0, nz)


def nh_p_grad(t: Tile, g, scr, u, v, pp, gz, pk3, delp, dt, ptop, akap):
    """NonHydrostaticPressureGradient.__call__ (nh_p_grad.py:147-206)."""
    s, e, js, je, nz, nk = t.isc, t.iec, t.jsc, t.jec, t.nz, t.nk
    ptk = ptop ** akap
    wk1 = scr["wk1"]
    a2b_ord4(t, g, pp, wk1, 1, nk, scr["a2b_k1"], replace=True)
    a2b_ord4(t, g, pk3, wk1, 1, nk, scr["a2b_k1"], replace=True)
    a2b_ord4(t, g, gz, wk1, 0, nk, scr["a2b_kbuffer"], replace=True)
    a2b_ord4(t, g, delp, wk1, 0, nz, scr["a2b_kstandard"], replace=False)
    # set_k0_and_calc_wk (nh_p_grad.py:11-18) on [is, ie+1] x [js, je+1]
    pp[s : e + 2, js : je + 2, 0] = 0.0
    pk3[s : e + 2, js : je + 2, 0] = ptk
    wk = scr["wk"]
    put(wk, sh(pk3, 0, 0, 1) - pk3, s, e + 2, js, je + 2, 0, nz)
    zk = lambda a: sh(a, 0, 0, 1)  # noqa: E731
    # calc_u (nh_p_grad.py:21-51) on [is, ie] x [js, je+1]
    du = dt / (wk + sh(wk, 1, 0)) * (
        (zk(gz) - sh(gz, 1, 0)) * (sh(pk3, 1, 0, 1) - pk3) + (gz - sh(gz, 1, 0, 1)) * (zk(pk3) - sh(pk3, 1, 0))
    )
    un = (u + du + dt / (wk1 + sh(wk1, 1, 0)) * (
        (zk(gz) - sh(gz, 1, 0)) * (sh(pp, 1, 0, 1) - pp) + (gz - sh(gz, 1, 0, 1)) * (zk(pp) - sh(pp, 1, 0))
    )) * c3(g.rdx)
    put(u, un, s, e + 1, js, je + 2, 0, nz)
    dv = dt / (wk + sh(wk, 0, 1)) * (
        (zk(gz) - sh(gz, 0, 1)) * (sh(pk3, 0, 1, 1) - pk3) + (gz - sh(gz, 0, 1, 1)) * (zk(pk3) - sh(pk3, 0, 1))
    )
    vn = (v + dv + dt / (wk1 + sh(wk1, 0, 1)) * (
        (zk(gz) - sh(gz, 0, 1)) * (sh(pp, 0, 1, 1) - pp) + (gz - sh(gz, 0, 1, 1)) * (zk(pp) - sh(pp, 0, 1))
    )) * c3(g.rdy)
    put(v, vn, s, e + 2, js, je + 1, 0, nz)


def ray_fast(t: Tile, u, v, w, dp, pfull, dt, ptop, rf_cutoff, tau, hydrostatic=False):
    """RayleighDamping.__call__ (ray_fast.py:169-192) and
    ray_fast_wind_compute (48-128) on X_INTERFACE x Y_INTERFACE compute."""
    s, e, js, je, nz = t.isc, t.iec, t.jsc, t.jec, t.nz
    nudge = rf_cutoff + min(100.0, 10.0 * ptop)
    pf = np.asarray(pfull)[:nz]
    dpk = np.asarray(dp)[:nz]
    tau0 = tau * C.SDAY
    with np.errstate(all="ignore"):
        rfv = dt / tau0 * _math.host_sin(0.5 * C.PI * _math.host_log(rf_cutoff / pf) / _math.host_log(
            rf_cutoff / ptop)) ** 2
        rf = np.where(pf < rf_cutoff, 1.0 / (1.0 + rfv), np.nan)
    dm = np.full(nz, np.nan)
    if pf[0] < nudge:
        dm[0] = dpk[0]
    for k in range(1, nz):
        dm[k] = dm[k - 1]
        if pf[k] < nudge:
            dm[k] += dpk[k]
    for k in range(nz - 2, -1, -1):
        if pf[k] < nudge:
            dm[k] = dm[k + 1]

    def damp_component(q, i1, j1):
        I, J = slice(s, i1), slice(js, j1)
        col = q[I, J, :nz]
        dmdir = np.full(col.shape, np.nan)
        dmk = np.broadcast_to(dm, col.shape).copy()
        if pf[0] < rf_cutoff:
            dmdir[:, :, 0] = (1.0 - rf[0]) * dpk[0] * col[:, :, 0]
            col[:, :, 0] *= rf[0]
        else:
            dmk[:, :, 0] = 0
        for k in range(1, nz):
            dmdir[:, :, k] = dmdir[:, :, k - 1]
            if pf[k] < rf_cutoff:
                dmdir[:, :, k] += (1.0 - rf[k]) * dpk[k] * col[:, :, k]
                col[:, :, k] *= rf[k]
        for k in range(nz - 2, -1, -1):
            if pf[k] < rf_cutoff:
                dmdir[:, :, k] = dmdir[:, :, k + 1]
        for k in range(nz):
            if pf[k] < nudge:
                col[:, :, k] += dmdir[:, :, k] / dmk[:, :, k]
        q[I, J, :nz] = col

    with np.errstate(all="ignore"):
        damp_component(u, e + 1, je + 2)
        damp_component(v, e + 2, je + 1)
    if not hydrostatic:
        for k in range(nz):
            if pf[k] < rf_cutoff:
                w[s : e + 1, js : je + 1, k] *= rf[k]


def edge_pe(t: Tile, pe, delp, ptop):
    """edge_pe (pe_halo.py:6-33): pe on the one-cell ring around the compute
    domain by summing delp."""
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    m = (
        region(t, s - 1, s, js, je + 1) | region(t, e + 1, e + 2, js, je + 1)
        | region(t, s - 1, e + 2, js - 1, js) | region(t, s - 1, e + 2, je + 1, je + 2)
    )[:, :, 0]
    pe[:, :, 0] = np.where(m, ptop, pe[:, :, 0])
    for k in range(1, t.nk):
        pe[:, :, k] = np.where(m, pe[:, :, k - 1] + delp[:, :, k - 1], pe[:, :, k])


def pk3_halo(t: Tile, pk3, delp, ptop, akap, pe_tmp):
    """PK3Halo.__call__ (pk3_halo.py:36-68): pk3 on the two-cell ring; pe_tmp
    is the instance's 2-D storage."""
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    m = (
        region(t, s - 2, s, js, je + 1) | region(t, e + 1, e + 3, js, je + 1)
        | region(t, s - 2, e + 3, js - 2, js) | region(t, s - 2, e + 3, je + 1, je + 3)
    )[:, :, 0]
    pe_tmp[:] = np.where(m, ptop, pe_tmp)
    for k in range(1, t.nk):
        pe_tmp[:] = np.where(m, pe_tmp + delp[:, :, k - 1], pe_tmp)
        pk3[:, :, k] = np.where(m, _math.power(pe_tmp, akap), pk3[:, :, k])


def del2cubed(t: Tile, g, qdel, cd, nmax, scr):
    """HyperdiffusionDamping.__call__ (del2cubed.py:152-181)."""
    s, e, js, je, nz = t.isc, t.iec, t.jsc, t.jec, t.nz
    full = t.m - 1
    ntimes = min(3, nmax)
    q = scr["q"]
    fx, fy = scr["fx"], scr["fy"]
    third = 1.0 / 3.0
    for n in range(ntimes):
        nt = ntimes - (n + 1)
        # corner_fill (del2cubed.py:41-75)
        qi = qdel
        v = qi.copy()
        pts = [
            ((s, js), (0, 0), (-1, 0), (0, -1)), ((s - 1, js), (1, 0), (0, 0), (1, -1)),
            ((s, js - 1), (0, 1), (-1, 1), (0, 0)), ((e, js), (0, 0), (1, 0), (0, -1)),
            ((e + 1, js), (-1, 0), (0, 0), (-1, -1)), ((e, js - 1), (0, 1), (1, 1), (0, 0)),
            ((e, je), (0, 0), (1, 0), (0, 1)), ((e + 1, je), (-1, 0), (0, 0), (-1, 1)),
            ((e, je + 1), (0, -1), (1, -1), (0, 0)), ((s, je), (0, 0), (-1, 0), (0, 1)),
            ((s - 1, je), (1, 0), (0, 0), (1, 1)), ((s, je + 1), (0, -1), (-1, -1), (0, 0)),
        ]
        for (i, j), a, b, c in pts:
            v[i, j, :nz] = (qi[i + a[0], j + a[1], :nz] + qi[i + b[0], j + b[1], :nz] + qi[i + c[0], j + c[1], :nz]) * third
        put(q, v, 0, full, 0, full, 0, nz)
        if nt > 0:
            put(q, corners.copy_corners(t, q, "x"), 0, full, 0, full, 0, t.nk)
        put(fx, c3(g.del6_v) * (sh(q, -1, 0) - q), s - nt, e + 2 + nt, js - nt, je + 1 + nt, 0, nz)
        if nt > 0:
            put(q, corners.copy_corners(t, q, "y"), 0, full, 0, full, 0, t.nk)
        put(fy, c3(g.del6_u) * (sh(q, 0, -1) - q), s - nt, e + 1 + nt, js - nt, je + 2 + nt, 0, nz)
        put(qdel, q, 0, full, 0, full, 0, nz)
        upd = qdel + cd * c3(g.rarea) * (fx - sh(fx, 1, 0) + fy - sh(fy, 0, 1))
        put(qdel, upd, s - nt, e + 1 + nt, js - nt, je + 1 + nt, 0, nz)


def sign(a, b):
    """basic_operations.sign (basic_operations.py:34-41): |a| with the sign
    of b, negative when b == 0."""
    asignb = np.abs(a)
    return np.where(b > 0, asignb, -asignb)


def pkz_tempadjust(t: Tile, delp, delz, cappa, heat_source, pt, pkz, dtf, nk_heat):
    """compute_pkz_tempadjust (temperature_adjust.py:8-44) on the compute
    domain, levels [0, nk_heat)."""
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    B = (slice(s, e + 1), slice(js, je + 1), slice(0, nk_heat))
    dp, dz, cp, hs = delp[B], delz[B], cappa[B], heat_source[B]
    p = pkz[B]
    # the reference first writes exp(cp/(1-cp) log(...)) and then overwrites it
    p[...] = _math.power(C.RDG * dp / dz * pt[B], cp / (1.0 - cp))
    dtmp = hs / (C.CV_AIR * dp)
    fac = np.array([0.1 if k == 0 else (0.5 if k == 1 else 1.0) for k in range(nk_heat)])[None, None, :]
    deltmin = sign(np.minimum(dtf * fac, np.abs(dtmp)), dtmp)
    pt[B] = pt[B] + deltmin / p


def dp_ref_compute(ak, bk, nz):
    """dp_ref_compute (dyn_core.py:66-77), the K part."""
    dp = np.full(nz + 1, np.nan)
    dp[:nz] = ak[1:] - ak[:-1] + (bk[1:] - bk[:-1]) * 1.0e5
    return dp


def nk_heat_dissipation(cfg_dsw, npz):
    """get_nk_heat_dissipation (dyn_core.py:148-163)."""
    if cfg_dsw.get("convert_ke", False) or cfg_dsw["vtdm4"] > 1.0e-4:
        return npz
    if cfg_dsw["d2_bg_k1"] < 1.0e-3:
        return 0
    if cfg_dsw["d2_bg_k2"] < 1.0e-3:
        return 1
    return 2


class AcousticDynamics:
    """AcousticDynamics (dyn_core.py:210-761) for all six tiles.

    ``grid`` is a CubedSphereGrid; ``metrics`` a list of six per-tile metric
    namespaces; ``cfg`` a dict with the acoustic namelist ("n_split",
    "k_split", "tau", "rf_cutoff", "rf_fast", "delt_max", "p_fac",
    "breed_vortex_inline", "use_old_omega") and ``cfg["dsw"]`` the D-grid
    namelist.
    """

    def __init__(self, grid, metrics, cfg, ak, bk, pfull, phis, nz):
        self.grid = grid
        self.g = metrics
        self.cfg = cfg
        n = grid.n
        self.t = Tile(n, nz)
        t = self.t
        self.nz = nz
        self.halo = HaloExchange(n, grid.halo)
        shp = (6, t.m, t.m, t.nk)
        self.tmp = {name: np.zeros(shp) for name in ("ut", "vt", "gz", "zh", "pem", "pkc", "pk3", "heat_source", "divgd")}
        self.tmp["ws3"] = np.zeros((6, t.m, t.m))
        for name in ("crx", "xfx", "cry", "yfx"):
            self.tmp[name] = np.zeros(shp)
        self.tmp["gz"][:] = HUGE_R
        self.tmp["pk3"][:] = HUGE_R
        self.dp_ref = dp_ref_compute(np.asarray(ak), np.asarray(bk), nz)
        # dp_ref_compute multiplies by the reciprocal (dyn_core.py:79)
        self.zs = phis * (1.0 / C.GRAV)
        self.pfull = np.asarray(pfull)
        dcfg = cfg["dsw"]
        self.dsw_states = [DSWState(t, metrics[tt], dcfg) for tt in range(6)]
        self.dzd_states = [UpdateDzDState(t, self.dp_ref, self.dsw_states[tt].col) for tt in range(6)]
        self.nh_scr = [
            {"wk": np.full((t.m, t.m, t.nk), np.nan), "wk1": np.full((t.m, t.m, t.nk), np.nan),
             "a2b_k1": A2BScratch((t.m, t.m, t.nk)), "a2b_kbuffer": A2BScratch((t.m, t.m, t.nk)),
             "a2b_kstandard": A2BScratch((t.m, t.m, t.nk))}
            for _ in range(6)
        ]
        self.pe_tmp = [np.full((t.m, t.m), np.nan) for _ in range(6)]
        self.del2_scr = [{"q": np.full((t.m, t.m, t.nk), np.nan), "fx": np.full((t.m, t.m, t.nk), np.nan),
                          "fy": np.full((t.m, t.m, t.nk), np.nan)} for _ in range(6)]
        self.nk_heat = nk_heat_dissipation(dcfg, nz)
        self.do_del2cubed = self.nk_heat != 0 and dcfg["d_con"] > 1.0e-5

    def __call__(self, st):
        """``st`` maps the reference's state names to six-tile arrays and the
        scalars mdt, n_map, ptop, ks, akap."""
        t, nz = self.t, self.nz
        cfg = self.cfg
        dcfg = cfg["dsw"]
        H = self.halo
        n_split = cfg["n_split"]
        end_step = st["n_map"] == cfg["k_split"]
        akap = C.KAPPA
        dt = st["mdt"] / n_split
        dt2 = 0.5 * dt
        T = self.tmp
        H.scalar(st["q_con"], st["cappa"], nk=nz)
        H.scalar(st["delp"], st["pt"], nk=nz)
        H.vector_d(st["u"], st["v"], nk=nz)
        # zero_data (dyn_core.py:47-63)
        full = t.m - 1
        for name in ("mfxd", "mfyd", "cxd", "cyd"):
            st[name][:, :full, :full, :nz] = 0.0
        if st["n_map"] == 1:
            st["diss_estd"][:, t.isc : t.iec + 1, t.jsc : t.jec + 1, :nz] = 0.0
        for it in range(n_split):
            remap_step = bool(cfg.get("breed_vortex_inline", False)) or it == n_split - 1
            H.scalar(st["w"], nk=nz)
            if it == 0:
                # set_gz (dyn_core.py:80-85) on the compute domain
                I, J = slice(t.isc, t.iec + 1), slice(t.jsc, t.jec + 1)
                T["gz"][:, I, J, nz] = self.zs[:, I, J]
                for k in range(nz - 1, -1, -1):
                    T["gz"][:, I, J, k] = T["gz"][:, I, J, k + 1] - st["delz"][:, I, J, k]
                H.scalar(T["gz"], nk=nz + 1)
            delpc = np.zeros_like(st["delp"])
            ptc = np.zeros_like(st["delp"])
            for tt in range(6):
                delpc[tt], ptc[tt] = c_sw(
                    t, self.g[tt], self.grid.fC[tt], st["delp"][tt], st["pt"][tt], st["u"][tt], st["v"][tt],
                    st["w"][tt], st["uc"][tt], st["vc"][tt], st["ua"][tt], st["va"][tt], T["ut"][tt], T["vt"][tt],
                    T["divgd"][tt], st["omga"][tt], dt2, dcfg["nord"],
                )
            if dcfg["nord"] > 0:
                H.scalar_corner(T["divgd"], nk=nz)
            full_b = (slice(None), slice(0, full), slice(0, full), slice(0, t.nk))
            if it == 0:
                T["zh"][full_b] = T["gz"][full_b]
            else:
                T["gz"][full_b] = T["zh"][full_b]
            for tt in range(6):
                update_dz_c(t, self.g[tt], self.dp_ref, self.zs[tt], T["ut"][tt], T["vt"][tt], T["gz"][tt],
                            T["ws3"][tt], dt2)
                riem_solver_c(dt2, st["cappa"][tt], st["ptop"], st["phis"][tt], T["ws3"][tt], ptc[tt],
                              st["q_con"][tt], delpc[tt], T["gz"][tt], T["pkc"][tt], st["omga"][tt], cfg["p_fac"],
                              t.n, nz)
                p_grad_c(t, self.g[tt], st["uc"][tt], st["vc"][tt], delpc[tt], T["pkc"][tt], T["gz"][tt], dt2)
            H.vector_c(st["uc"], st["vc"], nk=nz)
            for tt in range(6):
                d_sw(t, self.g[tt], self.grid.f0[tt], self.dsw_states[tt], dcfg, T["vt"][tt], st["delp"][tt],
                     ptc[tt], st["pt"][tt], st["u"][tt], st["v"][tt], st["w"][tt], st["uc"][tt], st["vc"][tt],
                     st["ua"][tt], st["va"][tt], T["divgd"][tt], st["mfxd"][tt], st["mfyd"][tt], st["cxd"][tt],
                     st["cyd"][tt], T["crx"][tt], T["cry"][tt], T["xfx"][tt], T["yfx"][tt], st["q_con"][tt],
                     T["zh"][tt], T["heat_source"][tt], st["diss_estd"][tt], dt)
            H.scalar(st["delp"], st["pt"], st["q_con"], nk=nz)
            for tt in range(6):
                update_dz_d(t, self.g[tt], self.dzd_states[tt], dcfg["hord_tm"], self.zs[tt], T["zh"][tt],
                            T["crx"][tt], T["cry"][tt], T["xfx"][tt], T["yfx"][tt], st["wsd"][tt], dt)
                riem_solver3(remap_step, dt, st["cappa"][tt], st["ptop"], self.zs[tt], st["wsd"][tt],
                             st["delz"][tt], st["q_con"][tt], st["delp"][tt], st["pt"][tt], T["zh"][tt],
                             st["pe"][tt], T["pkc"][tt], T["pk3"][tt], st["pk"][tt], st["peln"][tt], st["w"][tt],
                             cfg["p_fac"], t.n, nz)
            H.scalar(T["zh"], nk=nz + 1)
            H.scalar(T["pkc"], n_halo=2, nk=nz + 1)
            for tt in range(6):
                if remap_step:
                    edge_pe(t, st["pe"][tt], st["delp"][tt], st["ptop"])
                pk3_halo(t, T["pk3"][tt], st["delp"][tt], st["ptop"], akap, self.pe_tmp[tt])
            # compute_geopotential (dyn_core.py:96-98) with halo 2
            B = (slice(None), slice(t.isc - 2, t.iec + 3), slice(t.jsc - 2, t.jec + 3), slice(0, t.nk))
            T["gz"][B] = T["zh"][B] * C.GRAV
            for tt in range(6):
                nh_p_grad(t, self.g[tt], self.nh_scr[tt], st["u"][tt], st["v"][tt], T["pkc"][tt], T["gz"][tt],
                          T["pk3"][tt], st["delp"][tt], dt, st["ptop"], akap)
                if cfg["rf_fast"]:
                    ray_fast(t, st["u"][tt], st["v"][tt], st["w"][tt], self.dp_ref, self.pfull, dt, st["ptop"],
                             cfg["rf_cutoff"], cfg["tau"])
            if it != n_split - 1:
                H.vector_d(st["u"], st["v"], nk=nz)
            else:
                H.sync_vector_interfaces(st["u"], st["v"], nk=nz)
        if self.do_del2cubed:
            H.scalar(T["heat_source"], nk=nz)
            cd = C.CNST_0P20 * self.g[0].da_min
            for tt in range(6):
                del2cubed(t, self.g[tt], T["heat_source"][tt], cd, min(3, dcfg["nord"] + 1), self.del2_scr[tt])
                delt_time_factor = abs(dt * cfg["delt_max"])
                pkz_tempadjust(t, st["delp"][tt], st["delz"][tt], st["cappa"][tt], T["heat_source"][tt],
                               st["pt"][tt], st["pkz"][tt], delt_time_factor, self.nk_heat)

"""D-grid shallow water (reference ``fv3core/stencils/d_sw.py``) with
divergence damping (``fv3core/stencils/divergence_damping.py``).

``DSWState`` holds the storages the reference's DGridShallowWaterLagrangianDynamics
instance owns and reuses between calls (d_sw.py:636-660, fvtp2d and
delnflux scratch), so that halo points the reference never rewrites keep
the same contents here.
"""
import numpy as np

from . import corners
from ._util import Tile, at, c3, put, region, sh
from .a2b_ord4 import A2BScratch, a2b_ord4
from .fvtp2d import DelnScratch, FvTp2dScratch, calc_damp, copy_corners_xy, delnflux_nosg, fvtp2d
from .fxadv import fxadv
from .ppm import advect_along

DCON_THRESHOLD = 1e-5


def column_namelist(cfg, npz):
    """get_column_namelist (d_sw.py:512-563)."""
    n = npz + 1
    col = {name: np.zeros(n) for name in ("ke_bg", "d_con", "nord", "nord_v", "nord_w", "nord_t", "damp_vt", "damp_w", "damp_t", "d2_divg")}
    col["ke_bg"][:] = cfg["ke_bg"]
    col["d_con"][:] = cfg["d_con"]
    col["nord"][:] = cfg["nord"]
    col["d2_divg"][:] = min(0.2, cfg["d2_bg"])
    col["nord_v"][:] = min(2, col["nord"][0])
    col["nord_w"][:] = col["nord_v"][0]
    col["nord_t"][:] = col["nord_v"][0]
    col["damp_vt"][:] = cfg["vtdm4"] if cfg["do_vort_damp"] else 0.0
    col["damp_w"][:] = col["damp_vt"][0]
    col["damp_t"][:] = col["damp_vt"][0]

    def set_low(k):
        for name in ("nord", "nord_w", "d_con"):
            col[name][k] = 0
        col["damp_w"][k] = col["d2_divg"][k]

    def vort_opt(k):
        if cfg["do_vort_damp"]:
            col["nord_v"][k] = 0
            col["damp_vt"][k] = 0.5 * col["d2_divg"][k]

    if npz == 1 or cfg["n_sponge"] < 0:
        col["d2_divg"][0] = cfg["d2_bg"]
    else:
        col["d2_divg"][0] = max(0.01, cfg["d2_bg"], cfg["d2_bg_k1"])
        set_low(0)
        vort_opt(0)
        if cfg["d2_bg_k2"] > 0.01:
            col["d2_divg"][1] = max(cfg["d2_bg"], cfg["d2_bg_k2"])
            set_low(1)
            vort_opt(1)
        if cfg["d2_bg_k2"] > 0.05:
            col["d2_divg"][2] = max(cfg["d2_bg"], 0.2 * cfg["d2_bg_k2"])
            set_low(2)
    return col


class DSWState:
    def __init__(self, t: Tile, g, cfg):
        shp = (t.m, t.m, t.nk)
        nan = lambda: np.full(shp, np.nan)  # noqa: E731
        for name in (
            "tmp_heat_s", "vort_x_delta", "vort_y_delta", "tmp_ke", "tmp_vort", "uc_contra", "vc_contra",
            "tmp_ut", "tmp_vt", "tmp_fx", "tmp_fy", "tmp_gx", "tmp_gy", "tmp_dw", "tmp_wk", "tmp_fx2", "tmp_fy2",
            "advected_u", "advected_v", "ub_contra", "vb_contra", "y_temporary",
        ):
            setattr(self, name, nan())
        self.col = column_namelist(cfg, t.nz)
        self.fvtp_dp, self.fvtp_dp_t, self.fvtp_tm, self.fvtp_vt = (FvTp2dScratch(shp) for _ in range(4))
        d2_shape = (t.m - 1, t.m - 1, t.nz)
        self.deln_dp, self.deln_dp_t, self.deln_tm = (DelnScratch(shp) for _ in range(3))
        self.a2b = A2BScratch(shp)
        self.dd_corner_tmp = nan()
        c = self.col
        self.damp_vt = calc_damp(c["nord_v"], c["damp_vt"], g.da_min_c, t.nz)
        self.damp_w = calc_damp(c["nord_w"], c["damp_w"], g.da_min_c, t.nz)
        # divergence damping set-up (divergence_damping.py:164-327)
        nord_col = c["nord"]
        self.nonzero_nord_k = 0
        self.nonzero_nord = int(cfg["nord"])
        for k in range(len(nord_col)):
            if nord_col[k] > 0:
                self.nonzero_nord_k = k
                self.nonzero_nord = int(nord_col[k])
                break
        self.dd8 = (g.da_min_c * cfg["d4_bg"]) ** (self.nonzero_nord + 1)


def _kfield(col, nz):
    return np.asarray(col)[None, None, :nz]


def _fill_corners_bgrid(t: Tile, q, direction, k0, k1):
    """fill_corners_bgrid_{x,y}_defn (corners.py:598-722) in place on
    levels [k0, k1); q is read before any corner is written (the reference
    aliases q_in and q_out, but no rule reads a filled corner)."""
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    if direction == "x":
        rules = [
            ((s - 1, js - 1), (0, 2)), ((e + 2, js - 1), (0, 2)),
            ((s - 1, js - 2), (-1, 3)), ((e + 3, js - 1), (-1, 3)),
            ((s - 1, js - 3), (-2, 4)), ((e + 4, js - 1), (-2, 4)),
            ((s - 2, js - 1), (1, 3)), ((e + 2, js - 2), (1, 3)),
            ((s - 2, js - 2), (0, 4)), ((e + 3, js - 2), (0, 4)),
            ((s - 2, js - 3), (-1, 5)), ((e + 4, js - 2), (-1, 5)),
            ((s - 3, js - 1), (2, 4)), ((e + 2, js - 3), (2, 4)),
            ((s - 3, js - 2), (1, 5)), ((e + 3, js - 3), (1, 5)),
            ((s - 3, js - 3), (0, 6)), ((e + 4, js - 3), (0, 6)),
            ((s - 1, je + 2), (0, -2)), ((e + 2, je + 2), (0, -2)),
            ((s - 1, je + 3), (-1, -3)), ((e + 3, je + 2), (-1, -3)),
            ((s - 1, je + 4), (-2, -4)), ((e + 4, je + 2), (-2, -4)),
            ((s - 2, je + 2), (1, -3)), ((e + 2, je + 3), (1, -3)),
            ((s - 2, je + 3), (0, -4)), ((e + 3, je + 3), (0, -4)),
            ((s - 2, je + 4), (-1, -5)), ((e + 4, je + 3), (-1, -5)),
            ((s - 3, je + 2), (2, -4)), ((e + 2, je + 4), (2, -4)),
            ((s - 3, je + 3), (1, -5)), ((e + 3, je + 4), (1, -5)),
            ((s - 3, je + 4), (0, -6)), ((e + 4, je + 4), (0, -6)),
        ]
    else:
        rules = [
            ((s - 1, js - 1), (2, 0)), ((s - 1, je + 2), (2, 0)),
            ((s - 1, js - 2), (3, 1)), ((s - 2, je + 2), (3, 1)),
            ((s - 1, js - 3), (4, 2)), ((s - 3, je + 2), (4, 2)),
            ((s - 2, js - 1), (3, -1)), ((s - 1, je + 3), (3, -1)),
            ((s - 2, js - 2), (4, 0)), ((s - 2, je + 3), (4, 0)),
            ((s - 2, js - 3), (5, 1)), ((s - 3, je + 3), (5, 1)),
            ((s - 3, js - 1), (4, -2)), ((s - 1, je + 4), (4, -2)),
            ((s - 3, js - 2), (5, -1)), ((s - 2, je + 4), (5, -1)),
            ((s - 3, js - 3), (6, 0)), ((s - 3, je + 4), (6, 0)),
            ((e + 2, js - 1), (-2, 0)), ((e + 2, je + 2), (-2, 0)),
            ((e + 2, js - 2), (-3, 1)), ((e + 3, je + 2), (-3, 1)),
            ((e + 2, js - 3), (-4, 2)), ((e + 4, je + 2), (-4, 2)),
            ((e + 3, js - 1), (-3, -1)), ((e + 2, je + 3), (-3, -1)),
            ((e + 3, js - 2), (-4, 0)), ((e + 3, je + 3), (-4, 0)),
            ((e + 3, js - 3), (-5, 1)), ((e + 4, je + 3), (-5, 1)),
            ((e + 4, js - 1), (-4, -2)), ((e + 2, je + 4), (-4, -2)),
            ((e + 4, js - 2), (-5, -1)), ((e + 3, je + 4), (-5, -1)),
            ((e + 4, js - 3), (-6, 0)), ((e + 4, je + 4), (-6, 0)),
        ]
    for (i, j), (di, dj) in rules:
        q[i, j, k0:k1] = q[i + di, j + dj, k0:k1]


def _fill_corners_dgrid(t: Tile, x, y, mysign, k0, k1):
    """fill_corners_dgrid_defn (corners.py:993-1150) in place, statement by
    statement (x_in aliases x_out and y_in aliases y_out in the reference)."""
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    m = mysign
    # (target field, (i, j), source field, (di, dj), multiplier)
    R = []
    # sw corner
    sw = [((s - 1, js - 1), (0, 1), (1, 0)), ((s - 1, js - 2), (-1, 2), (2, 1)), ((s - 1, js - 3), (-2, 3), (3, 2)),
          ((s - 2, js - 1), (1, 2), (2, -1)), ((s - 2, js - 2), (0, 3), (3, 0)), ((s - 2, js - 3), (-1, 4), (4, 1)),
          ((s - 3, js - 1), (2, 3), (3, -2)), ((s - 3, js - 2), (1, 4), (4, -1)), ((s - 3, js - 3), (0, 5), (5, 0))]
    for (i, j), ox, oy in sw:
        R.append(("x", (i, j), "y", ox, m))
        R.append(("y", (i, j), "x", oy, m))
    # ne corner
    ne = [((e + 1, je + 2), "x", (1, -2)), ((e + 2, je + 1), "y", (-2, 1)), ((e + 1, je + 3), "x", (2, -3)),
          ((e + 2, je + 2), "y", (-3, 0)), ((e + 1, je + 4), "x", (3, -4)), ((e + 2, je + 3), "y", (-4, -1)),
          ((e + 2, je + 2), "x", (0, -3)), ((e + 3, je + 1), "y", (-3, 2)), ((e + 2, je + 3), "x", (1, -4)),
          ((e + 3, je + 2), "y", (-4, 1)), ((e + 2, je + 4), "x", (2, -5)), ((e + 3, je + 3), "y", (-5, 0)),
          ((e + 3, je + 2), "x", (-1, -4)), ((e + 4, je + 1), "y", (-4, 3)), ((e + 3, je + 3), "x", (0, -5)),
          ((e + 4, je + 2), "y", (-5, 2)), ((e + 3, je + 4), "x", (1, -6)), ((e + 4, je + 3), "y", (-6, 1))]
    for (i, j), f, o in ne:
        R.append((f, (i, j), "y" if f == "x" else "x", o, m))
    # nw corner (no sign)
    nw = [((s - 1, je + 2), "x", (0, -2)), ((s - 1, je + 1), "y", (1, 1)), ((s - 1, je + 3), "x", (-1, -3)),
          ((s - 1, je + 2), "y", (2, 0)), ((s - 1, je + 4), "x", (-2, -4)), ((s - 1, je + 3), "y", (3, -1)),
          ((s - 2, je + 2), "x", (1, -3)), ((s - 2, je + 1), "y", (2, 2)), ((s - 2, je + 3), "x", (0, -4)),
          ((s - 2, je + 2), "y", (3, 1)), ((s - 2, je + 4), "x", (-1, -5)), ((s - 2, je + 3), "y", (4, 0)),
          ((s - 3, je + 2), "x", (2, -4)), ((s - 3, je + 1), "y", (3, 3)), ((s - 3, je + 3), "x", (1, -5)),
          ((s - 3, je + 2), "y", (4, 2)), ((s - 3, je + 4), "x", (0, -6)), ((s - 3, je + 3), "y", (5, 1))]
    for (i, j), f, o in nw:
        R.append((f, (i, j), "y" if f == "x" else "x", o, 1.0))
    se = [((e + 1, js - 1), "x", (1, 1)), ((e + 2, js - 1), "y", (-2, 0)), ((e + 1, js - 2), "x", (2, 2)),
          ((e + 2, js - 2), "y", (-3, 1)), ((e + 1, js - 3), "x", (3, 3)), ((e + 2, js - 3), "y", (-4, 2)),
          ((e + 2, js - 1), "x", (0, 2)), ((e + 3, js - 1), "y", (-3, -1)), ((e + 2, js - 2), "x", (1, 3)),
          ((e + 3, js - 2), "y", (-4, 0)), ((e + 2, js - 3), "x", (2, 4)), ((e + 3, js - 3), "y", (-5, 1)),
          ((e + 3, js - 1), "x", (-1, 3)), ((e + 4, js - 1), "y", (-4, -2)), ((e + 3, js - 2), "x", (0, 4)),
          ((e + 4, js - 2), "y", (-5, -1)), ((e + 3, js - 3), "x", (1, 5)), ((e + 4, js - 3), "y", (-6, 0))]
    for (i, j), f, o in se:
        R.append((f, (i, j), "y" if f == "x" else "x", o, 1.0))
    arr = {"x": x, "y": y}
    for tf, (i, j), sf, (di, dj), mult in R:
        arr[tf][i, j, k0:k1] = mult * arr[sf][i + di, j + dj, k0:k1]


def divergence_damping(t: Tile, g, st: DSWState, cfg, u, v, va, u_contra_dyc, v_contra_dxc, ua, divg_d, vc, uc,
                       delpc, ke, wk, dt):
    """DivergenceDamping.__call__ (divergence_damping.py:329-413)."""
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    nz = t.nz
    kz = st.nonzero_nord_k
    d2_bg = st.col["d2_divg"]
    dddmp = cfg["dddmp"]
    da_min_c = g.da_min_c
    sin_sg = [None] + [c3(getattr(g, f"sin_sg{k}")) for k in range(1, 5)]
    cb = (s, e + 2, js, je + 2)  # X_INTERFACE x Y_INTERFACE compute
    if kz > 0:
        # get_delpc (divergence_damping.py:31-91) on levels [0, kz)
        ks = slice(0, kz)
        vfv = 0.5 * (sh(va, 0, -1) + va)
        u_contra = (u - vfv * c3(g.cosa_v)) * c3(g.sina_v)
        m = at(t, j=js) | at(t, j=je + 1)
        u_contra = np.where(m, np.where(vc > 0, u * sh(sin_sg[4], 0, -1), u * sin_sg[2]), u_contra)
        ucd = u_contra * c3(g.dyc)
        ufu = 0.5 * (sh(ua, -1, 0) + ua)
        v_contra = (v - ufu * c3(g.cosa_u)) * c3(g.sina_u)
        m = at(t, i=s) | at(t, i=e + 1)
        v_contra = np.where(m, np.where(uc > 0, v * sh(sin_sg[3], -1, 0), v * sin_sg[1]), v_contra)
        vcd = v_contra * c3(g.dxc)
        m = (
            region(t, s, s + 1, je + 1, je + 2) | region(t, e + 1, e + 2, je + 1, je + 2)
            | region(t, s, s + 1, js - 1, js) | region(t, e + 1, e + 2, js - 1, js)
        )
        vcd = np.where(m, 0.0, vcd)
        # API outputs u_contra_dyc / v_contra_dxc are written on the extent
        # the second computation reads: i in [is-1, ie+1], j in [js-1, je+1]
        put(u_contra_dyc, ucd, s - 1, e + 2, js, je + 2, 0, kz)
        put(v_contra_dxc, vcd, s, e + 2, js - 1, je + 2, 0, kz)
        dpc = sh(v_contra_dxc, 0, -1) - v_contra_dxc + sh(u_contra_dyc, -1, 0) - u_contra_dyc
        dpc = c3(g.rarea_c) * dpc
        put(delpc, dpc, *cb, 0, kz)
        # damping (divergence_damping.py:94-107)
        delpcdt = delpc * dt
        mintmp = np.minimum(0.2, dddmp * np.abs(delpcdt))
        damp = da_min_c * np.maximum(_kfield(d2_bg, t.nk), mintmp)
        put(v_contra_dxc, damp * delpc, *cb, 0, kz)
        put(ke, ke + v_contra_dxc, *cb, 0, kz)
    # copy_computeplus (divergence_damping.py:363)
    put(delpc, divg_d, *cb, kz, nz)
    nn = st.nonzero_nord
    rarea_c = c3(g.rarea_c)
    for n in range(nn):
        nt = nn - n - 1
        fillc = n + 1 != nn
        if fillc:
            _fill_corners_bgrid(t, divg_d, "x", kz, nz + 1)
        # vc_from_divg: origin (is-nt-1, js-nt), domain (n+2nt+2, n+2nt+1)
        put(vc, (sh(divg_d, 1, 0) - divg_d) * c3(g.divg_u), s - nt - 1, e + nt + 2, js - nt, je + nt + 2, kz, nz)
        if fillc:
            _fill_corners_bgrid(t, divg_d, "y", kz, nz + 1)
        put(uc, (sh(divg_d, 0, 1) - divg_d) * c3(g.divg_v), s - nt, e + nt + 2, js - nt - 1, je + nt + 2, kz, nz)
        if fillc:
            _fill_corners_dgrid(t, vc, uc, -1.0, kz, nz)
        # redo_divg_d (divergence_damping.py:136-151)
        dd = sh(uc, 0, -1) - uc + sh(vc, -1, 0) - vc
        m = region(t, s, s + 1, js, js + 1) | region(t, e + 1, e + 2, js, js + 1)
        dd = np.where(m, sh(vc, -1, 0) - vc - uc, dd)
        m = region(t, s, s + 1, je + 1, je + 2) | region(t, e + 1, e + 2, je + 1, je + 2)
        dd = np.where(m, sh(uc, 0, -1) + sh(vc, -1, 0) - vc, dd)
        dd = dd * rarea_c
        put(divg_d, dd, s - nt, e + nt + 2, js - nt, je + nt + 2, kz, nz)
    # _vorticity_calc (divergence_damping.py:481-490)
    if dddmp < 1e-5:
        put(v_contra_dxc, 0.0, s - 3, e + 5, js - 3, je + 5, kz, nz)
    else:
        a2b_ord4(t, g, wk, v_contra_dxc, kz, nz, st.a2b, replace=False)
        sm = abs(dt) * (delpc ** 2.0 + v_contra_dxc ** 2.0) ** 0.5
        put(v_contra_dxc, sm, *cb, kz, nz)
    # damping_nord_highorder_stencil (divergence_damping.py:110-123)
    mintmp = np.minimum(0.2, dddmp * np.abs(v_contra_dxc))
    damp = da_min_c * np.maximum(_kfield(d2_bg, t.nk), mintmp)
    vort = damp * delpc + st.dd8 * divg_d
    put(v_contra_dxc, vort, *cb, kz, nz)
    put(ke, ke + v_contra_dxc, *cb, kz, nz)


def d_sw(t: Tile, g, f0, st: DSWState, cfg, delpc, delp, ptc, pt, u, v, w, uc, vc, ua, va, divgd, mfx, mfy, cx, cy,
         crx, cry, xfx, yfx, q_con, zh, heat_source, diss_est, dt):
    """DGridShallowWaterLagrangianDynamics.__call__ (d_sw.py:843-1131)."""
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    nz, nk = t.nz, t.nk
    full = t.m - 1
    col = st.col
    rarea = c3(g.rarea)
    fxadv(t, g, uc, vc, crx, cry, xfx, yfx, st.uc_contra, st.vc_contra, dt)

    def copied(q):
        copy_corners_xy(t, q, st.y_temporary, nk)
        return q, q, st.y_temporary

    base, qx, qy = copied(delp)
    fvtp2d(t, g, base, qx, qy, crx, cry, xfx, yfx, st.tmp_fx, st.tmp_fy, cfg["hord_dp"], st.fvtp_dp,
           nord=col["nord_v"], damp_c=col["damp_vt"], deln_scratch=st.deln_dp)
    # flux_capacitor (d_sw.py:90-117): full halo domain
    fb = (0, full, 0, full, 0, nz)
    put(cx, cx + crx, *fb)
    put(cy, cy + cry, *fb)
    put(mfx, mfx + st.tmp_fx, *fb)
    put(mfy, mfy + st.tmp_fy, *fb)
    if not cfg["hydrostatic"]:
        delnflux_nosg(t, g, w, st.tmp_fx2, st.tmp_fy2, st.damp_w, st.tmp_wk, col["nord_w"])
        # heat_diss (d_sw.py:347-365): compute domain
        dampw = _kfield(col["damp_w"], nk)
        diss_e = diss_est.copy()
        cond = dampw > 1e-5
        dd8 = _kfield(col["ke_bg"], nk) * abs(dt)
        dw = (st.tmp_fx2 - sh(st.tmp_fx2, 1, 0) + st.tmp_fy2 - sh(st.tmp_fy2, 0, 1)) * rarea
        cb = (s, e + 1, js, je + 1, 0, nz)
        put(st.tmp_dw, np.where(cond, dw, st.tmp_dw), *cb)
        hs = dd8 - st.tmp_dw * (w + 0.5 * st.tmp_dw)
        put(st.tmp_heat_s, np.where(cond, hs, st.tmp_heat_s), *cb)
        put(diss_est, np.where(cond, diss_e + st.tmp_heat_s, diss_est), *cb)
        base, qx, qy = copied(w)
        fvtp2d(t, g, base, qx, qy, crx, cry, xfx, yfx, st.tmp_gx, st.tmp_gy, cfg["hord_vt"], st.fvtp_vt,
               x_mass_flux=st.tmp_fx, y_mass_flux=st.tmp_fy)
        # flux_adjust (d_sw.py:67-87) on w
        val = w * delp + (st.tmp_gx - sh(st.tmp_gx, 1, 0) + st.tmp_gy - sh(st.tmp_gy, 0, 1)) * rarea
        put(w, val, s, e + 1, js, je + 1, 0, nz)
    base, qx, qy = copied(q_con)
    fvtp2d(t, g, base, qx, qy, crx, cry, xfx, yfx, st.tmp_gx, st.tmp_gy, cfg["hord_dp"], st.fvtp_dp_t,
           x_mass_flux=st.tmp_fx, y_mass_flux=st.tmp_fy, mass=delp, nord=col["nord_t"], damp_c=col["damp_t"],
           deln_scratch=st.deln_dp_t)
    val = q_con * delp + (st.tmp_gx - sh(st.tmp_gx, 1, 0) + st.tmp_gy - sh(st.tmp_gy, 0, 1)) * rarea
    put(q_con, val, s, e + 1, js, je + 1, 0, nz)
    base, qx, qy = copied(pt)
    fvtp2d(t, g, base, qx, qy, crx, cry, xfx, yfx, st.tmp_gx, st.tmp_gy, cfg["hord_tm"], st.fvtp_tm,
           x_mass_flux=st.tmp_fx, y_mass_flux=st.tmp_fy, mass=delp, nord=col["nord_v"], damp_c=col["damp_vt"],
           deln_scratch=st.deln_tm)
    # apply_pt_delp_fluxes (d_sw.py:163-195): domain X_INTERFACE x Y_INTERFACE,
    # local region = compute domain
    ptn = pt * delp + (st.tmp_gx - sh(st.tmp_gx, 1, 0) + st.tmp_gy - sh(st.tmp_gy, 0, 1)) * rarea
    dpn = delp + (st.tmp_fx - sh(st.tmp_fx, 1, 0) + st.tmp_fy - sh(st.tmp_fy, 0, 1)) * rarea
    ptn = ptn / dpn
    put(pt, ptn, s, e + 1, js, je + 1, 0, nz)
    put(delp, dpn, s, e + 1, js, je + 1, 0, nz)
    # kinetic_energy_update_part_1 (d_sw.py:198-225), X_INTERFACE x Y_INTERFACE compute
    cosa, rsina = c3(g.cosa), c3(g.rsina)
    ub_cov = 0.5 * (sh(uc, 0, -1) + uc)
    vb_cov = 0.5 * (sh(vc, -1, 0) + vc)
    ubc = (ub_cov - vb_cov * cosa) * rsina
    vbc = (vb_cov - ub_cov * cosa) * rsina
    ucc, vcc = st.uc_contra, st.vc_contra
    m_ns = at(t, j=js) | at(t, j=je + 1)
    m_ew = at(t, i=s) | at(t, i=e + 1)
    ubc = np.where(m_ns, 0.25 * (-sh(ucc, 0, -2) + 3.0 * (sh(ucc, 0, -1) + ucc) - sh(ucc, 0, 1)), ubc)
    ubc = np.where(m_ew, 0.5 * (sh(ucc, 0, -1) + ucc), ubc)
    vbc = np.where(m_ew, 0.25 * (-sh(vcc, -2, 0) + 3.0 * (sh(vcc, -1, 0) + vcc) - sh(vcc, 1, 0)), vbc)
    vbc = np.where(m_ns, 0.5 * (sh(vcc, -1, 0) + vcc), vbc)
    kb = (s, e + 2, js, je + 2, 0, nz)
    put(st.ub_contra, ubc, *kb)
    put(st.vb_contra, vbc, *kb)
    adv_v = advect_along(t, v, vbc, g.rdy, g.dy, g.dya, dt, 1, cfg["hord_mt"])
    adv_u = advect_along(t, u, ubc, g.rdx, g.dx, g.dxa, dt, 0, cfg["hord_mt"])
    put(st.advected_v, adv_v, *kb)
    put(st.advected_u, adv_u, *kb)
    # kinetic_energy_update_part_2 (d_sw.py:228-246)
    ke = 0.5 * dt * (st.ub_contra * st.advected_u + st.vb_contra * st.advected_v)
    dt6 = dt / 6.0

    def corner_ke(io1, jo1, io2, vsign):
        ut_, vt_ = ucc, vcc
        return dt6 * (
            (ut_ + sh(ut_, 0, -1)) * ((io1 + 1) * u - (io1 * sh(u, -1, 0)))
            + (vt_ + sh(vt_, -1, 0)) * ((jo1 + 1) * v - (jo1 * sh(v, 0, -1)))
            + (((jo1 + 1) * ut_ - (jo1 * sh(ut_, 0, -1))) + vsign * ((io1 + 1) * vt_ - (io1 * sh(vt_, -1, 0))))
            * ((io2 + 1) * u - (io2 * sh(u, -1, 0)))
        )

    ke = np.where(region(t, s, s + 1, js, js + 1), corner_ke(0, 0, -1, 1), ke)
    ke = np.where(region(t, e + 1, e + 2, js, js + 1), corner_ke(-1, 0, 0, -1), ke)
    ke = np.where(region(t, e + 1, e + 2, je + 1, je + 2), corner_ke(-1, -1, 0, 1), ke)
    ke = np.where(region(t, s, s + 1, je + 1, je + 2), corner_ke(0, -1, -1, -1), ke)
    put(st.tmp_ke, ke, *kb)
    # compute_vorticity (d_sw.py:468-490): full halo domain
    dx, dy = c3(g.dx), c3(g.dy)
    rdy_tmp = rarea * dx
    rdx_tmp = rarea * dy
    vort = (u - sh(u, 0, 1) * sh(dx, 0, 1) / dx) * rdy_tmp + (sh(v, 1, 0) * sh(dy, 1, 0) / dy - v) * rdx_tmp
    put(st.tmp_wk, vort, *fb)
    # adjust_w_and_qcon (d_sw.py:324-335): compute domain
    cbz = (s, e + 1, js, je + 1, 0, nz)
    wn = w / delp
    wn = np.where(_kfield(col["damp_w"], nk) > 1e-5, wn + st.tmp_dw, wn)
    put(w, wn, *cbz)
    put(q_con, q_con / delp, *cbz)
    divergence_damping(t, g, st, cfg, u, v, va, ptc, st.tmp_vort, ua, divgd, vc, uc, delpc, st.tmp_ke, st.tmp_wk, dt)
    # vort_differencing (d_sw.py:249-265)
    dcon = _kfield(col["d_con"], nk)
    cond = dcon > DCON_THRESHOLD
    vx = st.tmp_vort - sh(st.tmp_vort, 1, 0)
    vy = st.tmp_vort - sh(st.tmp_vort, 0, 1)
    put(st.vort_x_delta, np.where(cond, vx, st.vort_x_delta), s, e + 1, js, je + 2, 0, nz)
    put(st.vort_y_delta, np.where(cond, vy, st.vort_y_delta), s, e + 2, js, je + 1, 0, nz)
    # compute_vort (d_sw.py:307-321): full halo domain
    if cfg.get("do_f3d", False) and not cfg["hydrostatic"]:
        raise NotImplementedError("do_f3d")
    put(st.tmp_vort, st.tmp_wk + c3(f0), *fb)
    base, qx, qy = copied(st.tmp_vort)
    fvtp2d(t, g, base, qx, qy, crx, cry, xfx, yfx, st.tmp_fx, st.tmp_fy, cfg["hord_vt"], st.fvtp_vt)
    # u_and_v_from_ke (d_sw.py:278-299)
    un = u * dx + st.tmp_ke - sh(st.tmp_ke, 1, 0) + st.tmp_fy
    vn = v * dy + st.tmp_ke - sh(st.tmp_ke, 0, 1) - st.tmp_fx
    put(u, un, s, e + 1, js, je + 2, 0, nz)
    put(v, vn, s, e + 2, js, je + 1, 0, nz)
    delnflux_nosg(t, g, st.tmp_wk, st.tmp_ut, st.tmp_vt, st.damp_vt, st.tmp_vort, col["nord_v"])
    # heat_source_from_vorticity_damping (d_sw.py:368-438)
    rdx, rdy = c3(g.rdx), c3(g.rdy)
    ubt = (st.vort_x_delta + st.tmp_vt) * rdx
    fy = u * rdx
    gy = fy * ubt
    vbt = (st.vort_y_delta - st.tmp_ut) * rdy
    fx = v * rdy
    gx = fx * vbt
    kf = _kfield(col["d_con"], nk)
    cond = kf > DCON_THRESHOLD
    u2 = fy + sh(fy, 0, 1)
    du2 = ubt + sh(ubt, 0, 1)
    v2 = fx + sh(fx, 1, 0)
    dv2 = vbt + sh(vbt, 1, 0)
    rsin2, cosa_s = c3(g.rsin2), c3(g.cosa_s)
    dampterm = rsin2 * (
        (ubt * ubt + sh(ubt, 0, 1) * sh(ubt, 0, 1) + vbt * vbt + sh(vbt, 1, 0) * sh(vbt, 1, 0))
        + 2.0 * (gy + sh(gy, 0, 1) + gx + sh(gx, 1, 0))
        - cosa_s * (u2 * dv2 + v2 * du2 + du2 * dv2)
    )
    hs = delp * (st.tmp_heat_s - 0.25 * kf * dampterm)
    hb = (s, e + 2, js, je + 2, 0, nz)
    put(st.tmp_heat_s, np.where(cond, hs, st.tmp_heat_s), *hb)
    if cfg["d_con"] > DCON_THRESHOLD:
        put(heat_source, heat_source + st.tmp_heat_s, s, e + 1, js, je + 1, 0, nz)
    # update_u_and_v (d_sw.py:441-465)
    cond = _kfield(col["damp_vt"], nk) > 1e-5
    put(u, np.where(cond, u + st.tmp_vt, u), s, e + 1, js, je + 2, 0, nz)
    put(v, np.where(cond, v - st.tmp_ut, v), s, e + 2, js, je + 1, 0, nz)

"""The fast saturation adjustment of the vertical remapping (reference
``fv3core/stencils/saturation_adjustment.py``, SatAdjust3d, run by
LagrangianToEulerian when do_sat_adj is set, remapping.py:570-598).

Test infrastructure: the oracle the CUDA saturation adjustment is checked
against, not part of the product.  One tile's storages ``[m, m, nk]``; the
stencil runs on the compute domain from level kmp down (SatAdjust3d,
saturation_adjustment.py:935-968).  Every point is independent: the
functions below take arrays of the box's points and follow the reference's
statements in order, a field ``if`` as a masked assignment whose condition
is evaluated before its body (gt4py's numpy backend).  The saturation
tables are computed on the fly from the point's table index, as the
reference does (qs_table*_fn, des*_table), with exp and log from ``_math``.
Expressions keep the reference's association.
"""
import math

import numpy as np

from fv3core_b200 import constants as C

from . import _math

# saturation_adjustment.py:16-39
DC_VAP = C.CP_VAP - C.C_LIQ
DC_ICE = C.C_LIQ - C.C_ICE
LV0 = C.HLV - DC_VAP * C.TICE
LI00 = C.HLF - DC_ICE * C.TICE
LI2 = LV0 + LI00
D2ICE = DC_VAP + DC_ICE
E00 = 611.21
TMIN = C.TICE - 160.0
DELT = 0.1
TICE = C.TICE
T_WFR = TICE - 40.0
TICE0 = TICE - 0.01
LAT2 = (C.HLV + C.HLF) ** 2
QS_LENGTH = 2621


def _w(c, a, b):
    return np.where(c, a, b)


def _min(a, b):
    """gtscript min (numpy minimum)."""
    return np.minimum(a, b)


def _max(a, b):
    return np.maximum(a, b)


def _dim(a, b):
    """basic_operations.dim (basic_operations.py:44-46)."""
    d = a - b
    return _w(d > 0, d, 0)


# ---------------------------------------------------------------- tables
def _tem_lower(i):
    return TMIN + DELT * i


def _tem_upper(i):
    return 253.16 + DELT * i


def _q_table_oneline(dhc, lhc, tem):
    """saturation_adjustment.py:52-60."""
    return E00 * _math.exp((dhc * _math.log(tem / TICE) + (tem - TICE) / (tem * TICE) * lhc) / C.RVGAS)


def _vapor(tem):
    return _q_table_oneline(DC_VAP, LV0, tem)


def _ice(tem):
    return _q_table_oneline(D2ICE, LI2, tem)


def qs_table2(i):
    """qs_table2_fn (saturation_adjustment.py:94-128)."""
    tem0 = _tem_lower(i)
    t2 = _w(i < 1600, _ice(tem0), _vapor(tem0))
    # i == 1599
    tt = _ice(tem0)
    tu = _tem_upper(i - 1400)
    tt = (0.05 * (TICE - tu)) * tt + (0.05 * (tu - 253.16)) * _vapor(tu)
    m1 = _ice(_tem_lower(1598))
    p1 = _vapor(_tem_lower(1600))
    t2 = _w(i == 1599, 0.25 * (m1 + 2.0 * tt + p1), t2)
    # i == 1600
    tt = _vapor(_tem_upper(i - 1400))
    m1 = _ice(_tem_lower(1599))
    p1 = _vapor(_tem_lower(1601))
    t2 = _w(i == 1600, 0.25 * (m1 + 2.0 * tt + p1), t2)
    return t2


def qs_tablew(i):
    """qs_tablew_fn (131-134)."""
    return _vapor(_tem_lower(i))


def _des_end(t, i, z, des, table_fn):
    """des_end (137-145)."""
    diff = t - table_fn(i - 1)
    return _w(i == QS_LENGTH - 1, _max(z, diff), des)


def des2(i):
    """des2_table (148-157)."""
    t = qs_table2(i)
    des = _max(0.0, qs_table2(i + 1) - t)
    return _des_end(t, i, 0.0, des, qs_table2)


def desw(i):
    """desw_table (160-167); its des_end reads qs_table2 (as the reference's
    shared des_end does)."""
    t = qs_tablew(i)
    des = _max(0.0, qs_tablew(i + 1) - t)
    return _des_end(t, i, 0.0, des, qs_table2)


def _ap1(ta):
    """ap1_for_wqs2 (454-457)."""
    ap1 = 10.0 * _dim(ta, TMIN) + 1.0
    return _min(ap1, QS_LENGTH) - 1


def _wqsat_and_dqdt(tab, des, des_2, des_p1, ap1, it, it2, ta, den):
    """wqsat_and_dqdt (487-494)."""
    es = tab + (ap1 - it) * des
    denom = C.RVGAS * ta * den
    wqsat = es / denom
    dqdt = 10.0 * (des_2 + (ap1 - it2) * (des_p1 - des_2))
    dqdt = dqdt / denom
    return wqsat, dqdt


def wqs2_w(ta, den):
    """wqs2_fn_w (512-519)."""
    ap1 = _ap1(ta)
    it = np.floor(ap1)
    it2 = np.floor(ap1 - 0.5)
    return _wqsat_and_dqdt(qs_tablew(it), desw(it), desw(it2), desw(it2 + 1), ap1, it, it2, ta, den)


def wqs2_2(ta, den):
    """wqs2_fn_2 (502-509)."""
    ap1 = _ap1(ta)
    it = np.floor(ap1)
    it2 = np.floor(ap1 - 0.5)
    return _wqsat_and_dqdt(qs_table2(it), des2(it), des2(it2), des2(it2 + 1), ap1, it, it2, ta, den)


def _wqs1(tab, des, ap1, it, ta, den):
    """wqsat_wsq1 (497-499)."""
    es = tab + (ap1 - it) * des
    return es / (C.RVGAS * ta * den)


# ---------------------------------------------------------------- processes
def _cvm(mc_air, qv, c_vap, q_liq, q_sol):
    """compute_cvm (170-172)."""
    return mc_air + qv * c_vap + q_liq * C.C_LIQ + q_sol * C.C_ICE


def _lat_i(pt1, cvm):
    """update_latent_heat_coefficient_i (398-402)."""
    lhi = LI00 + DC_ICE * pt1
    return lhi, lhi / cvm


def _lat(pt1, cvm, lv00, d0_vap):
    """update_latent_heat_coefficient (412-416)."""
    lhl = lv00 + d0_vap * pt1
    lcp2 = lhl / cvm
    lhi, icp2 = _lat_i(pt1, cvm)
    return lhl, lhi, lcp2, icp2


def _minmax_tmp(qa, qb):
    """minmax_tmp_h20 (202-205)."""
    return _min(-qa, _max(qb, 0.0))


def satadjust(peln, qv, ql, qi, qr, qs, cappa, qg, pt, dp, delz, te0, q_con, qa, area, hs, pkz, sdt, zvir,
              fac_i2s, do_qa, consv_te, c_air, c_vap, mdt, fac_r2g, fac_smlt, fac_l2r, fac_imlt, d0_vap, lv00,
              fac_v2l, fac_l2v, last_step, cfg):
    """satadjust (saturation_adjustment.py:544-932), nonhydrostatic, on
    arrays of the points; ``cfg`` holds the SatAdjustConfig externals.
    Returns the updated (qv, ql, qi, qr, qs, qg, cappa, pt, te0, q_con, qa,
    pkz)."""
    with np.errstate(all="ignore"):
        q_liq = ql + qr
        q_sol = qi + qs + qg
        qpz = q_liq + q_sol
        pt1 = pt / ((1.0 + zvir * qv) * (1.0 - qpz))
        t0 = pt1
        qpz = qpz + qv
        den = -dp / (C.GRAV * delz)
        mc_air = (1.0 - qpz) * c_air
        cvm = _cvm(mc_air, qv, c_vap, q_liq, q_sol)
        lhi, icp2 = _lat_i(pt1, cvm)
        if consv_te:
            te0 = -cvm * t0
        # fix negative cloud ice with snow
        c = qi < 0.0
        qs = _w(c, qs + qi, qs)
        qi = _w(c, 0.0, qi)
        # melt_cloud_ice (185-199)
        c = (qi > 1.0e-8) & (pt1 > TICE)
        factmp = fac_imlt * (pt1 - TICE) / icp2
        sink = _w(qi < factmp, qi, factmp)
        qi = _w(c, qi - sink, qi)
        ql = _w(c, ql + sink, ql)
        q_liq = _w(c, q_liq + sink, q_liq)
        q_sol = _w(c, q_sol - sink, q_sol)
        cvm = _w(c, _cvm(mc_air, qv, c_vap, q_liq, q_sol), cvm)
        pt1 = _w(c, pt1 + (-sink) * lhi / cvm, pt1)
        lhi, icp2 = _lat_i(pt1, cvm)
        # fix_negative_snow (208-218)
        c1 = qs < 0.0
        c2 = ~c1 & (qg < 0.0)
        tmp = _minmax_tmp(qg, qs)
        qg = _w(c1, qg + qs, _w(c2, qg + tmp, qg))
        qs = _w(c1, 0.0, _w(c2, qs - tmp, qs))
        # fix_negative_cloud_water (221-232)
        c1 = ql < 0.0
        c2 = ~c1 & (qr < 0.0)
        t1 = _minmax_tmp(ql, qr)
        t2 = _minmax_tmp(qr, ql)
        ql_n = _w(c1, ql + t1, _w(c2, ql - t2, ql))
        qr = _w(c1, qr - t1, _w(c2, qr + t2, qr))
        ql = ql_n
        # complete_freezing (235-246)
        dtmp = TICE - 48.0 - pt1
        c = (ql > 0.0) & (dtmp > 0.0)
        sink = _min(ql, dtmp / icp2)
        ql = _w(c, ql - sink, ql)
        qi = _w(c, qi + sink, qi)
        q_liq = _w(c, q_liq - sink, q_liq)
        q_sol = _w(c, q_sol + sink, q_sol)
        cvm = _w(c, _cvm(mc_air, qv, c_vap, q_liq, q_sol), cvm)
        pt1 = _w(c, pt1 + sink * lhi / cvm, pt1)
        wqsat, dq2dt = wqs2_w(pt1, den)
        lhl, lhi, lcp2, icp2 = _lat(pt1, cvm, lv00, d0_vap)
        diff_ice = _dim(TICE, pt1) / 48.0
        dimmin = _min(1.0, diff_ice)
        tcp3 = lcp2 + icp2 * dimmin
        dq0 = (qv - wqsat) / (1.0 + tcp3 * dq2dt)
        c = dq0 > 0
        src_sat = _min(cfg["sat_adj0"] * dq0, _max(cfg["ql_gen"] - ql, fac_v2l * dq0))
        factor = -_min(1, fac_l2v * 10.0 * (1.0 - qv / wqsat))
        src_ev = -_min(ql, factor * dq0)
        src = _w(c, src_sat, src_ev)
        # wqsat_correct (443-450)
        qv = qv - src
        ql = ql + src
        q_liq = q_liq + src
        cvm = _cvm(mc_air, qv, c_vap, q_liq, q_sol)
        pt1 = pt1 + src * lhl / cvm
        lhl, lhi, lcp2, icp2 = _lat(pt1, cvm, lv00, d0_vap)
        diff_ice = _dim(TICE, pt1) / 48.0
        dimmin = _min(1.0, diff_ice)
        tcp3 = lcp2 + icp2 * dimmin
        if last_step:
            wqsat, dq2dt = wqs2_w(pt1, den)
            dq0 = (qv - wqsat) / (1.0 + tcp3 * dq2dt)
            c = dq0 > 0
            factor = -_min(1, fac_l2v * 10.0 * (1.0 - qv / wqsat))
            src = _w(c, dq0, -_min(ql, factor * dq0))
            qv = qv - src
            ql = ql + src
            q_liq = q_liq + src
            cvm = _cvm(mc_air, qv, c_vap, q_liq, q_sol)
            pt1 = pt1 + src * lhl / cvm
            lhl, lhi, lcp2, icp2 = _lat(pt1, cvm, lv00, d0_vap)
        # homogenous_freezing (249-262)
        dtmp = T_WFR - pt1
        c = (ql > 0.0) & (dtmp > 0.0)
        sink = _min(ql, dtmp / icp2)
        sink = _min(sink, ql * dtmp * 0.125)
        ql = _w(c, ql - sink, ql)
        qi = _w(c, qi + sink, qi)
        q_liq = _w(c, q_liq - sink, q_liq)
        q_sol = _w(c, q_sol + sink, q_sol)
        cvm = _w(c, _cvm(mc_air, qv, c_vap, q_liq, q_sol), cvm)
        pt1 = _w(c, pt1 + sink * lhi / cvm, pt1)
        lhi, icp2 = _lat_i(pt1, cvm)
        exptc = _math.exp(0.66 * (TICE0 - pt1))
        # heterogeneous_freezing (265-280), dt_bigg = mdt
        tc = TICE0 - pt1
        c = (ql > 0.0) & (tc > 0.0)
        sink = 3.3333e-10 * mdt * (exptc - 1.0) * den * ql ** 2
        sink = _min(ql, sink)
        sink = _min(sink, tc / icp2)
        ql = _w(c, ql - sink, ql)
        qi = _w(c, qi + sink, qi)
        q_liq = _w(c, q_liq - sink, q_liq)
        q_sol = _w(c, q_sol + sink, q_sol)
        cvm = _w(c, _cvm(mc_air, qv, c_vap, q_liq, q_sol), cvm)
        pt1 = _w(c, pt1 + sink * lhi / cvm, pt1)
        lhi, icp2 = _lat_i(pt1, cvm)
        # make_graupel (283-297)
        dtmp = (TICE - 0.1) - pt1
        c = (qr > 1e-7) & (dtmp > 0.0)
        rainfac = (dtmp * 0.025) ** 2
        tmp = _w(1.0 < rainfac, qr, rainfac * qr)
        sink = _min(tmp, fac_r2g * dtmp / icp2)
        qr = _w(c, qr - sink, qr)
        qg = _w(c, qg + sink, qg)
        q_liq = _w(c, q_liq - sink, q_liq)
        q_sol = _w(c, q_sol + sink, q_sol)
        cvm = _w(c, _cvm(mc_air, qv, c_vap, q_liq, q_sol), cvm)
        pt1 = _w(c, pt1 + sink * lhi / cvm, pt1)
        lhi, icp2 = _lat_i(pt1, cvm)
        # melt_snow (300-320)
        dtmp = pt1 - (TICE + 0.1)
        dimqs = _dim(cfg["qs_mlt"], ql)
        c = (qs > 1e-7) & (dtmp > 0.0)
        snowfac = (dtmp * 0.1) ** 2
        tmp = _w(1.0 < snowfac, qs, snowfac * qs)
        sink = _min(tmp, fac_smlt * dtmp / icp2)
        tmp = _min(sink, dimqs)
        qs = _w(c, qs - sink, qs)
        ql = _w(c, ql + tmp, ql)
        qr = _w(c, qr + sink - tmp, qr)
        q_liq = _w(c, q_liq + sink, q_liq)
        q_sol = _w(c, q_sol - sink, q_sol)
        cvm = _w(c, _cvm(mc_air, qv, c_vap, q_liq, q_sol), cvm)
        pt1 = _w(c, pt1 - sink * lhi / cvm, pt1)
        # autoconversion_cloud_to_rain (323-329)
        c = ql > cfg["ql0_max"]
        sink = fac_l2r * (ql - cfg["ql0_max"])
        qr = _w(c, qr + sink, qr)
        ql = _w(c, ql - sink, ql)
        iqs2, dqsdt = wqs2_2(pt1, den)
        expsubl = _math.exp(0.875 * _math.log(qi * den))
        lhl, lhi, lcp2, icp2 = _lat(pt1, cvm, lv00, d0_vap)
        tcp2 = lcp2 + icp2
        adj_fac = 1.0 if last_step else cfg["sat_adj0"]
        # sublimation (332-395)
        t_sub, qi_gen, qi_lim = cfg["t_sub"], cfg["qi_gen"], cfg["qi_lim"]
        c_cold = pt1 < t_sub
        c_mid = ~c_cold & (pt1 < TICE0)
        dq = qv - iqs2
        sink = adj_fac * dq / (1.0 + tcp2 * dqsdt)
        pidep = _w(qi > 1.0e-8,
                   sdt * dq * 349138.78 * expsubl / (iqs2 * den * LAT2 / (0.0243 * C.RVGAS * pt1 ** 2.0)
                                                     + 4.42478e4), 0.0)
        tmp = TICE - pt1
        qi_crt = _w(qi_lim < 0.1 * tmp, qi_gen * qi_lim / den, qi_gen * 0.1 * tmp / den)
        maxtmp = _w(qi_crt - qi > pidep, qi_crt - qi, pidep)
        src_p = _w(sink < maxtmp, sink, maxtmp)
        src_p = _w(src_p < tmp / tcp2, src_p, tmp / tcp2)
        dimtmp = _dim(pt1, t_sub)
        pid_n = _w(1.0 < (dimtmp * 0.2), pidep, pidep * dimtmp * 0.2)
        src_n = _w(pid_n > sink, pid_n, sink)
        src_n = _w(src_n > -qi, src_n, -qi)
        src = _w(c_cold, _dim(qv, 1e-6), _w(c_mid, _w(dq > 0.0, src_p, src_n), 0.0))
        qv = qv - src
        qi = qi + src
        q_sol = q_sol + src
        cvm = _cvm(mc_air, qv, c_vap, q_liq, q_sol)
        lh = lhl + lhi
        pt1 = pt1 + src * lh / cvm
        # virtual temperature and cappa
        q_con = q_liq + q_sol
        tmp = 1.0 + zvir * qv
        pt = pt1 * tmp * (1.0 - q_con)
        tmp = tmp * C.RDGAS
        cappa = tmp / (tmp + cvm)
        # fix negative graupel with available cloud ice
        c = qg < 0
        mintmp = _min(-qg, _max(0.0, qi))
        qg = _w(c, qg + mintmp, qg)
        qi = _w(c, qi - mintmp, qi)
        # autoconversion from cloud ice to snow
        qim = cfg["qi0_max"] / den
        c = qi > qim
        sink = fac_i2s * (qi - qim)
        qi = _w(c, qi - sink, qi)
        qs = _w(c, qs + sink, qs)
        if consv_te:
            te0 = dp * (te0 + cvm * pt1)
        cvm = mc_air + (qv + q_liq + q_sol) * c_vap
        lhl, lhi, lcp2, icp2 = _lat(pt1, cvm, lv00, d0_vap)
        if do_qa and last_step:
            if cfg["rad_snow"]:
                q_sol = qi + qs + qg if cfg["rad_graupel"] else qi + qs
            else:
                q_sol = qi
            q_liq = ql + qr if cfg["rad_rain"] else ql
            q_cond = q_sol + q_liq
            tin = pt1 if cfg["tintqs"] else pt1 - (lcp2 * q_cond + icp2 * q_sol)
            ap1 = _ap1(tin)
            it = np.floor(ap1)
            wqs1 = _wqs1(qs_tablew(it), desw(it), ap1, it, tin, den)
            iqs1 = _wqs1(qs_table2(it), des2(it), ap1, it, tin, den)
            rqi = _w(q_cond > 1e-6, q_sol / q_cond, (TICE - tin) / (TICE - T_WFR))
            qstar = _w(tin < T_WFR, iqs1, _w(tin >= TICE, wqs1, rqi * iqs1 + (1.0 - rqi) * wqs1))
            mindw = _min(1.0, np.abs(hs) / (10.0 * C.GRAV))
            dw = cfg["dw_ocean"] + (cfg["dw_land"] - cfg["dw_ocean"]) * mindw
            dbl_sqrt_area = dw * (area ** 0.5 / 100.0e3) ** 0.5
            maxtmp = _max(0.01, dbl_sqrt_area)
            hvar = _min(0.2, maxtmp)
            rh = qpz / qstar
            cond = (rh > 0.75) & (qpz > 1.0e-8)
            dq = hvar * qpz
            q_plus = qpz + dq
            q_minus = qpz - dq
            icloud_f, cld_min = cfg["icloud_f"], cfg["cld_min"]
            if icloud_f == 2:
                qa_c = _w(qpz > qstar, 1.0, _w((qstar < q_plus) & (q_cond > 1.0e-8),
                                              _min(1.0, ((q_plus - qstar) / dq) ** 2), 0.0))
            else:
                inner = (q_plus - qstar) / (dq + dq) if icloud_f == 0 else \
                    (q_plus - qstar) / (2.0 * dq * (1.0 - q_cond))
                qa_m = _w(qstar < q_plus, inner, 0.0)
                qa_m = _w(q_cond > 1.0e-8, _max(cld_min, qa_m), qa_m)
                qa_m = _min(1, qa_m)
                qa_c = _w(qstar < q_minus, 1.0, qa_m)
            qa = _w(cond, qa_c, 0.0)
        pkz = _math.exp(cappa * _math.log(C.RDG * dp / delz * pt))
    return qv, ql, qi, qr, qs, qg, cappa, pt, te0, q_con, qa, pkz


def sat_adjust_3d(t, fields, cfg, area, hs, zvir, mdt, fast_mp_consv, last_step, kmp):
    """SatAdjust3d.__call__ (saturation_adjustment.py:970-1024) on one tile:
    ``fields`` holds te (the remap passes dp1), qvapor, qliquid, qice, qrain,
    qsnow, qgraupel, qcld, peln, delp, delz, q_con, pt, pkz, cappa (updated in
    place); area, hs 2-D; the stencil's box is the compute domain, levels
    [kmp, npz)."""
    sdt = 0.5 * mdt
    fac_i2s = 1.0 - math.exp(-mdt / cfg["tau_i2s"])
    fac_v2l = 1.0 - math.exp(-sdt / cfg["tau_v2l"])
    fac_r2g = 1.0 - math.exp(-mdt / cfg["tau_r2g"])
    fac_l2r = 1.0 - math.exp(-mdt / cfg["tau_l2r"])
    fac_l2v = 1.0 - math.exp(-sdt / cfg["tau_l2v"])
    fac_l2v = min(cfg["sat_adj0"], fac_l2v)
    fac_imlt = 1.0 - math.exp(-sdt / cfg["tau_imlt"])
    fac_smlt = 1.0 - math.exp(-mdt / cfg["tau_smlt"])
    c_air, c_vap = C.CV_AIR, C.CV_VAP
    d0_vap = c_vap - C.C_LIQ
    lv00 = C.HLV - d0_vap * TICE
    B = (slice(t.isc, t.iec + 1), slice(t.jsc, t.jec + 1), slice(kmp, t.nz))
    f = {k: v[B] for k, v in fields.items()}
    a2 = np.asarray(area)[B[:2]][..., None]
    h2 = np.asarray(hs)[B[:2]][..., None]
    out = satadjust(f["peln"], f["qvapor"], f["qliquid"], f["qice"], f["qrain"], f["qsnow"], f["cappa"],
                    f["qgraupel"], f["pt"], f["delp"], f["delz"], f["te"], f["q_con"], f["qcld"], a2, h2, f["pkz"],
                    sdt, zvir, fac_i2s, True, fast_mp_consv, c_air, c_vap, mdt, fac_r2g, fac_smlt, fac_l2r,
                    fac_imlt, d0_vap, lv00, fac_v2l, fac_l2v, last_step, cfg)
    names = ("qvapor", "qliquid", "qice", "qrain", "qsnow", "qgraupel", "cappa", "pt", "te", "q_con", "qcld", "pkz")
    for name, val in zip(names, out):
        fields[name][B] = np.broadcast_to(val, fields[name][B].shape)

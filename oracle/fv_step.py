"""The step preamble and epilogue of DynamicalCore.step_dynamics (reference
``fv3core/stencils/fv_dynamics.py``): compute_preamble (fv_setup,
moist_cv.py:197-228, and pt_adjust, fv_dynamics.py:32-34), post_remap
(set_omega 37-39 and the omega hyperdiffusion, 109-133) and wrapup
(AdjustNegativeTracerMixingRatio, neg_adj3.py; CubedToLatLon,
c2l_ord.py).

Test infrastructure: the oracle the CUDA kernels of these stages are
checked against.  One tile's storages ``[m, m, nk]``; every stage works on
the compute domain and the npz layers, as the reference's stencils are
built (origin_compute, domain_compute).  Column stencils follow the gt4py
numpy backend's order: FORWARD / BACKWARD levels one after another,
PARALLEL intervals in the order they are written, a field ``if`` as a
masked assignment whose condition is evaluated before its body.
"""
import numpy as np

from fv3core_b200 import constants as C

from . import _math
from ._util import Tile, c3, sh


def _comp(t: Tile):
    return slice(t.isc, t.iec + 1), slice(t.jsc, t.jec + 1), slice(0, t.nz)


def _sel(a, b):
    """The reference's ``a if a < b else b`` (min with its NaN behaviour)."""
    return np.where(a < b, a, b)


def _pos(a):
    """The reference's ``0.0 if 0.0 > a else a``."""
    return np.where(0.0 > a, 0.0, a)


# ------------------------------------------------------------ preamble
def fv_setup(t: Tile, qvapor, qliquid, qrain, qsnow, qice, qgraupel, q_con, cvm, pkz, pt, cappa, delp, delz,
             dp1):
    """moist_cv.fv_setup with moist_phys (moist_cv.py:197-228), nwat = 6."""
    I, J, K = _comp(t)
    qv = qvapor[I, J, K]
    ql = qliquid[I, J, K] + qrain[I, J, K]
    qs = qice[I, J, K] + qsnow[I, J, K] + qgraupel[I, J, K]
    gz = ql + qs
    cv = (1.0 - (qv + gz)) * C.CV_AIR + qv * C.CV_VAP + ql * C.C_LIQ + qs * C.C_ICE
    cvm[I, J, K] = cv
    q_con[I, J, K] = gz
    d1 = C.ZVIR * qv
    dp1[I, J, K] = d1
    ca = C.RDGAS / (C.RDGAS + cv / (1.0 + d1))
    cappa[I, J, K] = ca
    pkz[I, J, K] = _math.exp(ca * _math.log(C.RDG * delp[I, J, K] * pt[I, J, K] * (1.0 + d1) * (1.0 - gz) / delz[I, J, K]))


def pt_adjust(t: Tile, pkz, dp1, q_con, pt):
    """fv_dynamics.py:32-34."""
    I, J, K = _comp(t)
    pt[I, J, K] = pt[I, J, K] * (1.0 + dp1[I, J, K]) * (1.0 - q_con[I, J, K]) / pkz[I, J, K]


def set_omega(t: Tile, delp, delz, w, omga):
    """fv_dynamics.py:37-39."""
    I, J, K = _comp(t)
    omga[I, J, K] = delp[I, J, K] / delz[I, J, K] * w[I, J, K]


# ------------------------------------------------------------ neg_adj3
def _fix_negative_ice(qvapor, qice, qsnow, qgraupel, qrain, qliquid, pt, lcpk, icpk):
    """neg_adj3.py:12-55."""
    qsum = qice + qsnow
    pos = qsum > 0.0
    c1 = pos & (qice < 0.0)
    c2 = pos & ~(qice < 0.0) & (qsnow < 0.0)
    qice, qsnow = np.where(c1, 0.0, qice), np.where(c1, qsum, qsnow)
    qsnow, qice = np.where(c2, 0.0, qsnow), np.where(c2, qsum, qice)
    qice = np.where(~pos, 0.0, qice)
    qsnow = np.where(~pos, 0.0, qsnow)
    qgraupel = np.where(~pos, qgraupel + qsum, qgraupel)
    m = qgraupel < 0.0
    dq = _sel(qsnow, -qgraupel)
    qsnow = np.where(m, qsnow - dq, qsnow)
    qgraupel = np.where(m, qgraupel + dq, qgraupel)
    m2 = m & (qgraupel < 0.0)
    dq = _sel(qice, -qgraupel)
    qice = np.where(m2, qice - dq, qice)
    qgraupel = np.where(m2, qgraupel + dq, qgraupel)
    m = (qgraupel < 0.0) & (qrain > 0.0)
    dq = _sel(qrain, -qgraupel)
    qgraupel = np.where(m, qgraupel + dq, qgraupel)
    qliquid = np.where(m, qliquid - dq, qliquid)
    pt = np.where(m, pt + dq * icpk, pt)
    m = (qgraupel < 0.0) & (qliquid > 0.0)
    dq = _sel(qliquid, -qgraupel)
    qgraupel = np.where(m, qgraupel + dq, qgraupel)
    qliquid = np.where(m, qliquid - dq, qliquid)
    pt = np.where(m, pt + dq * icpk, pt)
    m = (qgraupel < 0.0) & (qvapor > 0.0)
    dq = _sel(0.999 * qvapor, -qgraupel)
    qgraupel = np.where(m, qgraupel + dq, qgraupel)
    qvapor = np.where(m, qvapor - dq, qvapor)
    pt = np.where(m, pt + dq * (icpk + lcpk), pt)
    return qvapor, qice, qsnow, qgraupel, qrain, qliquid, pt


def _fix_negative_liq(qvapor, qice, qsnow, qgraupel, qrain, qliquid, pt, lcpk, icpk):
    """neg_adj3.py:58-98."""
    qsum = qliquid + qrain
    pos_qgraupel = _pos(qgraupel)
    pos = qsum > 0.0
    c1 = pos & (qrain < 0.0)
    c2 = pos & ~(qrain < 0.0) & (qliquid < 0.0)
    qrain_in = qrain
    qrain, qliquid = np.where(c1, 0.0, qrain), np.where(c1, qsum, qliquid)
    qliquid, qrain = np.where(c2, 0.0, qliquid), np.where(c2, qsum, qrain)
    neg = ~pos
    qliquid = np.where(neg, 0.0, qliquid)
    qrain_tmp = np.where(neg, qsum, 0.0)
    dq = _sel(pos_qgraupel, -qrain_tmp)
    qrain_tmp = np.where(neg, qrain_tmp + dq, qrain_tmp)
    qgraupel = np.where(neg, qgraupel - dq, qgraupel)
    pt = np.where(neg, pt - dq * icpk, pt)
    m = neg & (qrain_in < 0.0)
    dq = _sel(qice + qsnow, -qrain_tmp)
    qrain_tmp = np.where(m, qrain_tmp + dq, qrain_tmp)
    dq1 = _sel(dq, qsnow)
    qsnow = np.where(m, qsnow - dq1, qsnow)
    qice = np.where(m, qice + dq1 - dq, qice)
    pt = np.where(m, pt - dq * icpk, pt)
    qrain = np.where(neg, qrain_tmp, qrain)
    m = neg & (qrain < 0.0) & (qvapor > 0.0)
    dq = _sel(0.999 * qvapor, -qrain)
    qvapor = np.where(m, qvapor - dq, qvapor)
    qrain = np.where(m, qrain + dq, qrain)
    pt = np.where(m, pt + dq * lcpk, pt)
    return qvapor, qice, qsnow, qgraupel, qrain, qliquid, pt


def fix_neg_water(t: Tile, pt, delz, qvapor, qliquid, qrain, qsnow, qice, qgraupel, lv00, d0_vap):
    """neg_adj3.py:101-145 (pointwise)."""
    I, J, K = _comp(t)
    qv, ql, qr, qs, qi, qg, p = (a[I, J, K] for a in (qvapor, qliquid, qrain, qsnow, qice, qgraupel, pt))
    q_liq = _pos(ql + qr)
    q_sol = _pos(qi + qs)
    cpm = (1.0 - (qv + q_liq + q_sol)) * C.CV_AIR + qv * C.CV_VAP + q_liq * C.C_LIQ + q_sol * C.C_ICE
    lcpk = (lv00 + d0_vap * p) / cpm
    icpk = (C.LI0 + C.DC_ICE * p) / cpm
    qv, qi, qs, qg, qr, ql, p = _fix_negative_ice(qv, qi, qs, qg, qr, ql, p, lcpk, icpk)
    qv, qi, qs, qg, qr, ql, p = _fix_negative_liq(qv, qi, qs, qg, qr, ql, p, lcpk, icpk)
    for a, v in zip((qvapor, qliquid, qrain, qsnow, qice, qgraupel, pt), (qv, ql, qr, qs, qi, qg, p)):
        a[I, J, K] = v


def fillq(t: Tile, q, dp):
    """neg_adj3.py:67-88 (column sums sum1, sum2 per column)."""
    I, J, _ = _comp(t)
    nz = t.nz
    Q, D = q[I, J, :nz], dp[I, J, :nz]
    sum1 = np.zeros(Q.shape[:2])
    sum2 = np.zeros(Q.shape[:2])
    for k in range(nz):
        m = Q[..., k] > 0
        sum1 = np.where(m, sum1 + Q[..., k] * D[..., k], sum1)
    for k in range(nz - 1, -1, -1):
        qk, dk = Q[..., k], D[..., k]
        m = (qk < 0.0) & (sum1 >= 0)
        dq = _sel(sum1, -qk * dk)
        sum1 = np.where(m, sum1 - dq, sum1)
        sum2 = np.where(m, sum2 + dq, sum2)
        Q[..., k] = np.where(m, qk + dq / dk, qk)
    for k in range(nz - 1, -1, -1):
        qk, dk = Q[..., k], D[..., k]
        m = (qk > 0.0) & (sum1 >= 1e-12) & (sum2 > 0)
        dq = _sel(sum2, qk * dk)
        sum2 = np.where(m, sum2 - dq, sum2)
        Q[..., k] = np.where(m, qk - dq / dk, qk)
    q[I, J, :nz] = Q


def fix_water_vapor_down(t: Tile, qvapor, dp):
    """neg_adj3.py:240-291.  The temporary dp_bot is written on the bottom
    level only; the numpy backend's other levels hold no value (NaN here),
    which the borrowing branch would read if the bottom level stayed
    negative."""
    I, J, _ = _comp(t)
    nz = t.nz
    Q, D = qvapor[I, J, :nz], dp[I, J, :nz]
    upper_fix = np.zeros(Q.shape)
    lower_fix = np.zeros(Q.shape)
    dp_bot = np.full(Q.shape, np.nan)
    Q[..., 0] = np.where(Q[..., 0] < 0.0, 0.0, Q[..., 0])
    Q[..., 1] = np.where(Q[..., 0] < 0, Q[..., 1] + Q[..., 0] * D[..., 0] / D[..., 1], Q[..., 1])
    for k in range(1, nz - 1):
        dq = Q[..., k - 1] * D[..., k - 1]
        m = lower_fix[..., k - 1] != 0
        Q[..., k] = np.where(m, Q[..., k] + lower_fix[..., k - 1] / D[..., k], Q[..., k])
        m = (Q[..., k] < 0) & (Q[..., k - 1] > 0)
        dq = np.where(m, _sel(dq, -Q[..., k] * D[..., k]), dq)
        upper_fix[..., k] = np.where(m, dq, upper_fix[..., k])
        Q[..., k] = np.where(m, Q[..., k] + dq / D[..., k], Q[..., k])
        m = Q[..., k] < 0
        lower_fix[..., k] = np.where(m, Q[..., k] * D[..., k], lower_fix[..., k])
        Q[..., k] = np.where(m, 0.0, Q[..., k])
    for k in range(0, nz - 2):
        m = upper_fix[..., k + 1] != 0
        Q[..., k] = np.where(m, Q[..., k] - upper_fix[..., k + 1] / D[..., k], Q[..., k])
    kb = nz - 1
    m = lower_fix[..., kb - 1] > 0
    Q[..., kb] = np.where(m, Q[..., kb] + lower_fix[..., kb] / D[..., kb], Q[..., kb])
    upper_fix[..., kb] = Q[..., kb]
    dp_bot[..., kb] = D[..., kb]
    for k in range(nz - 2, -1, -1):
        dq = Q[..., k] * D[..., k]
        m = (upper_fix[..., k + 1] < 0) & (Q[..., k] > 0)
        cap = dq >= -upper_fix[..., k + 1] * dp_bot[..., k]
        dq = np.where(m & cap, -upper_fix[..., k + 1] * dp_bot[..., k], dq)
        Q[..., k] = np.where(m, Q[..., k] - dq / D[..., k], Q[..., k])
        upper_fix[..., k] = np.where(m, upper_fix[..., k + 1] + dq / dp_bot[..., k], upper_fix[..., k + 1])
    for k in range(1, nz):
        upper_fix[..., k] = upper_fix[..., k - 1]
    Q[..., kb] = upper_fix[..., kb]
    qvapor[I, J, :nz] = Q


def fix_neg_cloud(t: Tile, dp, qcld):
    """neg_adj3.py:148-173."""
    I, J, _ = _comp(t)
    nz = t.nz
    Q, D = qcld[I, J, :nz], dp[I, J, :nz]
    for k in range(1, nz - 1):
        m = Q[..., k - 1] < 0.0
        Q[..., k] = np.where(m, Q[..., k] + Q[..., k - 1] * D[..., k - 1] / D[..., k], Q[..., k])
    for k in range(1, nz - 1):
        Q[..., k] = np.where(Q[..., k] < 0.0, 0.0, Q[..., k])
    k = nz - 2
    m = (Q[..., k + 1] < 0.0) & (Q[..., k] > 0)
    dq = _sel(-Q[..., k] * D[..., k], Q[..., k + 1] * D[..., k + 1])
    Q[..., k] = np.where(m, Q[..., k] - dq / D[..., k], Q[..., k])
    k = nz - 1
    m = (Q[..., k] < 0) & (Q[..., k - 1] > 0.0)
    dq = _sel(-Q[..., k] * D[..., k], Q[..., k - 1] * D[..., k - 1])
    qn = Q[..., k] + dq / D[..., k]
    Q[..., k] = np.where(m, _pos(qn), Q[..., k])
    qcld[I, J, :nz] = Q


def adjust_negative_tracers(t: Tile, qvapor, qliquid, qrain, qsnow, qice, qgraupel, qcld, pt, delp, delz, peln,
                            hydrostatic=False):
    """AdjustNegativeTracerMixingRatio.__call__ (neg_adj3.py:293-372)."""
    if hydrostatic:
        raise NotImplementedError("Unimplemented namelist hydrostatic=True")
    d0_vap = C.CV_VAP - C.C_LIQ
    lv00 = C.HLV - d0_vap * C.TICE
    fix_neg_water(t, pt, delz, qvapor, qliquid, qrain, qsnow, qice, qgraupel, lv00, d0_vap)
    fillq(t, qgraupel, delp)
    fillq(t, qrain, delp)
    fix_water_vapor_down(t, qvapor, delp)
    fix_neg_cloud(t, delp, qcld)


# ------------------------------------------------------------ c2l_ord
C1, C2 = 1.125, -0.125


def cubed_to_latlon_ord4(t: Tile, u, v, dx, dy, a11, a12, a21, a22, ua, va):
    """ord4_transform (c2l_ord.py:38-72) on the compute domain; u, v must
    hold their halo rows (the vector halo update runs first)."""
    I, J, K = _comp(t)
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    dx, dy = c3(dx), c3(dy)
    utmp = C2 * (sh(u, 0, -1) + sh(u, 0, 2)) + C1 * (u + sh(u, 0, 1))
    vtmp = C2 * (sh(v, -1, 0) + sh(v, 2, 0)) + C1 * (v + sh(v, 1, 0))
    v_e = 2.0 * ((v * dy) + (sh(v, 1, 0) * sh(dy, 1, 0))) / (dy + sh(dy, 1, 0))
    u_e = 2.0 * (u * dx + sh(u, 0, 1) * sh(dx, 0, 1)) / (dx + sh(dx, 0, 1))
    u_w = 2.0 * ((u * dx) + (sh(u, 0, 1) * sh(dx, 0, 1))) / (dx + sh(dx, 0, 1))
    rows = np.zeros((t.m, t.m, 1), dtype=bool)
    rows[:, js] = rows[:, je] = True
    cols = np.zeros((t.m, t.m, 1), dtype=bool)
    cols[s, :] = cols[e, :] = True
    vtmp = np.where(rows, v_e, vtmp)
    utmp = np.where(rows, u_e, utmp)
    utmp = np.where(cols, u_w, utmp)
    vtmp = np.where(cols, v_e, vtmp)
    a11, a12, a21, a22 = (c3(a) for a in (a11, a12, a21, a22))
    ua[I, J, K] = (a11 * utmp + a12 * vtmp)[I, J, K]
    va[I, J, K] = (a21 * utmp + a22 * vtmp)[I, J, K]

"""LagrangianToEulerian, the vertical remapping of DynamicalCore.step_dynamics
(reference ``fv3core/stencils/remapping.py``, ``map_single.py``,
``remap_profile.py``, ``mapn_tracer.py``, ``fillz.py``, ``moist_cv.py``).

Test infrastructure: the oracle the CUDA remapping is checked against, not
part of the product.  One tile's storages ``[m, m, nk]``; every stencil
works on the box the reference builds it over (origin and domain of
remapping.py:205-414), with the levels of its domain.  Column algorithms run
level by level, vectorised over the box's columns, in the gt4py numpy
backend's order: FORWARD / BACKWARD levels one after another, the intervals
of a computation in the order they are written, a field ``if`` as a masked
assignment whose condition is evaluated before its body, and a ``while`` as
a masked loop that runs while its test holds at any column.  Expressions
keep the reference's association, so FP64 results agree with the reference
bit for bit; exp and log come from ``_math`` (numpy's, or the library's own
functions under ``device_math()``).
"""
import numpy as np

from fv3core_b200 import constants as C

from . import _math
from ._util import Tile


# the remapped tracers in the reference's order (utils.tracer_variables[0:8])
TRACERS = ("qvapor", "qliquid", "qrain", "qice", "qsnow", "qgraupel", "qo3mr", "qsgs_tke")


def _lt_sel(a, b):
    """``a if a < b else b``."""
    return np.where(a < b, a, b)


def _gt_sel(a, b):
    """``a if a > b else b``."""
    return np.where(a > b, a, b)


def _min3(a, p, lac):
    """``a if (a < p) and (a < lac) else p if p < lac else lac``
    (remap_profile.py:362-368)."""
    return np.where((a < p) & (a < lac), a, np.where(p < lac, p, lac))


def _max3(a, p, lac):
    """``a if (a > p) and (a > lac) else p if p > lac else lac``."""
    return np.where((a > p) & (a > lac), a, np.where(p > lac, p, lac))


# ------------------------------------------------------------ constraints
def _posdef_iv1(a1, a2, a3, a4):
    """posdef_constraint_iv1 (remap_profile.py:73-92) on level arrays."""
    da1 = a3 - a2
    da2 = da1 * da1
    a6da = a4 * da1
    c1 = ((a1 - a2) * (a1 - a3)) >= 0.0
    c2 = ~c1 & (a6da < -1.0 * da2)
    c3 = ~c1 & ~c2 & (a6da > da2)
    n2 = np.where(c1, a1, a2)
    n3 = np.where(c1, a1, a3)
    n4 = np.where(c1, 0.0, a4)
    t4 = 3.0 * (a2 - a1)
    n4 = np.where(c2, t4, n4)
    n3 = np.where(c2, a2 - t4, n3)
    u4 = 3.0 * (a3 - a1)
    n4 = np.where(c3, u4, n4)
    n2 = np.where(c3, a3 - u4, n2)
    return a1, n2, n3, n4


def _remap_constraint(a1, a2, a3, a4, extm):
    """remap_constraint (remap_profile.py:95-115)."""
    da1 = a3 - a2
    da2 = da1 * da1
    a6da = a4 * da1
    c1 = extm
    c2 = ~c1 & (a6da < -da2)
    c3 = ~c1 & ~c2 & (a6da > da2)
    n2 = np.where(c1, a1, a2)
    n3 = np.where(c1, a1, a3)
    n4 = np.where(c1, 0.0, a4)
    t4 = 3.0 * (a2 - a1)
    n4 = np.where(c2, t4, n4)
    n3 = np.where(c2, a2 - t4, n3)
    u4 = 3.0 * (a3 - a1)
    n4 = np.where(c3, u4, n4)
    n2 = np.where(c3, a3 - u4, n2)
    return a1, n2, n3, n4


def _posdef_iv0(a1, a2, a3, a4):
    """posdef_constraint_iv0 (remap_profile.py:44-70)."""
    c_neg = a1 <= 0.0
    n2 = np.where(c_neg, a1, a2)
    n3 = np.where(c_neg, a1, a3)
    n4 = np.where(c_neg, 0.0, a4)
    with np.errstate(all="ignore"):
        inner = (~c_neg & (np.abs(a3 - a2) < -a4)
                 & ((a1 + 0.25 * (a3 - a2) ** 2 / a4 + a4 * (1.0 / 12.0)) < 0.0))
    b1 = inner & (a1 < a3) & (a1 < a2)
    b2 = inner & ~b1 & (a3 > a2)
    b3 = inner & ~b1 & ~b2
    n3 = np.where(b1, a1, n3)
    n2 = np.where(b1, a1, n2)
    n4 = np.where(b1, 0.0, n4)
    t4 = 3.0 * (a2 - a1)
    n4 = np.where(b2, t4, n4)
    n3 = np.where(b2, a2 - t4, n3)
    u4 = 3.0 * (a3 - a1)
    n4 = np.where(b3, u4, n4)
    n2 = np.where(b3, a3 - u4, n2)
    return a1, n2, n3, n4


# ------------------------------------------------------------ cs_profile
def remap_profile(qs, a4_1, delp, iv, kord, qmin=0.0):
    """RemapProfile (remap_profile.py:495-638) on columns ``[..., km]``:
    ``a4_1`` holds the layer means, ``delp`` the layer thicknesses, ``qs``
    ``[...]`` the bottom value (read when iv == -2).  Returns the four
    coefficients a4_1..a4_4, each ``[..., km]``."""
    assert abs(kord) <= 10, kord
    kord = abs(kord)
    km = a4_1.shape[-1]
    shp = a4_1.shape[:-1]
    q = np.full(shp + (km + 1,), np.nan)
    gam = np.full(shp + (km + 1,), np.nan)
    a1 = a4_1
    dp = delp
    with np.errstate(all="ignore"):
        # set_initial_vals (remap_profile.py:118-214)
        if iv == -2:
            q[..., 0] = 1.5 * a1[..., 0]
            gam[..., 1] = 0.5
            gr = dp[..., 0] / dp[..., 1]
            bet = 2.0 + gr + gr - gam[..., 1]
            q[..., 1] = (3.0 * (a1[..., 0] + a1[..., 1]) - q[..., 0]) / bet
            grid_ratio = np.full(shp + (km + 1,), np.nan)
            for k in range(2, km):
                ogr = dp[..., k - 2] / dp[..., k - 1]
                obet = 2.0 + ogr + ogr - gam[..., k - 1]
                gam[..., k] = ogr / obet
                grid_ratio[..., k] = dp[..., k - 1] / dp[..., k]
            for k in range(2, km - 1):
                gr = grid_ratio[..., k]
                bet = 2.0 + gr + gr - gam[..., k]
                q[..., k] = (3.0 * (a1[..., k - 1] + a1[..., k]) - q[..., k - 1]) / bet
            k = km - 1
            gr = grid_ratio[..., k]
            q[..., k] = (3.0 * (a1[..., k - 1] + a1[..., k]) - gr * qs - q[..., k - 1]) / (2.0 + gr + gr - gam[..., k])
            q[..., km] = qs
            for k in range(km - 2, -1, -1):
                q[..., k] = q[..., k] - gam[..., k + 1] * q[..., k + 1]
        else:
            gr = dp[..., 1] / dp[..., 0]
            bet = gr * (gr + 0.5)
            q[..., 0] = ((gr + gr) * (gr + 1.0) * a1[..., 0] + a1[..., 1]) / bet
            gam[..., 0] = (1.0 + gr * (gr + 1.5)) / bet
            for k in range(1, km):
                d4 = dp[..., k - 1] / dp[..., k]
                bet = 2.0 + d4 + d4 - gam[..., k - 1]
                q[..., k] = (3.0 * (a1[..., k - 1] + d4 * a1[..., k]) - q[..., k - 1]) / bet
                gam[..., k] = d4 / bet
            d4 = dp[..., km - 2] / dp[..., km - 1]
            a_bot = 1.0 + d4 * (d4 + 1.5)
            q[..., km] = ((2.0 * d4 * (d4 + 1.0) * a1[..., km - 1] + a1[..., km - 2] - a_bot * q[..., km - 1])
                          / (d4 * (d4 + 0.5) - a_bot * gam[..., km - 1]))
            for k in range(km - 1, -1, -1):
                q[..., k] = q[..., k] - gam[..., k] * q[..., k + 1]

        # apply_constraints (remap_profile.py:217-295)
        a1p = np.concatenate([np.full(shp + (1,), np.nan), a1[..., :-1]], axis=-1)  # a4_1[k - 1]
        tmp = np.where(a1p > a1, a1p, a1)
        tmp2 = np.where(a1p < a1, a1p, a1)
        gam[..., 1:km] = (a1 - a1p)[..., 1:km]
        k = 1
        q[..., k] = np.where(q[..., k] >= tmp[..., k], tmp[..., k], q[..., k])
        q[..., k] = np.where(q[..., k] <= tmp2[..., k], tmp2[..., k], q[..., k])
        for k in range(2, km - 1):
            qk = q[..., k]
            both = (gam[..., k - 1] * gam[..., k + 1]) > 0
            lmax = ~both & (gam[..., k - 1] > 0)
            lmin = ~both & ~lmax
            # both sides
            qb = np.where(qk >= tmp[..., k], tmp[..., k], qk)
            qb = np.where(qb <= tmp2[..., k], tmp2[..., k], qb)
            # local maximum
            qx = np.where(qk <= tmp2[..., k], tmp2[..., k], qk)
            # local minimum
            qn = np.where(qk >= tmp[..., k], tmp[..., k], qk)
            if iv == 0:
                qn = np.where(qn < 0.0, 0.0, qn)
            q[..., k] = np.where(both, qb, np.where(lmax, qx, qn))
        k = km - 1
        q[..., k] = np.where(q[..., k] >= tmp[..., k], tmp[..., k], q[..., k])
        q[..., k] = np.where(q[..., k] <= tmp2[..., k], tmp2[..., k], q[..., k])
        a2 = q[..., :km].copy()
        a3 = q[..., 1:km + 1].copy()
        extm = np.zeros(shp + (km,), dtype=bool)
        extm[..., 0] = (a2[..., 0] - a1[..., 0]) * (a3[..., 0] - a1[..., 0]) > 0.0
        extm[..., 1:km - 1] = gam[..., 1:km - 1] * gam[..., 2:km] < 0.0
        extm[..., km - 1] = (a2[..., km - 1] - a1[..., km - 1]) * (a3[..., km - 1] - a1[..., km - 1]) > 0.0
        a4 = np.zeros(shp + (km,))  # the profile's a4_4 storage on entry (zeros)
        ext5 = np.zeros(shp + (km,), dtype=bool)
        ext6 = np.zeros(shp + (km,), dtype=bool)
        if kord > 9:
            x0 = 2.0 * a1 - (a2 + a3)
            x1 = np.abs(a2 - a3)
            a4 = 3.0 * x0
            ext5 = np.abs(x0) > x1
            ext6 = np.abs(a4) > x1

        # set_interpolation_coefficients (remap_profile.py:298-492)
        a1 = a1.copy()
        if iv == 0:
            a2[..., 0] = np.where(a2[..., 0] < 0.0, 0.0, a2[..., 0])
        elif iv == -1:
            a2[..., 0] = np.where(a2[..., 0] * a1[..., 0] <= 0.0, 0.0, a2[..., 0])
        if iv == 2:
            a2[..., 0] = a1[..., 0]
            a3[..., 0] = a1[..., 0]
            a4[..., 0] = 0.0
            a4[..., 1] = 3.0 * (2.0 * a1[..., 1] - (a2[..., 1] + a3[..., 1]))
        else:
            for k in (0, 1):
                a4[..., k] = 3.0 * (2.0 * a1[..., k] - (a2[..., k] + a3[..., k]))
        if iv != 2:
            _, a2[..., 0], a3[..., 0], a4[..., 0] = _posdef_iv1(a1[..., 0], a2[..., 0], a3[..., 0], a4[..., 0])
        _, a2[..., 1], a3[..., 1], a4[..., 1] = _remap_constraint(a1[..., 1], a2[..., 1], a3[..., 1], a4[..., 1],
                                                                  extm[..., 1])
        if km - 2 > 2:
            s = slice(2, km - 2)
            b1, b2, b3, b4 = a1[..., s], a2[..., s], a3[..., s], a4[..., s]
            g0 = gam[..., 2:km - 2]
            gp = gam[..., 3:km - 1]
            gp2 = gam[..., 4:km]
            gm = gam[..., 1:km - 3]
            em, e0, ep = extm[..., 1:km - 3], extm[..., 2:km - 2], extm[..., 3:km - 1]
            if kord < 9:
                pmp_1 = b1 - gp
                lac_1 = pmp_1 + 1.5 * gp2
                tmin = _min3(b1, pmp_1, lac_1)
                tmax0 = np.where(b2 > tmin, b2, tmin)
                tmax = _max3(b1, pmp_1, lac_1)
                b2 = np.where(tmax0 < tmax, tmax0, tmax)
                pmp_2 = b1 + 2.0 * gp
                lac_2 = pmp_2 - 1.5 * gm
                tmin = _min3(b1, pmp_2, lac_2)
                tmax0 = np.where(b3 > tmin, b3, tmin)
                tmax = _max3(b1, pmp_2, lac_2)
                b3 = np.where(tmax0 < tmax, tmax0, tmax)
                b4 = 3.0 * (2.0 * b1 - (b2 + b3))
            elif kord == 9:
                pmp_1 = b1 - 2.0 * gp
                lac_1 = pmp_1 + 1.5 * gp2
                pmp_2 = b1 + 2.0 * g0
                lac_2 = pmp_2 - 1.5 * gm
                flat = (e0 & em) | (e0 & ep) | (e0 & ((qmin > 0.0) & (b1 < qmin)))
                n2 = np.where(flat, b1, b2)
                n3 = np.where(flat, b1, b3)
                n4 = np.where(flat, 0.0, 6.0 * b1 - 3.0 * (b2 + b3))
                lim = ~flat & (np.abs(n4) > np.abs(n2 - n3))
                tmin = _min3(b1, pmp_1, lac_1)
                tmax0 = np.where(b2 > tmin, b2, tmin)
                tmax = _max3(b1, pmp_1, lac_1)
                l2 = np.where(tmax0 < tmax, tmax0, tmax)
                tmin = _min3(b1, pmp_2, lac_2)
                tmax0 = np.where(b3 > tmin, b3, tmin)
                tmax = _max3(b1, pmp_2, lac_2)
                l3 = np.where(tmax0 < tmax, tmax0, tmax)
                b2 = np.where(lim, l2, n2)
                b3 = np.where(lim, l3, n3)
                b4 = np.where(lim, 6.0 * b1 - 3.0 * (l2 + l3), n4)
            elif kord == 10:
                pmp_1 = b1 - 2.0 * gp
                lac_1 = pmp_1 + 1.5 * gp2
                pmp_2 = b1 + 2.0 * g0
                lac_2 = pmp_2 - 1.5 * gm
                tmin2 = _min3(b1, pmp_1, lac_1)
                tmax2 = _max3(b1, pmp_1, lac_1)
                t2 = np.where(b2 > tmin2, b2, tmin2)
                tmin3 = np.where(b1 < pmp_2, b1, pmp_2)
                tmin3 = np.where(lac_2 < tmin3, lac_2, tmin3)
                tmax3 = np.where(b1 > pmp_2, b1, pmp_2)
                tmax3 = np.where(lac_2 > tmax3, lac_2, tmax3)
                t3 = np.where(b3 > tmin3, b3, tmin3)
                e5, e5m, e5p = ext5[..., s], ext5[..., 1:km - 3], ext5[..., 3:km - 1]
                e6m, e6p = ext6[..., 1:km - 3], ext6[..., 3:km - 1]
                e6 = ext6[..., s]
                flat = e5 & (e5m | e5p)
                limit = (e5 & ~flat & (e6m | e6p)) | (~e5 & e6 & (e5m | e5p))
                lim2 = np.where(t2 < tmax2, t2, tmax2)
                lim3 = np.where(t3 < tmax3, t3, tmax3)
                b2 = np.where(flat, b1, np.where(limit, lim2, b2))
                b3 = np.where(flat, b1, np.where(limit, lim3, b3))
                b4 = 3.0 * (2.0 * b1 - (b2 + b3))
            if iv == 0:
                b1, b2, b3, b4 = _posdef_iv0(b1, b2, b3, b4)
            a2[..., s], a3[..., s], a4[..., s] = b2, b3, b4
        k = km - 1
        if iv == 0:
            a3[..., k] = np.where(a3[..., k] < 0.0, 0.0, a3[..., k])
        if iv == -1:
            a3[..., k] = np.where(a3[..., k] * a1[..., k] <= 0.0, 0.0, a3[..., k])
        for k in (km - 2, km - 1):
            a4[..., k] = 3.0 * (2.0 * a1[..., k] - (a2[..., k] + a3[..., k]))
        k = km - 2
        _, a2[..., k], a3[..., k], a4[..., k] = _remap_constraint(a1[..., k], a2[..., k], a3[..., k], a4[..., k],
                                                                  extm[..., k])
        k = km - 1
        _, a2[..., k], a3[..., k], a4[..., k] = _posdef_iv1(a1[..., k], a2[..., k], a3[..., k], a4[..., k])
    return a1, a2, a3, a4


def lagrangian_contributions(pe1, pe2, a1, a2, a3, a4, dp1):
    """lagrangian_contributions (map_single.py:19-66): the mean of the
    source profile over each target layer ``[pe2[k], pe2[k+1]]``; columns
    ``[..., km(+1)]``.  ``L`` is the absolute source level (the reference's
    relative offset ``lev`` plus k)."""
    km = a1.shape[-1]
    shp = a1.shape[:-1]
    out = np.empty(shp + (km,))
    L = np.zeros(shp, dtype=np.int64)
    take = lambda f, idx: np.take_along_axis(f, np.minimum(idx, f.shape[-1] - 1)[..., None], axis=-1)[..., 0]
    with np.errstate(all="ignore"):
        for k in range(km):
            p1 = take(pe1, L)
            d1 = take(dp1, L)
            pl = (pe2[..., k] - p1) / d1
            inside = pe2[..., k + 1] <= take(pe1, L + 1)
            q2, q3, q4 = take(a2, L), take(a3, L), take(a4, L)
            pr = (pe2[..., k + 1] - p1) / d1
            q_in = q2 + 0.5 * (q4 + q3 - q2) * (pr + pl) - q4 * 1.0 / 3.0 * (pr * (pr + pl) + pl * pl)
            # the layer reaches past the source layer: partial top piece, whole
            # layers, partial bottom piece
            qsum = (take(pe1, L + 1) - pe2[..., k]) * (q2 + 0.5 * (q4 + q3 - q2) * (1.0 + pl)
                                                      - q4 * 1.0 / 3.0 * (1.0 + pl * (1.0 + pl)))
            Lx = np.where(inside, L, L + 1)
            for _ in range(km + 1):
                go = ~inside & (take(pe1, Lx + 1) < pe2[..., k + 1])
                if not go.any():
                    break
                qsum = np.where(go, qsum + take(dp1, Lx) * take(a1, Lx), qsum)
                Lx = np.where(go, Lx + 1, Lx)
            dp = pe2[..., k + 1] - take(pe1, Lx)
            esl = dp / take(dp1, Lx)
            qsum = qsum + dp * (take(a2, Lx) + 0.5 * esl * (take(a3, Lx) - take(a2, Lx)
                                                            + take(a4, Lx) * (1.0 - (2.0 / 3.0) * esl)))
            q_out = qsum / (pe2[..., k + 1] - pe2[..., k])
            out[..., k] = np.where(inside, q_in, q_out)
            L = Lx
    return out


def map_single(q1, pe1, pe2, box, kord, iv, qs=None, qmin=0.0):
    """MapSingle.__call__ (map_single.py:130-173) in place on the box
    ``(i0, i1, j0, j1)`` of one tile's storages, over the npz layers."""
    i0, i1, j0, j1 = box
    km = q1.shape[2] - 1
    B = (slice(i0, i1), slice(j0, j1))
    p1 = pe1[B][..., :km + 1]
    p2 = pe2[B][..., :km + 1]
    a1 = q1[B][..., :km].copy()
    with np.errstate(all="ignore"):
        dp1 = p1[..., 1:] - p1[..., :-1]
    qsv = np.zeros(a1.shape[:-1]) if qs is None else qs[B]
    c1, c2, c3, c4 = remap_profile(qsv, a1, dp1, iv, kord, qmin)
    q1[B + (slice(0, km),)] = lagrangian_contributions(p1, p2, c1, c2, c3, c4, dp1)


def fix_tracer(q, dp, box, dm, dm_pos):
    """fix_tracer (fillz.py:10-98) in place on the box, npz layers; ``dm``
    and ``dm_pos`` are the filler's storages (kept between tracers)."""
    i0, i1, j0, j1 = box
    km = q.shape[2] - 1
    B = (slice(i0, i1), slice(j0, j1))
    Q = q[B]  # views
    D = dp[B]
    DM = dm[B]
    DP = dm_pos[B]
    shp = Q.shape[:2]
    zfix = np.zeros(shp, dtype=np.int64)
    sum0 = np.zeros(shp)
    sum1 = np.zeros(shp)
    lower_fix = np.zeros(shp + (km,))
    upper_fix = np.zeros(shp + (km,))
    with np.errstate(all="ignore"):
        # fix_top
        Q[..., 0] = np.where(Q[..., 0] < 0, 0, Q[..., 0])
        DM[..., 0] = Q[..., 0] * D[..., 0]
        c = Q[..., 0] < 0.0
        Q[..., 1] = np.where(c, Q[..., 1] + Q[..., 0] * D[..., 0] / D[..., 1], Q[..., 1])
        # fix_interior
        for k in range(1, km - 1):
            c = lower_fix[..., k - 1] != 0.0
            Q[..., k] = np.where(c, Q[..., k] - (lower_fix[..., k - 1] / D[..., k]), Q[..., k])
            neg = Q[..., k] < 0.0
            zfix = np.where(neg, zfix + 1, zfix)
            up = neg & (Q[..., k - 1] > 0.0)
            a = Q[..., k - 1] * D[..., k - 1]
            b = -(Q[..., k] * D[..., k])
            dq = np.where(a < b, a, b)
            Q[..., k] = np.where(up, Q[..., k] + dq / D[..., k], Q[..., k])
            upper_fix[..., k] = np.where(up, dq, upper_fix[..., k])
            down = neg & (Q[..., k] < 0.0) & (Q[..., k + 1] > 0.0)
            a = Q[..., k + 1] * D[..., k + 1]
            b = -(Q[..., k] * D[..., k])
            dq = np.where(a < b, a, b)
            Q[..., k] = np.where(down, Q[..., k] + dq / D[..., k], Q[..., k])
            lower_fix[..., k] = np.where(down, dq, lower_fix[..., k])
        for k in range(0, km - 1):
            c = upper_fix[..., k + 1] != 0.0
            Q[..., k] = np.where(c, Q[..., k] - upper_fix[..., k + 1] / D[..., k], Q[..., k])
            DM[..., k] = Q[..., k] * D[..., k]
            DP[..., k] = np.where(DM[..., k] > 0.0, DM[..., k], 0.0)
        # fix_bottom
        k = km - 1
        c = lower_fix[..., k - 1] != 0.0
        Q[..., k] = np.where(c, Q[..., k] - (lower_fix[..., k - 1] / D[..., k]), Q[..., k])
        qup = Q[..., k - 1] * D[..., k - 1]
        qly = -Q[..., k] * D[..., k]
        dup = np.where(qup < qly, qup, qly)
        c = (Q[..., k] < 0.0) & (Q[..., k - 1] > 0.0)
        zfix = np.where(c, zfix + 1, zfix)
        Q[..., k] = np.where(c, Q[..., k] + (dup / D[..., k]), Q[..., k])
        upper_fix[..., k] = np.where(c, dup, upper_fix[..., k])
        DM[..., k] = Q[..., k] * D[..., k]
        DP[..., k] = np.where(DM[..., k] > 0.0, DM[..., k], 0.0)
        k = km - 2
        c = upper_fix[..., k + 1] != 0.0
        Q[..., k] = np.where(c, Q[..., k] - (upper_fix[..., k + 1] / D[..., k]), Q[..., k])
        DM[..., k] = np.where(c, Q[..., k] * D[..., k], DM[..., k])
        DP[..., k] = np.where(c, np.where(DM[..., k] > 0.0, DM[..., k], 0.0), DP[..., k])
        for k in range(1, km):
            sum0 = sum0 + DM[..., k]
            sum1 = sum1 + DP[..., k]
        # final_check
        fac = np.where(sum0 > 0.0, sum0 / sum1, 0.0)
        fix = (zfix > 0) & (fac > 0.0)
        for k in range(1, km):
            v = fac * DM[..., k] / D[..., k]
            Q[..., k] = np.where(fix, np.where(v > 0.0, v, 0.0), Q[..., k])


# ------------------------------------------------------------ the step
def _moist_cv_nwat6(qv, ql_, qr, qs_, qi, qg):
    """moist_cv_nwat6_fn and moist_cvm (moist_cv.py:14-39): (cvm, gz)."""
    ql = ql_ + qr
    qs = qi + qs_ + qg
    gz = ql + qs
    cvm = (1.0 - (qv + gz)) * C.CV_AIR + qv * C.CV_VAP + ql * C.C_LIQ + qs * C.C_ICE
    return cvm, gz


def _set_cappa(qv, cvm, r_vir):
    """set_cappa (moist_cv.py:8-11)."""
    return C.RDGAS / (C.RDGAS + cvm / (1.0 + r_vir * qv))


def kmp_of(pfull, npz):
    """The saturation adjustment's top level (remapping.py:396-400): the
    first level whose reference pressure exceeds 10 hPa."""
    for k in range(len(pfull)):
        if pfull[k] > 10.0e2:
            return k
    return npz - 1


def lagrangian_to_eulerian(t: Tile, tracers, st, ak, bk, ptop, akap, zvir, last_step, kord_tm=-9, kord_tr=9,
                           kord_wz=9, kord_mt=9, fill=True, sat_adjust=None):
    """LagrangianToEulerian.__call__ (remapping.py:416-628) on one tile,
    without the saturation adjustment (do_sat_adj False).  ``tracers`` maps
    the eight remapped tracer names, in the reference's order
    (qvapor, qliquid, qrain, qice, qsnow, qgraupel, qo3mr, qsgs_tke), to
    their storages; ``st`` holds pt, delp, delz, peln, u, v, w, ua, va,
    cappa, q_con, pkz, pk, pe, ps (2-D) and wsd (2-D).  Every field is
    updated in place.  ``sat_adjust`` (do_sat_adj): a dict with the
    SatAdjustConfig values (``cfg``), ``area``, ``hs`` (2-D), ``dp1``,
    ``qcld``, ``pfull`` and ``mdt``; the adjustment then runs after the
    remaps (remapping.py:570-589), with no total-energy fixer (consv_te 0)."""
    nz = t.nz
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    pe = st["pe"]
    m = t.m
    pe1 = np.zeros((m, m, nz + 1))
    pe2 = np.zeros((m, m, nz + 1))
    dp2 = np.zeros((m, m, nz + 1))
    pn2 = np.zeros((m, m, nz + 1))
    pe0 = np.zeros((m, m, nz + 1))
    pe3 = np.zeros((m, m, nz + 1))
    gz = np.zeros((m, m, nz + 1))
    cvm = np.zeros((m, m, nz + 1))
    ak = np.asarray(ak, dtype=np.float64)
    bk = np.asarray(bk, dtype=np.float64)
    I = slice(s, e + 1)
    J = slice(js, je + 1)
    Jx = slice(js, je + 2)
    K = slice(0, nz)
    q = tracers
    with np.errstate(all="ignore"):
        # init_pe (remapping.py:33-40) on [is, ie] x [js, je+1], levels 0..npz
        pe2[I, Jx, 0] = ptop
        pe2[I, Jx, nz] = pe[I, Jx, nz]
        pe1[I, Jx, :] = pe[I, Jx, :]
        # moist_cv_pt_pressure (57-120) on the compute domain, levels 0..npz
        pt, delp, delz, peln = st["pt"], st["delp"], st["delz"], st["peln"]
        cv, g = _moist_cv_nwat6(q["qvapor"][I, J, K], q["qliquid"][I, J, K], q["qrain"][I, J, K],
                                q["qsnow"][I, J, K], q["qice"][I, J, K], q["qgraupel"][I, J, K])
        cvm[I, J, K] = cv
        gz[I, J, K] = g
        st["q_con"][I, J, K] = g
        ca = _set_cappa(q["qvapor"][I, J, K], cv, zvir)
        st["cappa"][I, J, K] = ca
        pt[I, J, K] = pt[I, J, K] * _math.exp(ca / (1.0 - ca) * _math.log(C.RDG * delp[I, J, K] / delz[I, J, K]
                                                                           * pt[I, J, K]))
        delz[I, J, K] = -delz[I, J, K] / delp[I, J, K]
        st["ps"][I, J] = pe[I, J, nz]
        pn2[I, J, 0] = peln[I, J, 0]
        pe2[I, J, 1:nz] = ak[None, None, 1:nz] + bk[None, None, 1:nz] * st["ps"][I, J][..., None]
        pn2[I, J, nz] = peln[I, J, nz]
        dp2[I, J, K] = pe2[I, J, 1:nz + 1] - pe2[I, J, 0:nz]
        delp[I, J, K] = dp2[I, J, K]
        # pn2_pk_delp (123-134)
        delp[I, J, K] = dp2[I, J, K]
        pn2[I, J, K] = _math.log(pe2[I, J, K])
        st["pk"][I, J, K] = _math.exp(akap * pn2[I, J, K])
        # pt in log pressure (kord_tm, iv = 1, qmin 184 K)
        box = (s, e + 1, js, je + 1)
        map_single(pt, peln, pn2, box, abs(kord_tm), 1, qmin=184.0)
        # tracers (mapn_tracer.py:10-83): kord_tr, the sixth with kord 9
        names = [name for name in TRACERS if name in q]
        for n_, name in enumerate(names):
            map_single(q[name], pe1, pe2, box, 9 if n_ == 5 else abs(kord_tr), 0)
        if fill:
            dm = np.zeros((m + 1, m + 1, nz + 2))
            dm_pos = np.zeros((m + 1, m + 1, nz + 2))
            for name in names:
                fix_tracer(q[name][..., :nz + 1], dp2, box, dm, dm_pos)
        map_single(st["w"], pe1, pe2, box, kord_wz, -2, qs=st["wsd"])
        map_single(delz, pe1, pe2, box, kord_wz, 1)
        # undo_delz_adjust_and_copy_peln (43-54)
        delz[I, J, K] = -delz[I, J, K] * delp[I, J, K]
        pe0[I, J, :] = peln[I, J, :]
        peln[I, J, :] = pn2[I, J, :]
        # moist_cv_pkz (moist_cv.py:171-194)
        cv, g = _moist_cv_nwat6(q["qvapor"][I, J, K], q["qliquid"][I, J, K], q["qrain"][I, J, K],
                                q["qsnow"][I, J, K], q["qice"][I, J, K], q["qgraupel"][I, J, K])
        cvm[I, J, K] = cv
        gz[I, J, K] = g
        st["q_con"][I, J, K] = g
        ca = _set_cappa(q["qvapor"][I, J, K], cv, zvir)
        st["cappa"][I, J, K] = ca
        st["pkz"][I, J, K] = _math.exp(ca * _math.log(C.RDG * delp[I, J, K] / delz[I, J, K] * pt[I, J, K]))
        # pressures_mapu (137-159) on [is, ie] x [js, je+1]
        pbot = pe[:, :, nz]
        pe0[I, Jx, 0] = pe[I, Jx, 0]
        pe0[I, Jx, 1:nz + 1] = 0.5 * (pe[I, slice(js - 1, je + 1), 1:nz + 1] + pe1[I, Jx, 1:nz + 1])
        bkh = 0.5 * bk
        pe3[I, Jx, :] = ak[None, None, :] + bkh[None, None, :] * (pbot[I, slice(js - 1, je + 1)][..., None]
                                                                  + pbot[I, Jx][..., None])
        map_single(st["u"], pe0, pe3, (s, e + 1, js, je + 2), kord_mt, -1)
        # pressures_mapv (162-177) on [is, ie+1] x [js, je]
        Ix = slice(s, e + 2)
        Im = slice(s - 1, e + 1)
        pe3[Ix, J, 0] = ak[0]
        pe0[Ix, J, 0] = pe[Ix, J, 0]
        pe0[Ix, J, 1:nz + 1] = 0.5 * (pe[Im, J, 1:nz + 1] + pe[Ix, J, 1:nz + 1])
        pe3[Ix, J, 1:nz + 1] = ak[None, None, 1:] + bkh[None, None, 1:] * (pbot[Im, J][..., None]
                                                                            + pbot[Ix, J][..., None])
        map_single(st["v"], pe0, pe3, (s, e + 2, js, je + 1), kord_mt, -1)
        # update_ua (180-191) on [is, ie] x [js, je+1], npz layers
        ua = st["ua"]
        ua[I, Jx, K] = pe2[I, Jx, 1:nz + 1]
        ua[I, je + 1, 0:nz - 1] = pe2[I, je, 1:nz]
        # copy_from_below (194-196): pe[k] = ua[k - 1] on the compute domain
        pe[I, J, 1:nz] = ua[I, J, 0:nz - 1]
        if sat_adjust is not None:
            from .sat_adjust import sat_adjust_3d

            sa = sat_adjust
            fields = {"te": sa["dp1"], "qvapor": q["qvapor"], "qliquid": q["qliquid"], "qice": q["qice"],
                      "qrain": q["qrain"], "qsnow": q["qsnow"], "qgraupel": q["qgraupel"], "qcld": sa["qcld"],
                      "peln": peln, "delp": delp, "delz": delz, "q_con": st["q_con"], "pt": pt, "pkz": st["pkz"],
                      "cappa": st["cappa"]}
            sat_adjust_3d(t, fields, sa["cfg"], sa["area"], sa["hs"], zvir, sa["mdt"], False, last_step,
                          kmp_of(sa["pfull"], nz))
        if last_step:
            # moist_pt_last_step (moist_cv.py:139-162), dtmp = 0, levels 0..npz
            Kx = slice(0, nz + 1)
            g = (q["qliquid"][I, J, Kx] + q["qrain"][I, J, Kx] + q["qice"][I, J, Kx] + q["qsnow"][I, J, Kx]
                 + q["qgraupel"][I, J, Kx])
            gz[I, J, Kx] = g
            dtmp = 0.0
            pt[I, J, Kx] = (pt[I, J, Kx] + dtmp * st["pkz"][I, J, Kx]) / ((1.0 + zvir * q["qvapor"][I, J, Kx])
                                                                          * (1.0 - g))
        else:
            # adjust_divide_stencil (basic_operations.py:28-30)
            pt[I, J, K] = pt[I, J, K] / st["pkz"][I, J, K]

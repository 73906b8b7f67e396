"""Vertically implicit w / pressure solver (reference
``fv3core/stencils/sim1_solver.py:11-101``), restated column-wise in numpy.

All arguments are 3-D arrays over a box of columns (i, j) and interface
levels 0..nk-1 (``nk = npz + 1``); ``wsr`` is 2-D.  ``w``, ``pe`` and ``dz``
are updated in place, exactly over the box.
"""
import numpy as np

from fv3core_b200 import constants as C

from . import _math


def sim1_solver(w, dm, gm, dz, ptr, pm, pe, pem, wsr, cp3, dt, t1g, rdt, p_fac, nk):
    """Arrays are views [ni, nj, >=nk]; level nk-1 is the bottom interface."""
    K = nk
    sl = slice(0, K - 1)
    # PARALLEL interval(0, -1): pe, w1 (sim1_solver.py:27-29)
    pe[:, :, sl] = _math.exp(gm[:, :, sl] * _math.log(-dm[:, :, sl] / dz[:, :, sl] * C.RDGAS * ptr[:, :, sl])) - pm[:, :, sl]
    w1 = w.copy()
    shp = w.shape[:2] + (K,)
    g_rat = np.full(shp, np.nan)
    bb = np.full(shp, np.nan)
    dd = np.full(shp, np.nan)
    # FORWARD (sim1_solver.py:30-38)
    g_rat[:, :, : K - 2] = dm[:, :, : K - 2] / dm[:, :, 1 : K - 1]
    bb[:, :, : K - 2] = 2.0 * (1.0 + g_rat[:, :, : K - 2])
    dd[:, :, : K - 2] = 3.0 * (pe[:, :, : K - 2] + g_rat[:, :, : K - 2] * pe[:, :, 1 : K - 1])
    bb[:, :, K - 2] = 2.0
    dd[:, :, K - 2] = 3.0 * pe[:, :, K - 2]
    bet = np.full(shp, np.nan)
    bet[:, :, 0] = bb[:, :, 0]
    for k in range(1, K - 1):
        bet[:, :, k] = bet[:, :, k - 1]
    pp = np.full(shp, np.nan)
    pp[:, :, 0] = 0.0
    pp[:, :, 1] = dd[:, :, 0] / bet[:, :, 1]
    gam = np.full(shp, np.nan)
    # FORWARD interval(1, -1): gam, bet (sim1_solver.py:55-57)
    for k in range(1, K - 1):
        gam[:, :, k] = g_rat[:, :, k - 1] / bet[:, :, k - 1]
        bet[:, :, k] = bb[:, :, k] - gam[:, :, k]
    # FORWARD interval(2, None): pp (sim1_solver.py:58-59)
    for k in range(2, K):
        pp[:, :, k] = (dd[:, :, k - 1] - pp[:, :, k - 1]) / bet[:, :, k - 1]
    # BACKWARD interval(1, -1): pp, aa (sim1_solver.py:60-63)
    aa = np.full(shp, np.nan)
    for k in range(K - 2, 0, -1):
        pp[:, :, k] = pp[:, :, k] - gam[:, :, k] * pp[:, :, k + 1]
        aa[:, :, k] = t1g * 0.5 * (gm[:, :, k - 1] + gm[:, :, k]) / (dz[:, :, k - 1] + dz[:, :, k]) * (pem[:, :, k] + pp[:, :, k])
    # FORWARD: bet (sim1_solver.py:66-70)
    bet[:, :, 0] = dm[:, :, 0] - aa[:, :, 1]
    for k in range(1, K):
        bet[:, :, k] = bet[:, :, k - 1]
    # FORWARD: w (sim1_solver.py:72-88)
    w[:, :, 0] = (dm[:, :, 0] * w1[:, :, 0] + dt * pp[:, :, 1]) / bet[:, :, 0]
    for k in range(1, K - 2):
        gam[:, :, k] = aa[:, :, k] / bet[:, :, k - 1]
        bet[:, :, k] = dm[:, :, k] - (aa[:, :, k] + aa[:, :, k + 1] + aa[:, :, k] * gam[:, :, k])
        w[:, :, k] = (dm[:, :, k] * w1[:, :, k] + dt * (pp[:, :, k + 1] - pp[:, :, k]) - aa[:, :, k] * w[:, :, k - 1]) / bet[:, :, k]
    k = K - 2
    p1 = np.full(shp, np.nan)
    p1[:, :, k] = t1g * gm[:, :, k] / dz[:, :, k] * (pem[:, :, k + 1] + pp[:, :, k + 1])
    gam[:, :, k] = aa[:, :, k] / bet[:, :, k - 1]
    bet[:, :, k] = dm[:, :, k] - (aa[:, :, k] + p1[:, :, k] + aa[:, :, k] * gam[:, :, k])
    w[:, :, k] = (
        dm[:, :, k] * w1[:, :, k] + dt * (pp[:, :, k + 1] - pp[:, :, k]) - p1[:, :, k] * wsr - aa[:, :, k] * w[:, :, k - 1]
    ) / bet[:, :, k]
    # BACKWARD interval(0, -2) (sim1_solver.py:89-90)
    for k in range(K - 3, -1, -1):
        w[:, :, k] = w[:, :, k] - gam[:, :, k + 1] * w[:, :, k + 1]
    # FORWARD: pe (sim1_solver.py:91-95)
    pe[:, :, 0] = 0.0
    for k in range(1, K):
        pe[:, :, k] = pe[:, :, k - 1] + dm[:, :, k - 1] * (w[:, :, k - 1] - w1[:, :, k - 1]) * rdt
    # BACKWARD: p1 (sim1_solver.py:96-102)
    k = K - 2
    p1[:, :, k] = (pe[:, :, k] + 2.0 * pe[:, :, k + 1]) * 1.0 / 3.0
    for k in range(K - 3, -1, -1):
        p1[:, :, k] = (pe[:, :, k] + bb[:, :, k] * pe[:, :, k + 1] + g_rat[:, :, k] * pe[:, :, k + 2]) * 1.0 / 3.0 - g_rat[:, :, k] * p1[:, :, k + 1]
    # PARALLEL interval(0, -1): dz (sim1_solver.py:103-105)
    s = slice(0, K - 1)
    maxp = np.where(p_fac * dm[:, :, s] > p1[:, :, s] + pm[:, :, s], p_fac * pm[:, :, s], p1[:, :, s] + pm[:, :, s])
    dz[:, :, s] = -dm[:, :, s] * C.RDGAS * ptr[:, :, s] * _math.exp((cp3[:, :, s] - 1.0) * _math.log(maxp))

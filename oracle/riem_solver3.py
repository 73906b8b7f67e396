"""D-grid Riemann solver (reference ``fv3core/stencils/riem_solver3.py``,
``RiemannSolver3.__call__`` 145-242): precompute (24-67), Sim1 solve,
finalize (70-103) over the compute-domain columns and interface levels
0..npz.  Updates zh, pe, ppe, pk3, w, delz and, on the last call, peln and pk.
"""
import math

import numpy as np

from fv3core_b200 import constants as C

from . import _math
from .sim1 import sim1_solver


def riem_solver3(last_call, dt, cappa, ptop, zs, wsd, delz, q_con, delp, pt, zh, pe, ppe, pk3, pk, peln, w,
                 p_fac, n, nz, h=3, beta=0.0, use_logp=False):
    if use_logp:
        raise NotImplementedError("use_logp")
    I = slice(h, h + n)
    J = slice(h, h + n)
    K = nz + 1
    box = (I, J, slice(0, K))
    peln1 = math.log(ptop)
    ptk = math.exp(C.KAPPA * peln1)
    dm = delp[box].copy()
    pe_init = pe[box].copy()
    qc = q_con[box]
    shp = dm.shape
    pem = np.empty(shp)
    peln_run = np.empty(shp)
    peg = np.empty(shp)
    pelng = np.empty(shp)
    pem[:, :, 0] = ptop
    peln_run[:, :, 0] = peln1
    pk3[I, J, 0] = ptk
    peg[:, :, 0] = ptop
    pelng[:, :, 0] = peln1
    for k in range(1, K):
        pem[:, :, k] = pem[:, :, k - 1] + dm[:, :, k - 1]
        peln_run[:, :, k] = _math.log(pem[:, :, k])
        peg[:, :, k] = peg[:, :, k - 1] + dm[:, :, k - 1] * (1.0 - qc[:, :, k - 1])
        pelng[:, :, k] = _math.log(peg[:, :, k])
        pk3[I, J, k] = _math.exp(C.KAPPA * peln_run[:, :, k])
    gm = 1.0 / (1.0 - cappa[box])
    dm = dm * C.RGRAV
    pm = np.full(shp, np.nan)
    pm[:, :, : K - 1] = (peg[:, :, 1:] - peg[:, :, :-1]) / (pelng[:, :, 1:] - pelng[:, :, :-1])
    dz = delz[box]  # view: the solver updates delz in place
    z = zh[box]
    dz[:, :, : K - 1] = z[:, :, 1:] - z[:, :, :-1]
    t1g = 2.0 * dt * dt
    rdt = 1.0 / dt
    wv = w[box]
    pev = pe[box]
    sim1_solver(wv, dm, gm, dz, pt[box], pm, pev, pem, wsd[I, J], cappa[box], dt, t1g, rdt, p_fac, K)
    # finalize
    if beta < -0.1:
        ppe[box] = pe[box] + pem
    else:
        ppe[box] = pe[box]
    if last_call:
        peln[box] = peln_run
        pk[box] = pk3[box]
        pe[box] = pem
    else:
        pe[box] = pe_init
    zh[I, J, K - 1] = zs[I, J]
    for k in range(K - 2, -1, -1):
        zh[I, J, k] = zh[I, J, k + 1] - delz[I, J, k]

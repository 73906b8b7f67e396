"""C-grid Riemann solver (reference ``fv3core/stencils/riem_solver_c.py``).

``riem_solver_c`` restates ``RiemannSolverC.__call__`` (riem_solver_c.py:106-165):
``precompute`` (13-44), ``Sim1Solver`` (sim1_solver.py:11-101) and
``finalize`` (46-64) over columns is-1..ie+1, js-1..je+1 and interface levels
0..npz.  It updates ``gz`` and ``pef`` in place; ``w3`` is read only (the
reference solves w into a scratch array that it does not copy back).
"""
import numpy as np

from fv3core_b200 import constants as C

from . import _math
from .sim1 import sim1_solver


def riem_solver_c(dt2, cappa, ptop, hs, ws, ptc, q_con, delpc, gz, pef, w3, p_fac, n, nz, h=3):
    I = slice(h - 1, h + n + 1)
    J = slice(h - 1, h + n + 1)
    K = nz + 1
    box = (I, J, slice(0, K))
    # precompute (riem_solver_c.py:13-44)
    dm = delpc[box].copy()
    w = w3[box].copy()
    qc = q_con[box]
    pem = np.empty_like(dm)
    peg = np.empty_like(dm)
    pem[:, :, 0] = ptop
    peg[:, :, 0] = ptop
    for k in range(1, K):
        pem[:, :, k] = pem[:, :, k - 1] + dm[:, :, k - 1]
        peg[:, :, k] = peg[:, :, k - 1] + dm[:, :, k - 1] * (1.0 - qc[:, :, k - 1])
    dz = np.full_like(dm, np.nan)
    g = gz[box]
    dz[:, :, : K - 1] = g[:, :, 1:K] - g[:, :, : K - 1]
    gm = 1.0 / (1.0 - cappa[box])
    dm = dm / C.GRAV
    pm = np.full_like(dm, np.nan)
    pm[:, :, : K - 1] = (peg[:, :, 1:K] - peg[:, :, : K - 1]) / _math.log(peg[:, :, 1:K] / peg[:, :, : K - 1])
    # sim1 (riem_solver_c.py:152-164 -> sim1_solver.py)
    t1g = 2.0 * dt2 * dt2
    rdt = 1.0 / dt2
    pe = np.full_like(dm, np.nan)
    sim1_solver(w, dm, gm, dz, ptc[box], pm, pe, pem, ws[I, J], cappa[box], dt2, t1g, rdt, p_fac, K)
    # finalize (riem_solver_c.py:46-64)
    pef[I, J, 0] = ptop
    pef[I, J, 1:K] = pe[:, :, 1:K] + pem[:, :, 1:K]
    gz[I, J, K - 1] = hs[I, J]
    for k in range(K - 2, -1, -1):
        gz[I, J, k] = gz[I, J, k + 1] - dz[:, :, k] * C.GRAV

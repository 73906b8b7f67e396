"""PyTorch-ops references of the two vertically implicit solvers' column
work (test infrastructure): Sim1Solver (sim1_solver.py:11-105) with the
precompute of RiemannSolver3 (riem_solver3.py:24-67) and of RiemannSolverC
(riem_solver_c.py:13-64), written with differentiable torch operations, so
that torch autograd gives the reference gradients for the hand-written
adjoints.

Columns are rows of [ncol, K] tensors (K = npz + 1 interface levels; the
layer fields use the first K - 1 entries).
"""
import math

import torch

RDGAS = 287.05
GRAV = 9.80665
RGRAV = 1.0 / GRAV


def _sim1(DM, DZ, GM, PT, CP3, W1, pem, pm, wsr, dt, p_fac):
    """Sim1Solver on [ncol, N] layer tensors (pem on N + 1 interfaces):
    returns (new w, pe perturbation on interfaces as a list, new dz)."""
    ncol, N = DM.shape
    dtype = DM.dtype
    pe1 = torch.exp(GM * torch.log(-DM / DZ * RDGAS * PT)) - pm
    g_rat = DM[:, :-1] / DM[:, 1:]
    bb = [2.0 * (1.0 + g_rat[:, k]) for k in range(N - 1)] + [torch.full((ncol,), 2.0, dtype=dtype)]
    dd = [3.0 * (pe1[:, k] + g_rat[:, k] * pe1[:, k + 1]) for k in range(N - 1)] + [3.0 * pe1[:, N - 1]]
    bet = [bb[0]]
    gam = [None]
    for k in range(1, N):
        gam.append(g_rat[:, k - 1] / bet[k - 1])
        bet.append(bb[k] - gam[k])
    pp = [torch.zeros(ncol, dtype=dtype), dd[0] / bet[0]]
    for k in range(2, N + 1):
        pp.append((dd[k - 1] - pp[k - 1]) / bet[k - 1])
    for k in range(N - 1, 0, -1):
        pp[k] = pp[k] - gam[k] * pp[k + 1]
    t1g = 2.0 * dt * dt
    rdt = 1.0 / dt
    aa = [None] + [t1g * 0.5 * (GM[:, k - 1] + GM[:, k]) / (DZ[:, k - 1] + DZ[:, k]) * (pem[:, k] + pp[k])
                   for k in range(1, N)]
    betw = [DM[:, 0] - aa[1]]
    wv = [(DM[:, 0] * W1[:, 0] + dt * pp[1]) / betw[0]]
    gw = [None]
    for k in range(1, N - 1):
        gw.append(aa[k] / betw[k - 1])
        betw.append(DM[:, k] - (aa[k] + aa[k + 1] + aa[k] * gw[k]))
        wv.append((DM[:, k] * W1[:, k] + dt * (pp[k + 1] - pp[k]) - aa[k] * wv[k - 1]) / betw[k])
    k = N - 1
    p1t = t1g * GM[:, k] / DZ[:, k] * (pem[:, k + 1] + pp[k + 1])
    gw.append(aa[k] / betw[k - 1])
    betw.append(DM[:, k] - (aa[k] + p1t + aa[k] * gw[k]))
    wv.append((DM[:, k] * W1[:, k] + dt * (pp[k + 1] - pp[k]) - p1t * wsr - aa[k] * wv[k - 1]) / betw[k])
    for k in range(N - 2, -1, -1):
        wv[k] = wv[k] - gw[k + 1] * wv[k + 1]
    pe = [torch.zeros(ncol, dtype=dtype)]
    for k in range(1, N + 1):
        pe.append(pe[k - 1] + DM[:, k - 1] * (wv[k - 1] - W1[:, k - 1]) * rdt)
    p1 = [None] * N
    p1[N - 1] = (pe[N - 1] + 2.0 * pe[N]) * 1.0 / 3.0
    for k in range(N - 2, -1, -1):
        p1[k] = (pe[k] + bb[k] * pe[k + 1] + g_rat[:, k] * pe[k + 2]) * 1.0 / 3.0 - g_rat[:, k] * p1[k + 1]
    dz = []
    for k in range(N):
        maxp = torch.where(p_fac * DM[:, k] > p1[k] + pm[:, k], p_fac * pm[:, k], p1[k] + pm[:, k])
        dz.append(-DM[:, k] * RDGAS * PT[:, k] * torch.exp((CP3[:, k] - 1.0) * torch.log(maxp)))
    return torch.stack(wv, dim=1), pe, torch.stack(dz, dim=1)


def _column_sums(dp, q_con, ptop):
    ncol = dp.shape[0]
    zeros = torch.zeros(ncol, 1, dtype=dp.dtype)
    pem = torch.cat([zeros + ptop, ptop + torch.cumsum(dp, dim=1)], dim=1)
    peg = torch.cat([zeros + ptop, ptop + torch.cumsum(dp * (1.0 - q_con), dim=1)], dim=1)
    return pem, peg


def riem3_columns(w, zh, delp, pt, cappa, q_con, wsr, dt, ptop, p_fac):
    """RiemannSolver3 (riem_solver3.py:24-67 + sim1): new (w, delz)."""
    N = zh.shape[1] - 1
    dp = delp[:, :N]
    pem, peg = _column_sums(dp, q_con[:, :N], ptop)
    ncol = zh.shape[0]
    lg = torch.cat([torch.zeros(ncol, 1, dtype=zh.dtype) + math.log(ptop), torch.log(peg[:, 1:])], dim=1)
    pm = (peg[:, 1:] - peg[:, :-1]) / (lg[:, 1:] - lg[:, :-1])
    wv, _, dz = _sim1(dp * RGRAV, zh[:, 1:] - zh[:, :-1], 1.0 / (1.0 - cappa[:, :N]), pt[:, :N], cappa[:, :N],
                      w[:, :N], pem, pm, wsr, dt, p_fac)
    return wv, dz


def riemc_columns(w3, gz, delpc, ptc, cappa, q_con, hs, wsr, dt2, ptop, p_fac):
    """RiemannSolverC (riem_solver_c.py:13-64 + sim1): new (pef, gz) on the
    K interfaces."""
    N = gz.shape[1] - 1
    dp = delpc[:, :N]
    pem, peg = _column_sums(dp, q_con[:, :N], ptop)
    pm = (peg[:, 1:] - peg[:, :-1]) / torch.log(peg[:, 1:] / peg[:, :-1])
    _, pe, dz = _sim1(dp / GRAV, gz[:, 1:] - gz[:, :-1], 1.0 / (1.0 - cappa[:, :N]), ptc[:, :N], cappa[:, :N],
                      w3[:, :N], pem, pm, wsr, dt2, p_fac)
    ncol = gz.shape[0]
    pef = [torch.zeros(ncol, dtype=gz.dtype) + ptop] + [pe[k] + pem[:, k] for k in range(1, N + 1)]
    g = [None] * (N + 1)
    g[N] = hs
    for k in range(N - 1, -1, -1):
        g[k] = g[k + 1] - dz[:, k] * GRAV
    return torch.stack(pef, dim=1), torch.stack(g, dim=1)

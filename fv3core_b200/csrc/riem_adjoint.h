// Hand-written adjoints (reverse mode) of the two vertically implicit
// solvers' column work: Sim1Solver (sim1_solver.py:11-105) shared by both,
// with the precompute and finalize of RiemannSolver3 (riem_solver3.py:24-67)
// and of RiemannSolverC (riem_solver_c.py:13-64).  Written for both the
// device and the host
// (the tests build it with g++ and compare with torch autograd of a
// PyTorch-ops restatement).
//
// The forward values are recomputed first, with the same operations as the
// solver (the library's exp and log), and kept in per-level arrays; the
// reverse sweep then runs every forward step backwards.  The branch of the
// pressure floor (maxp) is taken as the forward took it.  Columns need at
// least four interface levels (three layers).  cappa, q_con and the
// surface height are held fixed; the surface w has its gradient.
#pragma once

#include "fmath.h"

namespace fv3b {
namespace adj {

constexpr double A_RDGAS = 287.05;
constexpr double A_GRAV = 9.80665;
constexpr double A_RGRAV = 1.0 / A_GRAV;

// Sim1Solver's adjoint for one column of N layers (N + 1 interfaces).
// Forward inputs: DM (delta p / g), DZ (layer depths), GM = 1 / (1 - cappa),
// PT, CP3 (cappa), W1 (w at the start), pem (edge pressures, N + 1) and pm
// (layer-mean pressures).  Forward outputs: w (aWF_in is its cotangent), the
// pressure perturbation pe at interfaces 0..N (aPE_in) and dz (aDZ_in).
// The adjoints of the inputs are added into aDM, aDZ, aPT, aW1, aPEM, aPM
// and *aWSR (the surface w).
template <int NK>
__host__ __device__ inline void sim1_column_adjoint(int N, const double* DM, const double* DZ, const double* GM,
                                                    const double* PT, const double* CP3, const double* W1,
                                                    const double* pem, const double* pm, double wsr, double dt,
                                                    double p_fac, const double* aWF_in, const double* aPE_in,
                                                    const double* aDZ_in, double* aDM, double* aDZ, double* aPT,
                                                    double* aW1, double* aPEM, double* aPM, double* aWSR) {
  double Xv[NK], Yv[NK], pe1[NK];
  double grat[NK], bb[NK], dd[NK], bet[NK], gam[NK], pp[NK], ppb[NK], aa[NK];
  double betw[NK], gw[NK], wpre[NK], wf[NK], pe[NK], p1[NK], maxp[NK], Ev[NK], dzv[NK];
  bool floor_branch[NK];
  // ---------------------------------------------------------------- forward
  for (int k = 0; k < N; ++k) {
    Xv[k] = -DM[k] / DZ[k] * A_RDGAS * PT[k];
    Yv[k] = fm::fm_exp(GM[k] * fm::fm_log(Xv[k]));
    pe1[k] = Yv[k] - pm[k];
  }
  for (int k = 0; k < N - 1; ++k) {
    grat[k] = DM[k] / DM[k + 1];
    bb[k] = 2.0 * (1.0 + grat[k]);
    dd[k] = 3.0 * (pe1[k] + grat[k] * pe1[k + 1]);
  }
  bb[N - 1] = 2.0;
  dd[N - 1] = 3.0 * pe1[N - 1];
  bet[0] = bb[0];
  for (int k = 1; k < N; ++k) {
    gam[k] = grat[k - 1] / bet[k - 1];
    bet[k] = bb[k] - gam[k];
  }
  pp[0] = 0.0;
  pp[1] = dd[0] / bet[0];
  for (int k = 2; k <= N; ++k) pp[k] = (dd[k - 1] - pp[k - 1]) / bet[k - 1];
  ppb[N] = pp[N];
  ppb[0] = pp[0];
  for (int k = N - 1; k >= 1; --k) ppb[k] = pp[k] - gam[k] * ppb[k + 1];
  const double t1g = 2.0 * dt * dt, rdt = 1.0 / dt;
  for (int k = 1; k < N; ++k) aa[k] = t1g * 0.5 * (GM[k - 1] + GM[k]) / (DZ[k - 1] + DZ[k]) * (pem[k] + ppb[k]);
  betw[0] = DM[0] - aa[1];
  wpre[0] = (DM[0] * W1[0] + dt * ppb[1]) / betw[0];
  for (int k = 1; k < N - 1; ++k) {
    gw[k] = aa[k] / betw[k - 1];
    betw[k] = DM[k] - (aa[k] + aa[k + 1] + aa[k] * gw[k]);
    wpre[k] = (DM[k] * W1[k] + dt * (ppb[k + 1] - ppb[k]) - aa[k] * wpre[k - 1]) / betw[k];
  }
  const int kl = N - 1;
  const double p1t = t1g * GM[kl] / DZ[kl] * (pem[kl + 1] + ppb[kl + 1]);
  gw[kl] = aa[kl] / betw[kl - 1];
  betw[kl] = DM[kl] - (aa[kl] + p1t + aa[kl] * gw[kl]);
  wpre[kl] = (DM[kl] * W1[kl] + dt * (ppb[kl + 1] - ppb[kl]) - p1t * wsr - aa[kl] * wpre[kl - 1]) / betw[kl];
  wf[N - 1] = wpre[N - 1];
  for (int k = N - 2; k >= 0; --k) wf[k] = wpre[k] - gw[k + 1] * wf[k + 1];
  pe[0] = 0.0;
  for (int k = 1; k <= N; ++k) pe[k] = pe[k - 1] + DM[k - 1] * (wf[k - 1] - W1[k - 1]) * rdt;
  p1[N - 1] = (pe[N - 1] + 2.0 * pe[N]) * 1.0 / 3.0;
  for (int k = N - 2; k >= 0; --k)
    p1[k] = (pe[k] + bb[k] * pe[k + 1] + grat[k] * pe[k + 2]) * 1.0 / 3.0 - grat[k] * p1[k + 1];
  for (int k = 0; k < N; ++k) {
    floor_branch[k] = p_fac * DM[k] > p1[k] + pm[k];
    maxp[k] = floor_branch[k] ? p_fac * pm[k] : p1[k] + pm[k];
    Ev[k] = fm::fm_exp((CP3[k] - 1.0) * fm::fm_log(maxp[k]));
    dzv[k] = -DM[k] * A_RDGAS * PT[k] * Ev[k];
  }
  // ---------------------------------------------------------------- reverse
  double aPE1[NK], aGR[NK], aBB[NK], aDD[NK], aBET[NK], aGAM[NK], aPP[NK], aPPB[NK], aAA[NK];
  double aBETW[NK], aGW[NK], aW[NK], aWF[NK], aPE[NK], aP1[NK];
  for (int k = 0; k < NK; ++k) {
    aPE1[k] = aGR[k] = aBB[k] = aDD[k] = aBET[k] = aGAM[k] = aPP[k] = aPPB[k] = aAA[k] = 0.0;
    aBETW[k] = aGW[k] = aW[k] = aWF[k] = aP1[k] = 0.0;
    aPE[k] = k <= N ? aPE_in[k] : 0.0;
  }
  // dz = -DM Rd PT exp((cp3 - 1) log(maxp)); maxp on the forward's branch
  for (int k = 0; k < N; ++k) {
    const double a = aDZ_in[k];
    aDM[k] += a * (-A_RDGAS * PT[k] * Ev[k]);
    aPT[k] += a * (-DM[k] * A_RDGAS * Ev[k]);
    const double amax = a * dzv[k] * (CP3[k] - 1.0) / maxp[k];
    if (floor_branch[k]) {
      aPM[k] += amax * p_fac;
    } else {
      aP1[k] += amax;
      aPM[k] += amax;
    }
  }
  // p1 recurrence (computed downwards, so its adjoint runs upwards)
  for (int k = 0; k <= N - 2; ++k) {
    const double a = aP1[k];
    aPE[k] += a / 3.0;
    aPE[k + 1] += a * bb[k] / 3.0;
    aPE[k + 2] += a * grat[k] / 3.0;
    aBB[k] += a * pe[k + 1] / 3.0;
    aGR[k] += a * (pe[k + 2] / 3.0 - p1[k + 1]);
    aP1[k + 1] += -a * grat[k];
  }
  aPE[N - 1] += aP1[N - 1] / 3.0;
  aPE[N] += aP1[N - 1] * 2.0 / 3.0;
  // pe[k] = pe[k-1] + DM[k-1] (wf[k-1] - W1[k-1]) rdt
  for (int k = 0; k < N; ++k) aWF[k] = aWF_in[k];
  for (int k = N; k >= 1; --k) {
    const double a = aPE[k];
    aPE[k - 1] += a;
    aDM[k - 1] += a * (wf[k - 1] - W1[k - 1]) * rdt;
    aWF[k - 1] += a * DM[k - 1] * rdt;
    aW1[k - 1] -= a * DM[k - 1] * rdt;
  }
  // back substitution of w (downwards, adjoint upwards)
  for (int k = 0; k <= N - 2; ++k) {
    aW[k] += aWF[k];
    aGW[k + 1] += -aWF[k] * wf[k + 1];
    aWF[k + 1] += -aWF[k] * gw[k + 1];
  }
  aW[N - 1] += aWF[N - 1];
  // forward sweep of the w system, last level first
  {
    const int k = kl;
    const double anum = aW[k] / betw[k];
    aBETW[k] += -aW[k] * wpre[k] / betw[k];
    aDM[k] += anum * W1[k];
    aW1[k] += anum * DM[k];
    aPPB[k + 1] += anum * dt;
    aPPB[k] -= anum * dt;
    double ap1t = -anum * wsr;
    *aWSR += -anum * p1t;
    aAA[k] += -anum * wpre[k - 1];
    aW[k - 1] += -anum * aa[k];
    const double ab = aBETW[k];
    aDM[k] += ab;
    aAA[k] += -ab * (1.0 + gw[k]);
    ap1t += -ab;
    aGW[k] += -ab * aa[k];
    aAA[k] += aGW[k] / betw[k - 1];
    aBETW[k - 1] += -aGW[k] * gw[k] / betw[k - 1];
    const double c = t1g * GM[k] / DZ[k];
    aDZ[k] += -ap1t * p1t / DZ[k];
    aPEM[k + 1] += ap1t * c;
    aPPB[k + 1] += ap1t * c;
  }
  for (int k = N - 2; k >= 1; --k) {
    const double anum = aW[k] / betw[k];
    aBETW[k] += -aW[k] * wpre[k] / betw[k];
    aDM[k] += anum * W1[k];
    aW1[k] += anum * DM[k];
    aPPB[k + 1] += anum * dt;
    aPPB[k] -= anum * dt;
    aAA[k] += -anum * wpre[k - 1];
    aW[k - 1] += -anum * aa[k];
    const double ab = aBETW[k];
    aDM[k] += ab;
    aAA[k] += -ab * (1.0 + gw[k]);
    aAA[k + 1] += -ab;
    aGW[k] += -ab * aa[k];
    aAA[k] += aGW[k] / betw[k - 1];
    aBETW[k - 1] += -aGW[k] * gw[k] / betw[k - 1];
  }
  {
    const double anum = aW[0] / betw[0];
    aBETW[0] += -aW[0] * wpre[0] / betw[0];
    aDM[0] += anum * W1[0];
    aW1[0] += anum * DM[0];
    aPPB[1] += anum * dt;
    aDM[0] += aBETW[0];
    aAA[1] += -aBETW[0];
  }
  // aa[k] = t1g 0.5 (GM[k-1] + GM[k]) / (DZ[k-1] + DZ[k]) (pem[k] + ppb[k])
  for (int k = 1; k < N; ++k) {
    const double S = DZ[k - 1] + DZ[k];
    const double c = t1g * 0.5 * (GM[k - 1] + GM[k]);
    const double aS = -aAA[k] * aa[k] / S;
    aDZ[k - 1] += aS;
    aDZ[k] += aS;
    const double aP = aAA[k] * c / S;
    aPEM[k] += aP;
    aPPB[k] += aP;
  }
  // back substitution of pp (downwards, adjoint upwards)
  for (int k = 1; k <= N - 1; ++k) {
    aPP[k] += aPPB[k];
    aGAM[k] += -aPPB[k] * ppb[k + 1];
    aPPB[k + 1] += -aPPB[k] * gam[k];
  }
  aPP[N] += aPPB[N];
  // forward recurrence of pp
  for (int k = N; k >= 2; --k) {
    const double a = aPP[k];
    aDD[k - 1] += a / bet[k - 1];
    aPP[k - 1] += -a / bet[k - 1];
    aBET[k - 1] += -a * pp[k] / bet[k - 1];
  }
  aDD[0] += aPP[1] / bet[0];
  aBET[0] += -aPP[1] * pp[1] / bet[0];
  // gam[k] = grat[k-1] / bet[k-1]; bet[k] = bb[k] - gam[k]
  for (int k = N - 1; k >= 1; --k) {
    aBB[k] += aBET[k];
    aGAM[k] += -aBET[k];
    aGR[k - 1] += aGAM[k] / bet[k - 1];
    aBET[k - 1] += -aGAM[k] * gam[k] / bet[k - 1];
  }
  aBB[0] += aBET[0];
  // bb, dd from grat and pe1; grat from DM
  for (int k = 0; k < N - 1; ++k) {
    aGR[k] += 2.0 * aBB[k];
    aPE1[k] += 3.0 * aDD[k];
    aGR[k] += 3.0 * aDD[k] * pe1[k + 1];
    aPE1[k + 1] += 3.0 * aDD[k] * grat[k];
  }
  aPE1[N - 1] += 3.0 * aDD[N - 1];
  for (int k = 0; k < N - 1; ++k) {
    aDM[k] += aGR[k] / DM[k + 1];
    aDM[k + 1] += -aGR[k] * grat[k] / DM[k + 1];
  }
  // pe1 = exp(GM log X) - pm, X = -DM / DZ Rd PT
  for (int k = 0; k < N; ++k) {
    const double aX = aPE1[k] * GM[k] * Yv[k] / Xv[k];
    aPM[k] += -aPE1[k];
    aDM[k] += aX * (-A_RDGAS * PT[k] / DZ[k]);
    aDZ[k] += aX * (DM[k] * A_RDGAS * PT[k] / (DZ[k] * DZ[k]));
    aPT[k] += aX * (-DM[k] * A_RDGAS / DZ[k]);
  }
}

// Adjoint of the layer-mean pressures pm = (peg[k+1] - peg[k]) / L with
// L = log(peg[k+1]) - log(peg[k]) (or log of their ratio: the same
// derivatives) and of the running sums peg (moist) and pem over delp; adds
// the result to a_dp.  peg[0] = pem[0] = ptop is fixed.
template <int NK>
__host__ __device__ inline void column_sums_adjoint(int N, const double* peg, const double* L, const double* pm,
                                                    const double* qc, double* aPM, double* aPEM, double* a_dp) {
  double aPEG[NK];
  for (int k = 0; k < NK; ++k) aPEG[k] = 0.0;
  for (int k = 0; k < N; ++k) {
    const double anum = aPM[k] / L[k];
    const double aden = -aPM[k] * pm[k] / L[k];
    aPEG[k + 1] += anum + aden / peg[k + 1];
    aPEG[k] += -anum - aden / peg[k];
  }
  for (int k = N - 1; k >= 0; --k) {
    aPEG[k] += aPEG[k + 1];
    a_dp[k] += aPEG[k + 1] * (1.0 - qc[k]);
    aPEM[k] += aPEM[k + 1];
    a_dp[k] += aPEM[k + 1];
  }
}

// RiemannSolver3's column (riem_solver3.py:24-67 + sim1): one column with K
// interface levels (N = K - 1 layers); every pointer steps sk elements per
// level.  Inputs w, zh, delp, pt, cappa, q_con; the cotangents gw_out (of
// the new w) and gdz_out (of the new delz); results g_w, g_delp, g_pt on
// layers, g_zh on interfaces and *g_wsr for the surface w (overwritten).
template <int NK, typename R, typename G>
__host__ __device__ inline void riem3_column_adjoint(int K, long long sk, double dt, double ptop, double p_fac,
                                                     double wsr, const R* w, const R* zh, const R* delp,
                                                     const R* pt, const R* cappa, const R* q_con,
                                                     const G* gw_out, const G* gdz_out, G* g_w, G* g_zh,
                                                     G* g_delp, G* g_pt, G* g_wsr) {
  const int N = K - 1;
  double DM[NK], DZ[NK], GM[NK], PT[NK], CP3[NK], W1[NK], QC[NK];
  double pem[NK], peg[NK], lg[NK], L[NK], pm[NK];
  for (int k = 0; k < N; ++k) {
    DM[k] = (double)delp[k * sk] * A_RGRAV;
    DZ[k] = (double)zh[(k + 1) * sk] - (double)zh[k * sk];
    GM[k] = 1.0 / (1.0 - (double)cappa[k * sk]);
    PT[k] = pt[k * sk];
    CP3[k] = cappa[k * sk];
    W1[k] = w[k * sk];
    QC[k] = q_con[k * sk];
  }
  pem[0] = ptop;
  peg[0] = ptop;
  lg[0] = fm::fm_log(ptop);
  for (int k = 0; k < N; ++k) {
    const double dp = delp[k * sk];
    pem[k + 1] = pem[k] + dp;
    peg[k + 1] = peg[k] + dp * (1.0 - QC[k]);
    lg[k + 1] = fm::fm_log(peg[k + 1]);
    L[k] = lg[k + 1] - lg[k];
    pm[k] = (peg[k + 1] - peg[k]) / L[k];
  }
  double aDM[NK], aDZ[NK], aPT[NK], aW1[NK], aPEM[NK], aPM[NK], aWF[NK], aPE[NK], aDZo[NK], a_dp[NK];
  for (int k = 0; k < NK; ++k) aDM[k] = aDZ[k] = aPT[k] = aW1[k] = aPEM[k] = aPM[k] = aPE[k] = a_dp[k] = 0.0;
  for (int k = 0; k < N; ++k) {
    aWF[k] = gw_out[k * sk];
    aDZo[k] = gdz_out[k * sk];
  }
  double aWSR = 0.0;
  sim1_column_adjoint<NK>(N, DM, DZ, GM, PT, CP3, W1, pem, pm, wsr, dt, p_fac, aWF, aPE, aDZo, aDM, aDZ, aPT, aW1,
                          aPEM, aPM, &aWSR);
  column_sums_adjoint<NK>(N, peg, L, pm, QC, aPM, aPEM, a_dp);
  *g_wsr = aWSR;
  for (int k = 0; k <= N; ++k) g_zh[k * sk] = 0.0;
  for (int k = 0; k < N; ++k) {
    g_delp[k * sk] = a_dp[k] + aDM[k] * A_RGRAV;
    g_pt[k * sk] = aPT[k];
    g_w[k * sk] = aW1[k];
    g_zh[(k + 1) * sk] += aDZ[k];
    g_zh[k * sk] -= aDZ[k];
  }
}

// RiemannSolverC's column (riem_solver_c.py:13-64 + sim1): inputs w3, gz
// (interface heights), delpc, ptc, cappa, q_con, the surface height hs and
// ws; outputs pef (pe + pem on interfaces 1..N, ptop on top) and gz
// (hs at the bottom, gz[k] = gz[k+1] - dz[k] g).  Cotangents gpef_out,
// ggz_out on interfaces; results g_w3, g_delpc, g_ptc on layers and g_gz on
// interfaces (the input heights), *g_wsr for the surface w ws.
template <int NK, typename R, typename G>
__host__ __device__ inline void riemc_column_adjoint(int K, long long sk, double dt2, double ptop, double p_fac,
                                                     double wsr, const R* w3, const R* gz, const R* delpc,
                                                     const R* ptc, const R* cappa, const R* q_con,
                                                     const G* gpef_out, const G* ggz_out, G* g_w3, G* g_gz,
                                                     G* g_delpc, G* g_ptc, G* g_wsr) {
  const int N = K - 1;
  double DM[NK], DZ[NK], GM[NK], PT[NK], CP3[NK], W1[NK], QC[NK];
  double pem[NK], peg[NK], L[NK], pm[NK];
  for (int k = 0; k < N; ++k) {
    DM[k] = (double)delpc[k * sk] / A_GRAV;
    DZ[k] = (double)gz[(k + 1) * sk] - (double)gz[k * sk];
    GM[k] = 1.0 / (1.0 - (double)cappa[k * sk]);
    PT[k] = ptc[k * sk];
    CP3[k] = cappa[k * sk];
    W1[k] = w3[k * sk];
    QC[k] = q_con[k * sk];
  }
  pem[0] = ptop;
  peg[0] = ptop;
  for (int k = 0; k < N; ++k) {
    const double dp = delpc[k * sk];
    pem[k + 1] = pem[k] + dp;
    peg[k + 1] = peg[k] + dp * (1.0 - QC[k]);
    L[k] = fm::fm_log(peg[k + 1] / peg[k]);
    pm[k] = (peg[k + 1] - peg[k]) / L[k];
  }
  double aDM[NK], aDZ[NK], aPT[NK], aW1[NK], aPEM[NK], aPM[NK], aWF[NK], aPE[NK], aDZo[NK], a_dp[NK];
  for (int k = 0; k < NK; ++k) {
    aDM[k] = aDZ[k] = aPT[k] = aW1[k] = aPEM[k] = aPM[k] = aWF[k] = aPE[k] = aDZo[k] = a_dp[k] = 0.0;
  }
  // pef[k] = pe[k] + pem[k] for k >= 1
  for (int k = 1; k <= N; ++k) {
    aPE[k] = gpef_out[k * sk];
    aPEM[k] += gpef_out[k * sk];
  }
  // gz[k] = hs - g sum_{m >= k} dz[m]: dz[m] collects -g times the
  // cotangents of gz[0..m]
  double acc = 0.0;
  for (int m = 0; m < N; ++m) {
    acc += ggz_out[m * sk];
    aDZo[m] = -A_GRAV * acc;
  }
  double aWSR = 0.0;
  sim1_column_adjoint<NK>(N, DM, DZ, GM, PT, CP3, W1, pem, pm, wsr, dt2, p_fac, aWF, aPE, aDZo, aDM, aDZ, aPT, aW1,
                          aPEM, aPM, &aWSR);
  column_sums_adjoint<NK>(N, peg, L, pm, QC, aPM, aPEM, a_dp);
  *g_wsr = aWSR;
  for (int k = 0; k <= N; ++k) g_gz[k * sk] = 0.0;
  for (int k = 0; k < N; ++k) {
    g_delpc[k * sk] = a_dp[k] + aDM[k] / A_GRAV;
    g_ptc[k * sk] = aPT[k];
    g_w3[k * sk] = aW1[k];
    g_gz[(k + 1) * sk] += aDZ[k];
    g_gz[k * sk] -= aDZ[k];
  }
}

}  // namespace adj
}  // namespace fv3b

// Vertically implicit acoustic solvers: RiemannSolverC and RiemannSolver3
// with the shared Sim1 tridiagonal solve.
//
// One thread owns one (tile, i, j) column and walks it top to bottom and
// back; neighbouring threads own neighbouring i, so every level load/store
// is a coalesced row access.  Column work arrays live in per-thread local
// memory (thread-interleaved, so also coalesced); MAXK bounds the number of
// interface levels.  exp and log are the library's own (fmath.h), whose
// host build the oracle uses, so results can be compared to the last bit.
#include <math.h>

#include "common.cuh"
#include "fmath.h"

namespace fv3b {

constexpr double GRAV = 9.80665;
constexpr double RDGAS = 287.05;
constexpr double RGRAV = 1.0 / GRAV;
constexpr double KAPPA = RDGAS / 1004.6;
constexpr int MAXK = 128;

// Sim1 solve on one column (reference fv3core/stencils/sim1_solver.py:11-101).
// K = number of interface levels (npz + 1).  On entry: dm (delta p / g),
// w (vertical velocity, kept as w1), dz (layer depth, negative), pem (edge
// pressure), pm (layer mean pressure); gm, ptr, cp3 come from the lambdas
// (per level).  On exit: w (levels 0..K-2), pe (0..K-1, pressure
// perturbation), dz (0..K-2).
template <typename GM, typename PTR, typename CP3>
__device__ __forceinline__ void sim1_column(int K, const double* dm, double* w, double* w1, double* dz,
                                            const double* pem, const double* pm, double* pe, double* pp,
                                            double* gam, double* aa, GM gm, PTR ptr, CP3 cp3, double wsr,
                                            double dt, double t1g, double rdt, double p_fac) {
  // pe = exp(gm*log(-dm/dz*Rd*ptr)) - pm   (sim1_solver.py:27-29)
  for (int k = 0; k < K - 1; ++k) {
    pe[k] = fm::fm_exp(gm(k) * fm::fm_log(-dm[k] / dz[k] * RDGAS * ptr(k))) - pm[k];
    w1[k] = w[k];
  }
  // forward elimination of the pressure system (sim1_solver.py:30-59)
  double bb0 = (K - 2 > 0) ? 2.0 * (1.0 + dm[0] / dm[1]) : 2.0;
  pp[0] = 0.0;
  pp[1] = (K > 2 ? 3.0 * (pe[0] + (dm[0] / dm[1]) * pe[1]) : 3.0 * pe[0]) / bb0;
  double bet = bb0;
  for (int k = 1; k <= K - 2; ++k) {
    double grm = dm[k - 1] / dm[k];
    double g = grm / bet;
    double bbk, ddk;
    if (k < K - 2) {
      double grk = dm[k] / dm[k + 1];
      bbk = 2.0 * (1.0 + grk);
      ddk = 3.0 * (pe[k] + grk * pe[k + 1]);
    } else {
      bbk = 2.0;
      ddk = 3.0 * pe[k];
    }
    gam[k] = g;
    bet = bbk - g;
    pp[k + 1] = (ddk - pp[k]) / bet;
  }
  // back substitution and w coefficients (sim1_solver.py:60-63)
  for (int k = K - 2; k >= 1; --k) {
    pp[k] = pp[k] - gam[k] * pp[k + 1];
    aa[k] = t1g * 0.5 * (gm(k - 1) + gm(k)) / (dz[k - 1] + dz[k]) * (pem[k] + pp[k]);
  }
  // w solve (sim1_solver.py:65-90)
  bet = dm[0] - aa[1];
  w[0] = (dm[0] * w1[0] + dt * pp[1]) / bet;
  for (int k = 1; k <= K - 3; ++k) {
    double g = aa[k] / bet;
    gam[k] = g;
    bet = dm[k] - (aa[k] + aa[k + 1] + aa[k] * g);
    w[k] = (dm[k] * w1[k] + dt * (pp[k + 1] - pp[k]) - aa[k] * w[k - 1]) / bet;
  }
  {
    int k = K - 2;
    double p1 = t1g * gm(k) / dz[k] * (pem[k + 1] + pp[k + 1]);
    double g = aa[k] / bet;
    gam[k] = g;
    bet = dm[k] - (aa[k] + p1 + aa[k] * g);
    w[k] = (dm[k] * w1[k] + dt * (pp[k + 1] - pp[k]) - p1 * wsr - aa[k] * w[k - 1]) / bet;
  }
  for (int k = K - 3; k >= 0; --k) w[k] = w[k] - gam[k + 1] * w[k + 1];
  // pressure perturbation from the w change (sim1_solver.py:91-95)
  pe[0] = 0.0;
  for (int k = 1; k < K; ++k) pe[k] = pe[k - 1] + dm[k - 1] * (w[k - 1] - w1[k - 1]) * rdt;
  // layer-mean perturbation and new dz (sim1_solver.py:96-105)
  double p1n = 0.0;
  for (int k = K - 2; k >= 0; --k) {
    double p1;
    if (k == K - 2) {
      p1 = (pe[k] + 2.0 * pe[k + 1]) * 1.0 / 3.0;
    } else {
      double gr = dm[k] / dm[k + 1];
      double bbk = 2.0 * (1.0 + gr);
      p1 = (pe[k] + bbk * pe[k + 1] + gr * pe[k + 2]) * 1.0 / 3.0 - gr * p1n;
    }
    p1n = p1;
    double maxp = (p_fac * dm[k] > p1 + pm[k]) ? p_fac * pm[k] : p1 + pm[k];
    dz[k] = -dm[k] * RDGAS * ptr(k) * fm::fm_exp((cp3(k) - 1.0) * fm::fm_log(maxp));
  }
}

}  // namespace fv3b

using namespace fv3b;

extern "C" int fv3b_riem_solver_c(const fv3b_grid_dims* dims, double dt2, double ptop, double p_fac,
                                  const double* cappa, const double* hs, const double* ws,
                                  const double* ptc, const double* q_con, const double* delpc,
                                  double* gz, double* pef, const double* w3, void* stream) {
  FV3B_REQUIRE(dims && cappa && hs && ws && ptc && q_con && delpc && gz && pef && w3,
               "fv3b_riem_solver_c: null argument");
  Dims d = make_dims(dims);
  FV3B_REQUIRE(d.nk <= MAXK && d.nk >= 3, "fv3b_riem_solver_c: npz out of range (2..127)");
  cudaStream_t s = (cudaStream_t)stream;
  const int K = d.nk;
  const double t1g = 2.0 * dt2 * dt2;
  const double rdt = 1.0 / dt2;
  auto body = [=] __device__(int t, int i, int j) {
    double dm[MAXK], w[MAXK], w1[MAXK], dz[MAXK], pem[MAXK], pm[MAXK], pe[MAXK], pp[MAXK], gam[MAXK],
        aa[MAXK];
    // precompute (riem_solver_c.py:13-44)
    double pem_k = ptop, peg_k = ptop;
    double gz_prev = gz[idx3(d, t, i, j, 0)];
    for (int k = 0; k < K; ++k) {
      long long o = idx3(d, t, i, j, k);
      double dmk = delpc[o];
      pem[k] = pem_k;
      double peg_next = peg_k + dmk * (1.0 - q_con[o]);
      if (k < K - 1) {
        double gz_next = gz[o + d.sk];
        dz[k] = gz_next - gz_prev;
        gz_prev = gz_next;
        pm[k] = (peg_next - peg_k) / fm::fm_log(peg_next / peg_k);
      }
      pem_k = pem_k + dmk;
      peg_k = peg_next;
      dm[k] = dmk / GRAV;
      w[k] = w3[o];
    }
    auto gm = [&](int k) { return 1.0 / (1.0 - cappa[idx3(d, t, i, j, k)]); };
    auto ptr = [&](int k) { return ptc[idx3(d, t, i, j, k)]; };
    auto cp3 = [&](int k) { return cappa[idx3(d, t, i, j, k)]; };
    sim1_column(K, dm, w, w1, dz, pem, pm, pe, pp, gam, aa, gm, ptr, cp3, ws[idx2(d, t, i, j)], dt2, t1g,
                rdt, p_fac);
    // finalize (riem_solver_c.py:46-64)
    pef[idx3(d, t, i, j, 0)] = ptop;
    for (int k = 1; k < K; ++k) pef[idx3(d, t, i, j, k)] = pe[k] + pem[k];
    double g = hs[idx2(d, t, i, j)];
    gz[idx3(d, t, i, j, K - 1)] = g;
    for (int k = K - 2; k >= 0; --k) {
      g = g - dz[k] * GRAV;
      gz[idx3(d, t, i, j, k)] = g;
    }
  };
  FV3B_CHECK(launch_columns(d.isc - 1, d.iec + 2, d.jsc - 1, d.jec + 2, s, body));
  return FV3B_OK;
}

// RiemannSolver3.__call__ (riem_solver3.py:145-242): precompute (24-67),
// Sim1 solve, finalize (70-103) on the compute-domain columns, interface
// levels 0..npz.
extern "C" int fv3b_riem_solver3(const fv3b_grid_dims* dims, int last_call, double dt, double ptop, double p_fac,
                                 const double* cappa, const double* zs, const double* wsd, double* delz,
                                 const double* q_con, const double* delp, const double* pt, double* zh, double* pe,
                                 double* ppe, double* pk3, double* pk, double* peln, double* w, void* stream) {
  FV3B_REQUIRE(dims && cappa && zs && wsd && delz && q_con && delp && pt && zh && pe && ppe && pk3 && pk && peln && w,
               "fv3b_riem_solver3: null argument");
  Dims d = make_dims(dims);
  FV3B_REQUIRE(d.nk <= MAXK && d.nk >= 3, "fv3b_riem_solver3: npz out of range (2..127)");
  cudaStream_t s = (cudaStream_t)stream;
  const int K = d.nk;
  const double peln1 = log(ptop);
  const double ptk = exp(KAPPA * peln1);
  const double t1g = 2.0 * dt * dt;
  const double rdt = 1.0 / dt;
  const bool last = last_call != 0;
  auto body = [=] __device__(int t, int i, int j) {
    double dm[MAXK], wc[MAXK], w1[MAXK], dz[MAXK], pem[MAXK], pm[MAXK], pec[MAXK], pp[MAXK], gam[MAXK],
        aa[MAXK], peln_run[MAXK];
    const long long o0 = idx3(d, t, i, j, 0);
    // precompute
    double pem_k = ptop, peg_k = ptop, pelng_k = peln1;
    pem[0] = ptop;
    peln_run[0] = peln1;
    pk3[o0] = ptk;
    for (int k = 0; k < K; ++k) {
      long long o = o0 + k * d.sk;
      double dmk = delp[o];
      if (k < K - 1) {
        double pem_n = pem_k + dmk;
        double peg_n = peg_k + dmk * (1.0 - q_con[o]);
        double pelng_n = fm::fm_log(peg_n);
        double peln_n = fm::fm_log(pem_n);
        pem[k + 1] = pem_n;
        peln_run[k + 1] = peln_n;
        pk3[o + d.sk] = fm::fm_exp(KAPPA * peln_n);
        pm[k] = (peg_n - peg_k) / (pelng_n - pelng_k);
        dz[k] = zh[o + d.sk] - zh[o];
        pem_k = pem_n;
        peg_k = peg_n;
        pelng_k = pelng_n;
      }
      dm[k] = dmk * RGRAV;
      wc[k] = w[o];
    }
    auto gm = [&](int k) { return 1.0 / (1.0 - cappa[o0 + k * d.sk]); };
    auto ptr = [&](int k) { return pt[o0 + k * d.sk]; };
    auto cp3 = [&](int k) { return cappa[o0 + k * d.sk]; };
    sim1_column(K, dm, wc, w1, dz, pem, pm, pec, pp, gam, aa, gm, ptr, cp3, wsd[idx2(d, t, i, j)], dt, t1g, rdt,
                p_fac);
    // finalize (beta = 0, use_logp = False)
    for (int k = 0; k < K; ++k) {
      long long o = o0 + k * d.sk;
      ppe[o] = pec[k];
      if (last) {
        peln[o] = peln_run[k];
        pk[o] = pk3[o];
        pe[o] = pem[k];
      }
      if (k < K - 1) {
        w[o] = wc[k];
        delz[o] = dz[k];
      }
    }
    double z = zs[idx2(d, t, i, j)];
    zh[o0 + (K - 1) * d.sk] = z;
    for (int k = K - 2; k >= 0; --k) {
      z = z - dz[k];
      zh[o0 + k * d.sk] = z;
    }
  };
  FV3B_CHECK(launch_columns(d.isc, d.iec + 1, d.jsc, d.jec + 1, s, body));
  return FV3B_OK;
}

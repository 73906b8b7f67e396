// Vertically implicit acoustic solvers: RiemannSolverC and RiemannSolver3
// with the shared Sim1 tridiagonal solve.
//
// One thread owns one (tile, i, j) column and walks it top to bottom and
// back; neighbouring threads own neighbouring i, so every level load/store
// is a coalesced row access.  Only four per-level work arrays stay in the
// thread's local memory (pm, pp/pe, gam, w); the edge pressures are running
// sums rebuilt where they are used, everything else is re-read from the
// input fields or computed on the fly, and the outputs are written in the
// same bottom-up pass that produces them.  The arrays are sized by a
// compile-time level bucket >= npz+1, so an L79 column keeps 2.5 KB.
// exp and log are the library's own (fmath.h), whose host build the oracle
// uses, so results can be compared to the last bit.  The column arithmetic
// is FP64 in both builds; in the mixed-precision build the fields it reads
// and writes are FP32.
#include <math.h>

#include "common.cuh"
#include "fmath.h"

namespace fv3b {

constexpr double GRAV = 9.80665;
constexpr double RDGAS = 287.05;
constexpr double RGRAV = 1.0 / GRAV;
constexpr double KAPPA = RDGAS / 1004.6;
constexpr int MAXK = 128;

// Requests the 128-byte line holding *p into L2 (PTX prefetch): the column
// loops walk the levels one after another, so each loop asks for the inputs
// a few levels ahead while it works on the current one.
__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}
constexpr int PF_AHEAD = 3;

// Per-column inputs of the Sim1 solve (fv3core/stencils/sim1_solver.py:11-101).
// K = number of interface levels (npz + 1).  DM(k): delta p / g; DP(k):
// delta p, whose running sums from ptop are the edge pressures pem; W1(k): w
// at the start; DZ(k): layer depth at the start (negative); GM, PTR, CP3:
// 1/(1-cappa), pt, cappa per level; pm: layer-mean pressure.  Results: w[0..K-2] (new w), pe[0..K-1] (pressure perturbation,
// delivered through PE_OUT(k, value) in increasing k) and the new layer
// depths through DZ_OUT(k, value) for k = K-2 .. 0 (bottom up).
template <int NK, typename DMF, typename DPF, typename W1F, typename DZF, typename GMF, typename PTRF,
          typename CP3F, typename PEOUT, typename DZOUT, typename PFF>
__device__ __forceinline__ void sim1_column(int K, DMF DM, DPF DP, double ptop, W1F W1, DZF DZ, GMF GM, PTRF PTR,
                                            CP3F CP3, const double* pm, double* pp, double* gam, double* w,
                                            double wsr, double dt, double t1g, double rdt, double p_fac,
                                            PEOUT PE_OUT, DZOUT DZ_OUT, PFF PF) {
  // pe = exp(gm*log(-dm/dz*Rd*ptr)) - pm   (sim1_solver.py:27-29), on the fly
  auto pe1 = [&](int k) { return fm::fm_exp(GM(k) * fm::fm_log(-DM(k) / DZ(k) * RDGAS * PTR(k))) - pm[k]; };
  // forward elimination of the pressure system (sim1_solver.py:30-59)
  double pe_k = pe1(0);
  double pe_k1 = pe1(1);
  double bb0 = (K - 2 > 0) ? 2.0 * (1.0 + DM(0) / DM(1)) : 2.0;
  pp[0] = 0.0;
  pp[1] = (K > 2 ? 3.0 * (pe_k + (DM(0) / DM(1)) * pe_k1) : 3.0 * pe_k) / bb0;
  double bet = bb0;
  for (int k = 1; k <= K - 2; ++k) {
    PF(k + 1 + PF_AHEAD);
    pe_k = pe_k1;
    double grm = DM(k - 1) / DM(k);
    double g = grm / bet;
    double bbk, ddk;
    if (k < K - 2) {
      pe_k1 = pe1(k + 1);
      double grk = DM(k) / DM(k + 1);
      bbk = 2.0 * (1.0 + grk);
      ddk = 3.0 * (pe_k + grk * pe_k1);
    } else {
      bbk = 2.0;
      ddk = 3.0 * pe_k;
    }
    gam[k] = g;
    bet = bbk - g;
    pp[k + 1] = (ddk - pp[k]) / bet;
  }
  // back substitution (sim1_solver.py:60-63)
  for (int k = K - 2; k >= 1; --k) pp[k] = pp[k] - gam[k] * pp[k + 1];
  // edge pressures pem[k] = ptop + sum of dp above, rebuilt by the same
  // running sum as the callers' precompute (no per-level array)
  double pem_run = ptop + DP(0);  // pem[1]
  auto AA = [&](int k, double pem_k) {
    return t1g * 0.5 * (GM(k - 1) + GM(k)) / (DZ(k - 1) + DZ(k)) * (pem_k + pp[k]);
  };
  // w solve (sim1_solver.py:65-90)
  double aak = AA(1, pem_run);
  bet = DM(0) - aak;
  w[0] = (DM(0) * W1(0) + dt * pp[1]) / bet;
  PF(1);
  PF(2);
  for (int k = 1; k <= K - 3; ++k) {
    PF(k + 1 + PF_AHEAD);
    pem_run = pem_run + DP(k);  // pem[k + 1]
    double aak1 = AA(k + 1, pem_run);
    double g = aak / bet;
    gam[k] = g;
    bet = DM(k) - (aak + aak1 + aak * g);
    w[k] = (DM(k) * W1(k) + dt * (pp[k + 1] - pp[k]) - aak * w[k - 1]) / bet;
    aak = aak1;
  }
  {
    int k = K - 2;
    pem_run = pem_run + DP(k);  // pem[K - 1]
    double p1 = t1g * GM(k) / DZ(k) * (pem_run + pp[k + 1]);
    double g = aak / bet;
    gam[k] = g;
    bet = DM(k) - (aak + p1 + aak * g);
    w[k] = (DM(k) * W1(k) + dt * (pp[k + 1] - pp[k]) - p1 * wsr - aak * w[k - 1]) / bet;
  }
  for (int k = K - 3; k >= 0; --k) w[k] = w[k] - gam[k + 1] * w[k + 1];
  // pressure perturbation from the w change (sim1_solver.py:91-95); pp's
  // storage is reused for it
  double* pe = pp;
  pe[0] = 0.0;
  PE_OUT(0, 0.0);
  PF(0);
  PF(1);
  for (int k = 1; k < K; ++k) {
    PF(k + PF_AHEAD);
    pe[k] = pe[k - 1] + DM(k - 1) * (w[k - 1] - W1(k - 1)) * rdt;
    PE_OUT(k, pe[k]);
  }
  // layer-mean perturbation and new dz (sim1_solver.py:96-105), bottom up
  double p1n = 0.0;
  for (int k = K - 2; k >= 0; --k) {
    PF(k - PF_AHEAD);
    double p1;
    if (k == K - 2) {
      p1 = (pe[k] + 2.0 * pe[k + 1]) * 1.0 / 3.0;
    } else {
      double gr = DM(k) / DM(k + 1);
      double bbk = 2.0 * (1.0 + gr);
      p1 = (pe[k] + bbk * pe[k + 1] + gr * pe[k + 2]) * 1.0 / 3.0 - gr * p1n;
    }
    p1n = p1;
    double maxp = (p_fac * DM(k) > p1 + pm[k]) ? p_fac * pm[k] : p1 + pm[k];
    DZ_OUT(k, -DM(k) * RDGAS * PTR(k) * fm::fm_exp((CP3(k) - 1.0) * fm::fm_log(maxp)));
  }
}

struct RiemCArgs {
  double dt2, ptop, p_fac;
  const real *cappa, *hs, *ws, *ptc, *q_con, *delpc;
  real *gz, *pef;
  const real* w3;
};

// RiemannSolverC.__call__ body for one column (riem_solver_c.py:13-64)
template <int NK>
struct RiemC {
  static __device__ __forceinline__ void run(const Dims& d, int t, int i, int j, const RiemCArgs& a) {
    const double dt2 = a.dt2, ptop = a.ptop, p_fac = a.p_fac;
    const real *cappa = a.cappa, *hs = a.hs, *ws = a.ws, *ptc = a.ptc, *q_con = a.q_con, *delpc = a.delpc;
    real *gz = a.gz, *pef = a.pef;
    const real* w3 = a.w3;
    double pm[NK], pp[NK], gam[NK], w[NK];
    const int K = d.nk;
    const idx_t o0 = idx3(d, t, i, j, 0);
    const idx_t sk = d.sk;
    const double t1g = 2.0 * dt2 * dt2;
    const double rdt = 1.0 / dt2;
    // precompute (riem_solver_c.py:13-44); the edge pressures pem are
    // running sums rebuilt where they are used
    double peg_k = ptop;
    for (int k = 0; k < K - 1; ++k) {
      if (k + PF_AHEAD < K) {
        prefetch_l2(delpc + o0 + (k + PF_AHEAD) * sk);
        prefetch_l2(q_con + o0 + (k + PF_AHEAD) * sk);
      }
      const double dmk = __ldg(&delpc[o0 + k * sk]);
      const double peg_next = peg_k + dmk * (1.0 - __ldg(&q_con[o0 + k * sk]));
      pm[k] = (peg_next - peg_k) / fm::fm_log(peg_next / peg_k);
      peg_k = peg_next;
    }
    auto DM = [&](int k) { return __ldg(&delpc[o0 + k * sk]) / GRAV; };
    auto DP = [&](int k) { return (double)__ldg(&delpc[o0 + k * sk]); };
    auto W1 = [&](int k) { return __ldg(&w3[o0 + k * sk]); };
    auto DZ = [&](int k) { return (double)gz[o0 + (k + 1) * sk] - (double)gz[o0 + k * sk]; };
    auto GM = [&](int k) { return 1.0 / (1.0 - __ldg(&cappa[o0 + k * sk])); };
    auto PTR = [&](int k) { return __ldg(&ptc[o0 + k * sk]); };
    auto CP3 = [&](int k) { return (double)__ldg(&cappa[o0 + k * sk]); };
    // finalize (riem_solver_c.py:46-64) fused with the solve's outputs; gz
    // is rewritten bottom up only after its last read as an input
    double pem_pe = ptop;
    auto PE_OUT = [&](int k, double pe) {
      if (k > 0) pem_pe = pem_pe + DP(k - 1);
      pef[o0 + k * sk] = k == 0 ? ptop : pe + pem_pe;
    };
    double g = hs[idx2(d, t, i, j)];
    auto DZ_OUT = [&](int k, double dz) {
      if (k == K - 2) gz[o0 + (K - 1) * sk] = g;
      g = g - dz * GRAV;
      gz[o0 + k * sk] = g;
    };
    auto PF = [&](int k) {
      if (k < 0 || k >= K) return;
      const idx_t o = o0 + k * sk;
      prefetch_l2(delpc + o);
      prefetch_l2(gz + o);
      prefetch_l2(cappa + o);
      prefetch_l2(ptc + o);
      prefetch_l2(w3 + o);
    };
    sim1_column<NK>(K, DM, DP, ptop, W1, DZ, GM, PTR, CP3, pm, pp, gam, w, ws[idx2(d, t, i, j)], dt2, t1g, rdt,
                    p_fac, PE_OUT, DZ_OUT, PF);
  }
};

struct Riem3Args {
  bool last;
  double dt, ptop, p_fac, peln1, ptk;
  const real *cappa, *zs, *wsd;
  real* delz;
  const real *q_con, *delp, *pt;
  real *zh, *pe, *ppe, *pk3, *pk, *peln, *w;
};

// RiemannSolver3.__call__ body for one column (riem_solver3.py:24-103)
template <int NK>
struct Riem3 {
  static __device__ __forceinline__ void run(const Dims& d, int t, int i, int j, const Riem3Args& a) {
    const bool last = a.last;
    const double dt = a.dt, ptop = a.ptop, p_fac = a.p_fac, peln1 = a.peln1, ptk = a.ptk;
    const real *cappa = a.cappa, *zs = a.zs, *wsd = a.wsd, *q_con = a.q_con, *delp = a.delp, *pt = a.pt;
    real *delz = a.delz, *zh = a.zh, *pe = a.pe, *ppe = a.ppe, *pk3 = a.pk3, *pk = a.pk, *peln = a.peln;
    real* w_io = a.w;
    double pm[NK], pp[NK], gam[NK], w[NK];
    const int K = d.nk;
    const idx_t o0 = idx3(d, t, i, j, 0);
    const idx_t sk = d.sk;
    const double t1g = 2.0 * dt * dt;
    const double rdt = 1.0 / dt;
    // precompute (riem_solver3.py:24-67); on the last call peln, pk and pe
    // take their final values here (finalize, riem_solver3.py:70-103)
    double pem_k = ptop, peg_k = ptop, pelng_k = peln1;
    pk3[o0] = ptk;
    if (last) {
      peln[o0] = peln1;
      pk[o0] = ptk;
      pe[o0] = ptop;
    }
    for (int k = 0; k < K - 1; ++k) {
      const idx_t o = o0 + k * sk;
      if (k + PF_AHEAD < K) {
        prefetch_l2(delp + o + PF_AHEAD * sk);
        prefetch_l2(q_con + o + PF_AHEAD * sk);
      }
      const double dmk = delp[o];
      const double pem_n = pem_k + dmk;
      const double peg_n = peg_k + dmk * (1.0 - q_con[o]);
      const double pelng_n = fm::fm_log(peg_n);
      const double peln_n = fm::fm_log(pem_n);
      const double pk3_n = fm::fm_exp(KAPPA * peln_n);
      pk3[o + sk] = pk3_n;
      if (last) {
        peln[o + sk] = peln_n;
        pk[o + sk] = pk3_n;
        pe[o + sk] = pem_n;
      }
      pm[k] = (peg_n - peg_k) / (pelng_n - pelng_k);
      pem_k = pem_n;
      peg_k = peg_n;
      pelng_k = pelng_n;
    }
    auto DM = [&](int k) { return __ldg(&delp[o0 + k * sk]) * RGRAV; };
    auto DP = [&](int k) { return (double)__ldg(&delp[o0 + k * sk]); };
    auto W1 = [&](int k) { return w_io[o0 + k * sk]; };
    auto DZ = [&](int k) { return (double)zh[o0 + (k + 1) * sk] - (double)zh[o0 + k * sk]; };
    auto GM = [&](int k) { return 1.0 / (1.0 - __ldg(&cappa[o0 + k * sk])); };
    auto PTR = [&](int k) { return __ldg(&pt[o0 + k * sk]); };
    auto CP3 = [&](int k) { return (double)__ldg(&cappa[o0 + k * sk]); };
    auto PE_OUT = [&](int k, double v) { ppe[o0 + k * sk] = v; };
    // finalize: zh rebuilt from the new layer depths bottom up, after its
    // last read as an input
    double z = zs[idx2(d, t, i, j)];
    auto DZ_OUT = [&](int k, double dz) {
      if (k == K - 2) zh[o0 + (K - 1) * sk] = z;
      delz[o0 + k * sk] = dz;
      z = z - dz;
      zh[o0 + k * sk] = z;
    };
    auto PF = [&](int k) {
      if (k < 0 || k >= K) return;
      const idx_t o = o0 + k * sk;
      prefetch_l2(delp + o);
      prefetch_l2(zh + o);
      prefetch_l2(cappa + o);
      prefetch_l2(pt + o);
      prefetch_l2(w_io + o);
    };
    sim1_column<NK>(K, DM, DP, ptop, W1, DZ, GM, PTR, CP3, pm, pp, gam, w, wsd[idx2(d, t, i, j)], dt, t1g, rdt,
                    p_fac, PE_OUT, DZ_OUT, PF);
    for (int k = 0; k < K - 1; ++k) w_io[o0 + k * sk] = w[k];
  }
};

// Runs Body<NK>::run over the columns with NK the smallest level bucket >= K.
template <template <int> class Body, typename A>
cudaError_t launch_riemann(const Dims& d, int i0, int i1, int j0, int j1, cudaStream_t s, A args) {
  const int K = d.nk;
  const Dims dd = d;
#define FV3B_RIEM_BUCKET(NK)                                                                             \
  if (K <= NK)                                                                                           \
    return launch_columns(i0, i1, j0, j1, s,                                                            \
                          [=] __device__(int t, int i, int j) { Body<NK>::run(dd, t, i, j, args); });
  FV3B_RIEM_BUCKET(16)
  FV3B_RIEM_BUCKET(32)
  FV3B_RIEM_BUCKET(64)
  FV3B_RIEM_BUCKET(80)
  FV3B_RIEM_BUCKET(96)
  FV3B_RIEM_BUCKET(MAXK)
#undef FV3B_RIEM_BUCKET
  return cudaErrorInvalidValue;
}

}  // namespace fv3b

using namespace fv3b;

extern "C" int fv3b_riem_solver_c(const fv3b_grid_dims* dims, double dt2, double ptop, double p_fac,
                                  const real* cappa, const real* hs, const real* ws,
                                  const real* ptc, const real* q_con, const real* delpc,
                                  real* gz, real* pef, const real* w3, void* stream) {
  FV3B_REQUIRE(dims && cappa && hs && ws && ptc && q_con && delpc && gz && pef && w3,
               "fv3b_riem_solver_c: null argument");
  FV3B_REQUIRE(dims_fit(dims), "fv3b_riem_solver_c: a 3-D field of the six tiles must hold fewer than 2^31 elements");
  Dims d = make_dims(dims);
  FV3B_REQUIRE(d.nk <= MAXK && d.nk >= 3, "fv3b_riem_solver_c: npz out of range (2..127)");
  RiemCArgs a{dt2, ptop, p_fac, cappa, hs, ws, ptc, q_con, delpc, gz, pef, w3};
  FV3B_CHECK(launch_riemann<RiemC>(d, d.isc - 1, d.iec + 2, d.jsc - 1, d.jec + 2, (cudaStream_t)stream, a));
  return FV3B_OK;
}

// RiemannSolver3.__call__ (riem_solver3.py:145-242): precompute (24-67),
// Sim1 solve, finalize (70-103) on the compute-domain columns, interface
// levels 0..npz.
extern "C" int fv3b_riem_solver3(const fv3b_grid_dims* dims, int last_call, double dt, double ptop, double p_fac,
                                 const real* cappa, const real* zs, const real* wsd, real* delz,
                                 const real* q_con, const real* delp, const real* pt, real* zh, real* pe,
                                 real* ppe, real* pk3, real* pk, real* peln, real* w, void* stream) {
  FV3B_REQUIRE(dims && cappa && zs && wsd && delz && q_con && delp && pt && zh && pe && ppe && pk3 && pk && peln && w,
               "fv3b_riem_solver3: null argument");
  FV3B_REQUIRE(dims_fit(dims), "fv3b_riem_solver3: a 3-D field of the six tiles must hold fewer than 2^31 elements");
  Dims d = make_dims(dims);
  FV3B_REQUIRE(d.nk <= MAXK && d.nk >= 3, "fv3b_riem_solver3: npz out of range (2..127)");
  const double peln1 = log(ptop);
  const double ptk = exp(KAPPA * peln1);
  Riem3Args a{last_call != 0, dt, ptop, p_fac, peln1, ptk, cappa, zs, wsd, delz, q_con, delp, pt, zh, pe, ppe, pk3,
              pk, peln, w};
  FV3B_CHECK(launch_riemann<Riem3>(d, d.isc, d.iec + 1, d.jsc, d.jec + 1, (cudaStream_t)stream, a));
  return FV3B_OK;
}

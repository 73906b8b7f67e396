// Vertically implicit acoustic solvers: RiemannSolverC and RiemannSolver3
// with the shared Sim1 tridiagonal solve.
//
// One thread owns one (tile, i, j) column and walks it top to bottom and
// back; neighbouring threads own neighbouring i, so every level load/store
// is a coalesced row access.  A column keeps three per-level work arrays in
// the thread's local memory: the layer-mean pressures pm, the elimination
// factors gam, and one array that holds, in turn, the pressure solution
// pp, the new w and the pressure perturbation pe (each slot is overwritten
// only after its last read).  The solve is a long chain of dependent FP64
// operations (seven exp/log per level), so it needs many columns in flight
// to hide latency; the arrays therefore stay in local memory (L1/L2) rather
// than in shared memory, which would cap the columns in flight (measured
// three times slower with five 32-column blocks per SM).  The edge
// pressures are running sums rebuilt where they are used, everything else
// is re-read from the input fields or computed on the fly, and the outputs
// are written in the pass that produces them.  The arrays are sized by a
// compile-time level bucket >= npz+1, so an L79 column keeps 1.9 KB.
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

// A per-level work array of one column in the thread's local memory.
struct ColArr {
  double* p;
  __device__ __forceinline__ double& operator[](int k) const { return p[k]; }
};

// Per-column inputs of the Sim1 solve (fv3core/stencils/sim1_solver.py:11-101).
// K = number of interface levels (npz + 1).  DM(k): delta p / g; DP(k):
// delta p, whose running sums from ptop are the edge pressures pem; W1(k): w
// at the start; DZ(k): layer depth at the start (negative); GM, PTR, CP3:
// 1/(1-cappa), pt, cappa per level; pm: layer-mean pressure.  gam and pw are
// the shared-memory work arrays (pw holds pp, then the new w, then pe
// shifted down one slot).  Results: the new w through W_OUT(k, value), k =
// 0 .. K-2, pe[0..K-1] (pressure perturbation, through PE_OUT(k, value) in
// increasing k) and the new layer depths through DZ_OUT(k, value) for
// k = K-2 .. 0 (bottom up).
template <int NK, typename DMF, typename DPF, typename W1F, typename DZF, typename GMF, typename PTRF,
          typename CP3F, typename PEOUT, typename DZOUT, typename WOUT, typename PFF>
__device__ __forceinline__ void sim1_column(int K, DMF DM, DPF DP, double ptop, W1F W1, DZF DZ, GMF GM, PTRF PTR,
                                            CP3F CP3, const double* pm, ColArr pw, ColArr gam, double wsr,
                                            double dt, double t1g, double rdt, double p_fac, PEOUT PE_OUT,
                                            DZOUT DZ_OUT, WOUT W_OUT, PFF PF) {
  // pe = exp(gm*log(-dm/dz*Rd*ptr)) - pm   (sim1_solver.py:27-29), on the fly
  auto pe1 = [&](int k) { return fm::fm_exp(GM(k) * fm::fm_log(-DM(k) / DZ(k) * RDGAS * PTR(k))) - pm[k]; };
  // forward elimination of the pressure system (sim1_solver.py:30-59); pw = pp
  double pe_k = pe1(0);
  double pe_k1 = pe1(1);
  double bb0 = (K - 2 > 0) ? 2.0 * (1.0 + DM(0) / DM(1)) : 2.0;
  pw[0] = 0.0;
  double pp_k = (K > 2 ? 3.0 * (pe_k + (DM(0) / DM(1)) * pe_k1) : 3.0 * pe_k) / bb0;
  pw[1] = pp_k;
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
    pp_k = (ddk - pp_k) / bet;
    pw[k + 1] = pp_k;
  }
  // back substitution (sim1_solver.py:60-63)
  double pp_next = pw[K - 1];
  for (int k = K - 2; k >= 1; --k) {
    pp_next = pw[k] - gam[k] * pp_next;
    pw[k] = pp_next;
  }
  // edge pressures pem[k] = ptop + sum of dp above, rebuilt by the same
  // running sum as the callers' precompute (no per-level array)
  double pem_run = ptop + DP(0);  // pem[1]
  auto AA = [&](int k, double pem_k, double pp_kk) {
    return t1g * 0.5 * (GM(k - 1) + GM(k)) / (DZ(k - 1) + DZ(k)) * (pem_k + pp_kk);
  };
  // w solve (sim1_solver.py:65-90); w[k] replaces pp[k] in pw once pp[k]
  // has had its last read
  double pp_c = pw[1];  // pp[k + 1] of the step below
  double aak = AA(1, pem_run, pp_c);
  bet = DM(0) - aak;
  double w_prev = (DM(0) * W1(0) + dt * pp_c) / bet;
  pw[0] = w_prev;
  PF(1);
  PF(2);
  for (int k = 1; k <= K - 3; ++k) {
    PF(k + 1 + PF_AHEAD);
    pem_run = pem_run + DP(k);  // pem[k + 1]
    const double pp_k0 = pp_c, pp_k1 = pw[k + 1];
    double aak1 = AA(k + 1, pem_run, pp_k1);
    double g = aak / bet;
    gam[k] = g;
    bet = DM(k) - (aak + aak1 + aak * g);
    w_prev = (DM(k) * W1(k) + dt * (pp_k1 - pp_k0) - aak * w_prev) / bet;
    pw[k] = w_prev;
    pp_c = pp_k1;
    aak = aak1;
  }
  {
    int k = K - 2;
    pem_run = pem_run + DP(k);  // pem[K - 1]
    const double pp_k1 = pw[k + 1];
    double p1 = t1g * GM(k) / DZ(k) * (pem_run + pp_k1);
    double g = aak / bet;
    gam[k] = g;
    bet = DM(k) - (aak + p1 + aak * g);
    w_prev = (DM(k) * W1(k) + dt * (pp_k1 - pp_c) - p1 * wsr - aak * w_prev) / bet;
    pw[k] = w_prev;
  }
  for (int k = K - 3; k >= 0; --k) {
    w_prev = pw[k] - gam[k + 1] * w_prev;
    pw[k] = w_prev;
  }
  // pressure perturbation from the w change (sim1_solver.py:91-95): pe[k]
  // goes to slot k - 1 of pw, right after that slot's w has been read and
  // handed out
  double pe_prev = 0.0;
  PE_OUT(0, 0.0);
  PF(0);
  PF(1);
  for (int k = 1; k < K; ++k) {
    PF(k + PF_AHEAD);
    const double wk = pw[k - 1];
    pe_prev = pe_prev + DM(k - 1) * (wk - W1(k - 1)) * rdt;
    W_OUT(k - 1, wk);
    pw[k - 1] = pe_prev;
    PE_OUT(k, pe_prev);
  }
  auto PE = [&](int k) { return k == 0 ? 0.0 : (double)pw[k - 1]; };
  // layer-mean perturbation and new dz (sim1_solver.py:96-105), bottom up
  double p1n = 0.0;
  for (int k = K - 2; k >= 0; --k) {
    PF(k - PF_AHEAD);
    double p1;
    if (k == K - 2) {
      p1 = (PE(k) + 2.0 * PE(k + 1)) * 1.0 / 3.0;
    } else {
      double gr = DM(k) / DM(k + 1);
      double bbk = 2.0 * (1.0 + gr);
      p1 = (PE(k) + bbk * PE(k + 1) + gr * PE(k + 2)) * 1.0 / 3.0 - gr * p1n;
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
  static __device__ __forceinline__ void run(const Dims& d, int t, int i, int j, const RiemCArgs& a, ColArr pw,
                                             ColArr gam) {
    const double dt2 = a.dt2, ptop = a.ptop, p_fac = a.p_fac;
    const real *cappa = a.cappa, *hs = a.hs, *ws = a.ws, *ptc = a.ptc, *q_con = a.q_con, *delpc = a.delpc;
    real *gz = a.gz, *pef = a.pef;
    const real* w3 = a.w3;
    double pm[NK];
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
    sim1_column<NK>(K, DM, DP, ptop, W1, DZ, GM, PTR, CP3, pm, pw, gam, ws[idx2(d, t, i, j)], dt2, t1g, rdt,
                    p_fac, PE_OUT, DZ_OUT, [](int, double) {}, PF);
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
  static __device__ __forceinline__ void run(const Dims& d, int t, int i, int j, const Riem3Args& a, ColArr pw,
                                             ColArr gam) {
    const bool last = a.last;
    const double dt = a.dt, ptop = a.ptop, p_fac = a.p_fac, peln1 = a.peln1, ptk = a.ptk;
    const real *cappa = a.cappa, *zs = a.zs, *wsd = a.wsd, *q_con = a.q_con, *delp = a.delp, *pt = a.pt;
    real *delz = a.delz, *zh = a.zh, *pe = a.pe, *ppe = a.ppe, *pk3 = a.pk3, *pk = a.pk, *peln = a.peln;
    real* w_io = a.w;
    double pm[NK];
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
    // the new w replaces the old after the old value's last read (W1 of the
    // same level in the pressure-perturbation loop)
    auto W_OUT = [&](int k, double wk) { w_io[o0 + k * sk] = wk; };
    sim1_column<NK>(K, DM, DP, ptop, W1, DZ, GM, PTR, CP3, pm, pw, gam, wsd[idx2(d, t, i, j)], dt, t1g, rdt,
                    p_fac, PE_OUT, DZ_OUT, W_OUT, PF);
  }
};

// One thread per column; the work arrays in local memory.
template <int NK, template <int> class Body, typename A>
cudaError_t launch_riemann_nk(const Dims& d, int i0, int i1, int j0, int j1, cudaStream_t s, const A& args) {
  const Dims dd = d;
  return launch_columns(i0, i1, j0, j1, s, [=] __device__(int t, int i, int j) {
    double pw[NK], gam[NK];
    Body<NK>::run(dd, t, i, j, args, ColArr{pw}, ColArr{gam});
  });
}

// Runs Body<NK>::run over the columns with NK the smallest level bucket >= K.
template <template <int> class Body, typename A>
cudaError_t launch_riemann(const Dims& d, int i0, int i1, int j0, int j1, cudaStream_t s, A args) {
  const int K = d.nk;
  if (K <= 16) return launch_riemann_nk<16, Body>(d, i0, i1, j0, j1, s, args);
  if (K <= 32) return launch_riemann_nk<32, Body>(d, i0, i1, j0, j1, s, args);
  if (K <= 64) return launch_riemann_nk<64, Body>(d, i0, i1, j0, j1, s, args);
  if (K <= 80) return launch_riemann_nk<80, Body>(d, i0, i1, j0, j1, s, args);
  if (K <= 96) return launch_riemann_nk<96, Body>(d, i0, i1, j0, j1, s, args);
  if (K <= MAXK) return launch_riemann_nk<MAXK, Body>(d, i0, i1, j0, j1, s, args);
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

// The step preamble and epilogue of DynamicalCore.step_dynamics
// (fv3core/stencils/fv_dynamics.py:54-169) around the acoustic loop:
//
// * fv3b_compute_preamble: fv_setup (moist_cv.py:197-228, moist_phys, nwat
//   = 6) and pt_adjust (fv_dynamics.py:32-34), one pointwise pass;
// * fv3b_post_remap: set_omega (fv_dynamics.py:37-39), then, for nf_omega >
//   0, the omega halo update and the del-2 filter with 0.18 da_min
//   (fv_dynamics.py:109-133);
// * fv3b_adjust_negative_tracers: AdjustNegativeTracerMixingRatio
//   (neg_adj3.py:293-372), every column in one thread: the pointwise fixes
//   of fix_neg_water, then fillq on graupel and rain, fix_water_vapor_down
//   and fix_neg_cloud, each a walk down and up the column;
// * fv3b_cubed_to_latlon: CubedToLatLon (c2l_ord.py:75-141), order 4 with
//   its vector halo update, or order 2.
//
// Every stencil runs on the compute domain and the npz layers, as the
// reference builds them.  Statement order and branch structure follow the
// reference, and exp / log are the library's own (fmath.h), so FP64 results
// agree with the oracle running the same functions bit for bit.
#include <math.h>

#include "ctx.cuh"
#include "fmath.h"
#include "halo_ops.cuh"
#include "stencil.cuh"

using namespace fv3b;

namespace {

// fv3core/utils/global_constants.py
constexpr double RDGAS_D = 287.05, RVGAS_D = 461.50, GRAV_D = 9.80665, CP_AIR_D = 1004.6;
constexpr double CV_AIR_D = CP_AIR_D - RDGAS_D, RDG_D = -RDGAS_D / GRAV_D, ZVIR_D = RVGAS_D / RDGAS_D - 1.0;
constexpr double HLV_D = 2.5e6, HLF_D = 3.3358e5, CV_VAP_D = 3.0 * RVGAS_D, C_ICE_D = 1972.0, C_LIQ_D = 4.1855e3;
constexpr double TICE_D = 273.16, DC_ICE_D = C_LIQ_D - C_ICE_D, LI0_D = HLF_D - DC_ICE_D * TICE_D;

// the reference's "a if a < b else b" and "0.0 if 0.0 > a else a"
__device__ __forceinline__ real sel_lt(real a, real b) { return a < b ? a : b; }
__device__ __forceinline__ real pos0(real a) { return RC(0.0) > a ? RC(0.0) : a; }

// fix_negative_ice (neg_adj3.py:12-55) at one point
__device__ __forceinline__ void fix_negative_ice(real& qvapor, real& qice, real& qsnow, real& qgraupel, real& qrain,
                                                 real& qliquid, real& pt, real lcpk, real icpk) {
  const real qsum = qice + qsnow;
  if (qsum > RC(0.0)) {
    if (qice < RC(0.0)) {
      qice = RC(0.0);
      qsnow = qsum;
    } else if (qsnow < RC(0.0)) {
      qsnow = RC(0.0);
      qice = qsum;
    }
  } else {
    qice = RC(0.0);
    qsnow = RC(0.0);
    qgraupel = qgraupel + qsum;
  }
  if (qgraupel < RC(0.0)) {
    real dq = sel_lt(qsnow, -qgraupel);
    qsnow = qsnow - dq;
    qgraupel = qgraupel + dq;
    if (qgraupel < RC(0.0)) {
      dq = sel_lt(qice, -qgraupel);
      qice = qice - dq;
      qgraupel = qgraupel + dq;
    }
  }
  if (qgraupel < RC(0.0) && qrain > RC(0.0)) {
    const real dq = sel_lt(qrain, -qgraupel);
    qgraupel = qgraupel + dq;
    qliquid = qliquid - dq;
    pt = pt + dq * icpk;
  }
  if (qgraupel < RC(0.0) && qliquid > RC(0.0)) {
    const real dq = sel_lt(qliquid, -qgraupel);
    qgraupel = qgraupel + dq;
    qliquid = qliquid - dq;
    pt = pt + dq * icpk;
  }
  if (qgraupel < RC(0.0) && qvapor > RC(0.0)) {
    const real dq = sel_lt(RC(0.999) * qvapor, -qgraupel);
    qgraupel = qgraupel + dq;
    qvapor = qvapor - dq;
    pt = pt + dq * (icpk + lcpk);
  }
}

// fix_negative_liq (neg_adj3.py:58-98) at one point
__device__ __forceinline__ void fix_negative_liq(real& qvapor, real& qice, real& qsnow, real& qgraupel, real& qrain,
                                                 real& qliquid, real& pt, real lcpk, real icpk) {
  const real qsum = qliquid + qrain;
  const real pos_qgraupel = pos0(qgraupel);
  if (qsum > RC(0.0)) {
    if (qrain < RC(0.0)) {
      qrain = RC(0.0);
      qliquid = qsum;
    } else if (qliquid < RC(0.0)) {
      qliquid = RC(0.0);
      qrain = qsum;
    }
  } else {
    qliquid = RC(0.0);
    real qrain_tmp = qsum;
    real dq = sel_lt(pos_qgraupel, -qrain_tmp);
    qrain_tmp = qrain_tmp + dq;
    qgraupel = qgraupel - dq;
    pt = pt - dq * icpk;
    if (qrain < RC(0.0)) {
      dq = sel_lt(qice + qsnow, -qrain_tmp);
      qrain_tmp = qrain_tmp + dq;
      const real dq1 = sel_lt(dq, qsnow);
      qsnow = qsnow - dq1;
      qice = qice + dq1 - dq;
      pt = pt - dq * icpk;
    }
    qrain = qrain_tmp;
    if (qrain < RC(0.0) && qvapor > RC(0.0)) {
      dq = sel_lt(RC(0.999) * qvapor, -qrain);
      qvapor = qvapor - dq;
      qrain = qrain + dq;
      pt = pt + dq * lcpk;
    }
  }
}

// A column of one field: at(k) is level k.
struct Col {
  real* p;
  idx_t sk;
  __device__ __forceinline__ real& operator[](int k) const { return p[k * sk]; }
};

// fillq (neg_adj3.py:67-88) on one column
__device__ __forceinline__ void fillq(const Col& q, const Col& dp, int nz) {
  real sum1 = RC(0.0), sum2 = RC(0.0);
  for (int k = 0; k < nz; ++k)
    if (q[k] > 0) sum1 = sum1 + q[k] * dp[k];
  for (int k = nz - 1; k >= 0; --k) {
    const real qk = q[k], dk = dp[k];
    if (qk < RC(0.0) && sum1 >= 0) {
      const real dq = sel_lt(sum1, -qk * dk);
      sum1 = sum1 - dq;
      sum2 = sum2 + dq;
      q[k] = qk + dq / dk;
    }
  }
  for (int k = nz - 1; k >= 0; --k) {
    const real qk = q[k], dk = dp[k];
    if (qk > RC(0.0) && sum1 >= RC(1e-12) && sum2 > 0) {
      const real dq = sel_lt(sum2, qk * dk);
      sum2 = sum2 - dq;
      q[k] = qk - dq / dk;
    }
  }
}

constexpr int MAXNZ = 128;

// fix_water_vapor_down (neg_adj3.py:240-291) on one column.  The
// reference's temporary dp_bot is written on the bottom level only and read
// on the others when the bottom layer is still negative after the first
// walk; here it is the bottom layer's thickness on every level, as in the
// column routine this stencil restates (neg_adj3.py:196-208).
__device__ __forceinline__ void fix_water_vapor_down(const Col& q, const Col& dp, int nz) {
  real upper_fix[MAXNZ], lower_fix[MAXNZ];
  for (int k = 0; k < nz; ++k) upper_fix[k] = lower_fix[k] = RC(0.0);
  if (q[0] < RC(0.0)) q[0] = RC(0.0);
  if (q[0] < 0) q[1] = q[1] + q[0] * dp[0] / dp[1];
  for (int k = 1; k < nz - 1; ++k) {
    real dq = q[k - 1] * dp[k - 1];
    if (lower_fix[k - 1] != 0) q[k] = q[k] + lower_fix[k - 1] / dp[k];
    if (q[k] < 0 && q[k - 1] > 0) {
      dq = sel_lt(dq, -q[k] * dp[k]);
      upper_fix[k] = dq;
      q[k] = q[k] + dq / dp[k];
    }
    if (q[k] < 0) {
      lower_fix[k] = q[k] * dp[k];
      q[k] = RC(0.0);
    }
  }
  for (int k = 0; k < nz - 2; ++k)
    if (upper_fix[k + 1] != 0) q[k] = q[k] - upper_fix[k + 1] / dp[k];
  const int kb = nz - 1;
  if (lower_fix[kb - 1] > 0) q[kb] = q[kb] + lower_fix[kb] / dp[kb];
  upper_fix[kb] = q[kb];
  const real dp_bot = dp[kb];
  for (int k = nz - 2; k >= 0; --k) {
    real dq = q[k] * dp[k];
    if (upper_fix[k + 1] < 0 && q[k] > 0) {
      if (dq >= -upper_fix[k + 1] * dp_bot) dq = -upper_fix[k + 1] * dp_bot;
      q[k] = q[k] - dq / dp[k];
      upper_fix[k] = upper_fix[k + 1] + dq / dp_bot;
    } else {
      upper_fix[k] = upper_fix[k + 1];
    }
  }
  // the bottom value carried up by the walk above comes back down
  q[kb] = upper_fix[0];
}

// fix_neg_cloud (neg_adj3.py:148-173) on one column
__device__ __forceinline__ void fix_neg_cloud(const Col& dp, const Col& q, int nz) {
  for (int k = 1; k < nz - 1; ++k)
    if (q[k - 1] < RC(0.0)) q[k] = q[k] + q[k - 1] * dp[k - 1] / dp[k];
  for (int k = 1; k < nz - 1; ++k)
    if (q[k] < RC(0.0)) q[k] = RC(0.0);
  int k = nz - 2;
  if (q[k + 1] < RC(0.0) && q[k] > 0) {
    const real dq = sel_lt(-q[k] * dp[k], q[k + 1] * dp[k + 1]);
    q[k] = q[k] - dq / dp[k];
  }
  k = nz - 1;
  if (q[k] < 0 && q[k - 1] > RC(0.0)) {
    const real dq = sel_lt(-q[k] * dp[k], q[k - 1] * dp[k - 1]);
    q[k] = q[k] + dq / dp[k];
    q[k] = pos0(q[k]);
  }
}

}  // namespace

extern "C" int fv3b_compute_preamble(fv3b_ctx* ctx, const real* qvapor, const real* qliquid, const real* qrain,
                                     const real* qsnow, const real* qice, const real* qgraupel, real* q_con,
                                     real* cvm, real* pkz, real* pt, real* cappa, const real* delp,
                                     const real* delz, real* dp1, void* stream) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && qvapor && qliquid && qrain && qsnow && qice && qgraupel && q_con && cvm && pkz && pt && cappa &&
                   delp && delz && dp1,
               "fv3b_compute_preamble: null argument");
  const Dims d = ctx->d;
  const real cv_air = RC(CV_AIR_D), cv_vap = RC(CV_VAP_D), c_liq = RC(C_LIQ_D), c_ice = RC(C_ICE_D);
  const real zvir = RC(ZVIR_D), rdgas = RC(RDGAS_D), rdg = RC(RDG_D);
  FV3B_CHECK(launch_box(Box{d.isc, d.iec + 1, d.jsc, d.jec + 1, 0, d.nz}, (cudaStream_t)stream,
                        [=] __device__(int t, int i, int j, int k) {
                          PT_SETUP(d, t, k);
                          // fv_setup: moist_cv_nwat6_fn, then cappa and pkz
                          const real qv = F3(qvapor, i, j);
                          const real ql = F3(qliquid, i, j) + F3(qrain, i, j);
                          const real qs = F3(qice, i, j) + F3(qsnow, i, j) + F3(qgraupel, i, j);
                          const real gz = ql + qs;
                          const real cv = (RC(1.0) - (qv + gz)) * cv_air + qv * cv_vap + ql * c_liq + qs * c_ice;
                          W3(cvm, i, j) = cv;
                          W3(q_con, i, j) = gz;
                          const real d1 = zvir * qv;
                          W3(dp1, i, j) = d1;
                          const real ca = rdgas / (rdgas + cv / (RC(1.0) + d1));
                          W3(cappa, i, j) = ca;
                          const real p0 = F3(pt, i, j);
                          const real pk = fm::fm_exp(ca * fm::fm_log(rdg * F3(delp, i, j) * p0 * (RC(1.0) + d1) *
                                                                     (RC(1.0) - gz) / F3(delz, i, j)));
                          W3(pkz, i, j) = pk;
                          // pt_adjust
                          W3(pt, i, j) = p0 * (RC(1.0) + d1) * (RC(1.0) - gz) / pk;
                        }));
  return FV3B_OK;
}

extern "C" int fv3b_post_remap(fv3b_ctx* ctx, const real* delp, const real* delz, const real* w, real* omga,
                               int nf_omega, void* stream) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && delp && delz && w && omga, "fv3b_post_remap: null argument");
  FV3B_REQUIRE(nf_omega >= 0, "fv3b_post_remap: nf_omega must be >= 0");
  const Dims d = ctx->d;
  cudaStream_t st = (cudaStream_t)stream;
  // set_omega
  FV3B_CHECK(launch_box(Box{d.isc, d.iec + 1, d.jsc, d.jec + 1, 0, d.nz}, st, [=] __device__(int t, int i, int j,
                                                                                               int k) {
    PT_SETUP(d, t, k);
    W3(omga, i, j) = F3(delp, i, j) / F3(delz, i, j) * F3(w, i, j);
  }));
  if (nf_omega > 0) {
    FV3B_CHECK(halo_scalars(d, &omga, 1, 1, d.h, d.nz, st));
    const int rc = fv3b_del2cubed(ctx, omga, 0.18 * ctx->m.da_min, nf_omega, stream);
    if (rc != FV3B_OK) return rc;
  }
  return FV3B_OK;
}

extern "C" int fv3b_adjust_negative_tracers(fv3b_ctx* ctx, real* qvapor, real* qliquid, real* qrain, real* qsnow,
                                            real* qice, real* qgraupel, real* qcld, real* pt, const real* delp,
                                            const real* delz, const real* peln, int hydrostatic, void* stream) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && qvapor && qliquid && qrain && qsnow && qice && qgraupel && qcld && pt && delp && delz && peln,
               "fv3b_adjust_negative_tracers: null argument");
  if (hydrostatic) {
    set_last_error_msg("fv3b_adjust_negative_tracers: Unimplemented namelist hydrostatic=True");
    return FV3B_ERR_UNSUPPORTED;
  }
  const Dims d = ctx->d;
  FV3B_REQUIRE(d.nz >= 3 && d.nz <= MAXNZ, "fv3b_adjust_negative_tracers: npz must be 3..128");
  const real d0_vap = RC(CV_VAP_D - C_LIQ_D);
  const real lv00 = RC(HLV_D - (CV_VAP_D - C_LIQ_D) * TICE_D);
  const real cv_air = RC(CV_AIR_D), cv_vap = RC(CV_VAP_D), c_liq = RC(C_LIQ_D), c_ice = RC(C_ICE_D);
  const real li0 = RC(LI0_D), dc_ice = RC(DC_ICE_D);
  const int nz = d.nz;
  FV3B_CHECK(launch_columns(d.isc, d.iec + 1, d.jsc, d.jec + 1, (cudaStream_t)stream, [=] __device__(int t, int i,
                                                                                                  int j) {
    const idx_t o = idx3(d, t, i, j, 0), sk = d.sk;
    // fix_neg_water (neg_adj3.py:101-145), pointwise
    for (int k = 0; k < nz; ++k) {
      const idx_t ok = o + k * sk;
      real qv = qvapor[ok], ql = qliquid[ok], qr = qrain[ok], qs = qsnow[ok], qi = qice[ok], qg = qgraupel[ok];
      real p = pt[ok];
      const real q_liq = pos0(ql + qr);
      const real q_sol = pos0(qi + qs);
      const real cpm = (RC(1.0) - (qv + q_liq + q_sol)) * cv_air + qv * cv_vap + q_liq * c_liq + q_sol * c_ice;
      const real lcpk = (lv00 + d0_vap * p) / cpm;
      const real icpk = (li0 + dc_ice * p) / cpm;
      fix_negative_ice(qv, qi, qs, qg, qr, ql, p, lcpk, icpk);
      fix_negative_liq(qv, qi, qs, qg, qr, ql, p, lcpk, icpk);
      qvapor[ok] = qv;
      qliquid[ok] = ql;
      qrain[ok] = qr;
      qsnow[ok] = qs;
      qice[ok] = qi;
      qgraupel[ok] = qg;
      pt[ok] = p;
    }
    const Col dp{const_cast<real*>(delp) + o, sk};
    fillq(Col{qgraupel + o, sk}, dp, nz);
    fillq(Col{qrain + o, sk}, dp, nz);
    fix_water_vapor_down(Col{qvapor + o, sk}, dp, nz);
    fix_neg_cloud(dp, Col{qcld + o, sk}, nz);
  }));
  return FV3B_OK;
}

extern "C" int fv3b_cubed_to_latlon(fv3b_ctx* ctx, real* u, real* v, const real* a11, const real* a12,
                                    const real* a21, const real* a22, real* ua, real* va, int order, void* stream) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && u && v && a11 && a12 && a21 && a22 && ua && va, "fv3b_cubed_to_latlon: null argument");
  FV3B_REQUIRE(order == 2 || order == 4, "fv3b_cubed_to_latlon: order must be 2 or 4");
  const Dims d = ctx->d;
  const fv3b_metrics g = ctx->m;
  cudaStream_t st = (cudaStream_t)stream;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  if (order == 4) {
    // vector halo update of the D-grid winds, then ord4_transform
    // (c2l_ord.py:38-72) on the compute domain
    FV3B_CHECK(halo_vector(d, u, v, false, d.nz, st));
    FV3B_CHECK(launch_box(Box{s, e + 1, js, je + 1, 0, d.nz}, st, [=] __device__(int t, int i, int j, int k) {
      PT_SETUP(d, t, k);
      const real c1 = RC(1.125), c2 = RC(-0.125);
      real utmp = c2 * (F3(u, i, j - 1) + F3(u, i, j + 2)) + c1 * (F3(u, i, j) + F3(u, i, j + 1));
      real vtmp = c2 * (F3(v, i - 1, j) + F3(v, i + 2, j)) + c1 * (F3(v, i, j) + F3(v, i + 1, j));
      const bool row = j == js || j == je, col = i == s || i == e;
      if (row || col) {
        vtmp = RC(2.0) * ((F3(v, i, j) * F2(g.dy, i, j)) + (F3(v, i + 1, j) * F2(g.dy, i + 1, j))) /
               (F2(g.dy, i, j) + F2(g.dy, i + 1, j));
        utmp = RC(2.0) * (F3(u, i, j) * F2(g.dx, i, j) + F3(u, i, j + 1) * F2(g.dx, i, j + 1)) /
               (F2(g.dx, i, j) + F2(g.dx, i, j + 1));
      }
      W3(ua, i, j) = F2(a11, i, j) * utmp + F2(a12, i, j) * vtmp;
      W3(va, i, j) = F2(a21, i, j) * utmp + F2(a22, i, j) * vtmp;
    }));
  } else {
    // c2l_ord2 (c2l_ord.py:17-35) on the compute domain plus one halo row
    FV3B_CHECK(launch_box(Box{s - 1, e + 2, js - 1, je + 2, 0, d.nz}, st, [=] __device__(int t, int i, int j, int k) {
      PT_SETUP(d, t, k);
      const real wu0 = F3(u, i, j) * F2(g.dx, i, j), wu1 = F3(u, i, j + 1) * F2(g.dx, i, j + 1);
      const real wv0 = F3(v, i, j) * F2(g.dy, i, j), wv1 = F3(v, i + 1, j) * F2(g.dy, i + 1, j);
      const real u1 = RC(2.0) * (wu0 + wu1) / (F2(g.dx, i, j) + F2(g.dx, i, j + 1));
      const real v1 = RC(2.0) * (wv0 + wv1) / (F2(g.dy, i, j) + F2(g.dy, i + 1, j));
      W3(ua, i, j) = F2(a11, i, j) * u1 + F2(a12, i, j) * v1;
      W3(va, i, j) = F2(a21, i, j) * u1 + F2(a22, i, j) * v1;
    }));
  }
  return FV3B_OK;
}

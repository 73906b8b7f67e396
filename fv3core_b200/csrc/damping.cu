// Damping stages of the acoustic substep:
//   RayleighDamping (fv3core/stencils/ray_fast.py), the fast Rayleigh
//     friction on the top layers;
//   HyperdiffusionDamping (fv3core/stencils/del2cubed.py), the del-2
//     filter of the dissipation heat source;
//   compute_pkz_tempadjust (fv3core/stencils/temperature_adjust.py), the
//     temperature change from that heat;
// and the adjoints of the Rayleigh damping (ray_adjoint.h), of the del-2
// filter (del2cubed_adjoint.h) and of the temperature adjustment
// (tempadjust_adjoint.h).
#include <math.h>

#include <vector>

#include "corners.cuh"
#include "ctx.cuh"
#include "del2cubed_adjoint.h"
#include "fmath.h"
#include "ray_adjoint.h"
#include "stencil.cuh"
#include "tempadjust_adjoint.h"

using namespace fv3b;

namespace {
constexpr double PI = 3.1415926535897931;
constexpr double SDAY = 86400.0;
constexpr real GRAV = RC(9.80665);
constexpr real RDGAS = RC(287.05);
constexpr real CP_AIR = RC(1004.6);
constexpr real CV_AIR = CP_AIR - RDGAS;
constexpr real RDG = -RDGAS / GRAV;
}  // namespace

// RayleighDamping.__call__ (ray_fast.py:169-192) with ray_fast_wind_compute
// (48-128).  dp and pfull are host arrays of npz layer values.  The
// per-level factors depend only on (dt, ptop, dp, pfull) and are uploaded
// when those change.  In each column the friction removed from the levels
// with pfull < rf_cutoff is summed top down and given back, divided by the
// accumulated layer mass, to the levels with pfull < rf_cutoff +
// min(100, 10 ptop); pfull increases with k, so both level sets are
// prefixes [0, k_rf) and [0, k_nudge).
extern "C" int fv3b_ray_fast(fv3b_ctx* ctx, real* u, real* v, real* w, const double* dp, const double* pfull,
                             double dt, double ptop, double rf_cutoff, double tau, int hydrostatic, void* stream) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && u && v && w && dp && pfull, "fv3b_ray_fast: null argument");
  const Dims d = ctx->d;
  const int nz = d.nz;
  cudaStream_t st = (cudaStream_t)stream;
  RayState& rs = ctx->ray;
  bool same = rs.ready && rs.dt == dt && rs.ptop == ptop && rs.rf_cutoff == rf_cutoff && rs.tau == tau;
  for (int k = 0; same && k < nz; ++k) same = rs.dp[k] == dp[k] && rs.pfull[k] == pfull[k];
  if (!same) {
    for (int k = 1; k < nz; ++k)
      FV3B_REQUIRE(pfull[k] >= pfull[k - 1], "fv3b_ray_fast: pfull must increase with k");
    const double nudge = rf_cutoff + (100.0 < 10.0 * ptop ? 100.0 : 10.0 * ptop);
    const double tau0 = tau * SDAY;
    std::vector<double> c((size_t)2 * MAXLEV, 0.0);
    double *rf = c.data(), *dm = c.data() + MAXLEV;
    int k_rf = 0, k_nudge = 0;
    while (k_rf < nz && pfull[k_rf] < rf_cutoff) ++k_rf;
    while (k_nudge < nz && pfull[k_nudge] < nudge) ++k_nudge;
    if (k_rf == 0) k_nudge = 0;  // nothing removed, nothing given back
    for (int k = 0; k < k_rf; ++k) {
      double sn = sin(0.5 * PI * log(rf_cutoff / pfull[k]) / log(rf_cutoff / ptop));
      double rfv = dt / tau0 * (sn * sn);
      rf[k] = 1.0 / (1.0 + rfv);
    }
    // layer mass accumulated down to the last nudged level, then copied up
    if (k_nudge > 0) {
      dm[0] = dp[0];
      for (int k = 1; k < k_nudge; ++k) dm[k] = dm[k - 1] + dp[k];
      for (int k = k_nudge - 2; k >= 0; --k) dm[k] = dm[k + 1];
    }
    std::vector<real> c_r(c.begin(), c.end());
    FV3B_CHECK(cudaMemcpy(colp(ctx, COL_RF), c_r.data(), sizeof(real) * c_r.size(), cudaMemcpyHostToDevice));
    std::vector<real> dp_r(dp, dp + nz);
    FV3B_CHECK(cudaMemcpy(colp(ctx, COL_DP_RAY), dp_r.data(), sizeof(real) * nz, cudaMemcpyHostToDevice));
    rs.ready = true;
    rs.dt = dt;
    rs.ptop = ptop;
    rs.rf_cutoff = rf_cutoff;
    rs.tau = tau;
    for (int k = 0; k < nz; ++k) {
      rs.dp[k] = dp[k];
      rs.pfull[k] = pfull[k];
    }
    rs.k_rf = k_rf;
    rs.k_nudge = k_nudge;
  }
  const int k_rf = rs.k_rf, k_nudge = rs.k_nudge;
  if (k_rf == 0) return FV3B_OK;
  const real* rf = colp(ctx, COL_RF);
  const real* dm = colp(ctx, COL_RF_DM);
  const real* dpc = colp(ctx, COL_DP_RAY);
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  const bool do_w = hydrostatic == 0;
  FV3B_CHECK(launch_columns(s, e + 2, js, je + 2, st, [=] __device__(int t, int i, int j) {
    const idx_t o0 = idx3(d, t, i, j, 0);
    auto damp = [&](real* q) {
      double total = 0.0;  // column sum in double in every build
      for (int k = 0; k < k_rf; ++k) {
        idx_t o = o0 + k * d.sk;
        real c = q[o];
        real lost = (RC(1.0) - rf[k]) * dpc[k] * c;
        total = k == 0 ? lost : total + lost;
        q[o] = c * rf[k];
      }
      for (int k = 0; k < k_nudge; ++k) {
        idx_t o = o0 + k * d.sk;
        q[o] = q[o] + static_cast<real>(total / dm[k]);
      }
    };
    if (i <= e) damp(u);
    if (j <= je) damp(v);
    if (do_w && i <= e && j <= je)
      for (int k = 0; k < k_rf; ++k) w[o0 + k * d.sk] = w[o0 + k * d.sk] * rf[k];
  }));
  return FV3B_OK;
}

// Adjoint of fv3b_ray_fast (no reference counterpart), in place on the
// cotangents gu, gv, gw of the new winds.  The damping constants are those
// the last fv3b_ray_fast call on this context derived; the arguments must
// match that call's.
extern "C" int fv3b_ray_fast_adjoint(fv3b_ctx* ctx, real* gu, real* gv, real* gw, const double* dp,
                                     const double* pfull, double dt, double ptop, double rf_cutoff, double tau,
                                     int hydrostatic, void* stream) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && gu && gv && gw && dp && pfull, "fv3b_ray_fast_adjoint: null argument");
  const Dims d = ctx->d;
  const RayState& rs = ctx->ray;
  bool same = rs.ready && rs.dt == dt && rs.ptop == ptop && rs.rf_cutoff == rf_cutoff && rs.tau == tau;
  for (int k = 0; same && k < d.nz; ++k) same = rs.dp[k] == dp[k] && rs.pfull[k] == pfull[k];
  FV3B_REQUIRE(same, "fv3b_ray_fast_adjoint: call fv3b_ray_fast first with the same constants");
  const int k_rf = rs.k_rf, k_nudge = rs.k_nudge;
  if (k_rf == 0) return FV3B_OK;
  const real* rf = colp(ctx, COL_RF);
  const real* dm = colp(ctx, COL_RF_DM);
  const real* dpc = colp(ctx, COL_DP_RAY);
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  const bool do_w = hydrostatic == 0;
  FV3B_CHECK(launch_columns(s, e + 2, js, je + 2, (cudaStream_t)stream, [=] __device__(int t, int i, int j) {
    const idx_t o0 = idx3(d, t, i, j, 0);
    if (i <= e) adj::ray_column_adjoint<real>(k_rf, k_nudge, d.sk, rf, dm, dpc, gu + o0);
    if (j <= je) adj::ray_column_adjoint<real>(k_rf, k_nudge, d.sk, rf, dm, dpc, gv + o0);
    if (do_w && i <= e && j <= je) adj::ray_w_column_adjoint<real>(k_rf, d.sk, rf, gw + o0);
  }));
  return FV3B_OK;
}

// HyperdiffusionDamping.__call__ (del2cubed.py:152-181): ntimes = min(3,
// nmax) del-2 passes on qdel with coefficient cd; pass n works on the
// compute domain plus nt = ntimes-1-n halo rows.  The reference's corner
// copies of its scratch q (copy_corners_x before the x fluxes, _y before
// the y fluxes and the copy back) are reads through the corner rules.
extern "C" int fv3b_del2cubed(fv3b_ctx* ctx, real* qdel, double cd_in, int nmax, void* stream) {
  FV3B_TILES(ctx);
  // the build's precision inside the kernels (the same value in FP64 builds)
  const real cd = static_cast<real>(cd_in);
  FV3B_REQUIRE(ctx && qdel, "fv3b_del2cubed: null argument");
  const Dims d = ctx->d;
  const fv3b_metrics g = ctx->m;
  cudaStream_t st = (cudaStream_t)stream;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec, nz = d.nz;
  const int full = d.ni - 1;
  real *q = ctx->ws[0], *fx = ctx->ws[1], *fy = ctx->ws[2];
  const int ntimes = nmax < 3 ? nmax : 3;
  for (int n = 0; n < ntimes; ++n) {
    const int nt = ntimes - (n + 1);
    // corner_fill (del2cubed.py:41-75) into q, full domain
    FV3B_CHECK(launch_box(Box{0, full, 0, full, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
      PT_SETUP(d, t, k);
      const real third = RC(1.0) / RC(3.0);
      real out = F3(qdel, i, j);
      auto Q = [&](int di, int dj) { return F3(qdel, i + di, j + dj); };
      if (j == js) {
        if (i == s) out = (Q(0, 0) + Q(-1, 0) + Q(0, -1)) * third;
        else if (i == s - 1) out = (Q(1, 0) + Q(0, 0) + Q(1, -1)) * third;
        else if (i == e) out = (Q(0, 0) + Q(1, 0) + Q(0, -1)) * third;
        else if (i == e + 1) out = (Q(-1, 0) + Q(0, 0) + Q(-1, -1)) * third;
      } else if (j == js - 1) {
        if (i == s) out = (Q(0, 1) + Q(-1, 1) + Q(0, 0)) * third;
        else if (i == e) out = (Q(0, 1) + Q(1, 1) + Q(0, 0)) * third;
      } else if (j == je) {
        if (i == e) out = (Q(0, 0) + Q(1, 0) + Q(0, 1)) * third;
        else if (i == e + 1) out = (Q(-1, 0) + Q(0, 0) + Q(-1, 1)) * third;
        else if (i == s) out = (Q(0, 0) + Q(-1, 0) + Q(0, 1)) * third;
        else if (i == s - 1) out = (Q(1, 0) + Q(0, 0) + Q(1, 1)) * third;
      } else if (j == je + 1) {
        if (i == e) out = (Q(0, -1) + Q(1, -1) + Q(0, 0)) * third;
        else if (i == s) out = (Q(0, -1) + Q(-1, -1) + Q(0, 0)) * third;
      }
      W3(q, i, j) = out;
    }));
    // compute_zonal_flux / compute_meridional_flux on the X / Y interfaces
    FV3B_CHECK(launch_box(Box{s - nt, e + 2 + nt, js - nt, je + 2 + nt, 0, nz}, st,
                          [=] __device__(int t, int i, int j, int k) {
                            PT_SETUP(d, t, k);
                            auto qx = [&](int ii, int jj) {
                              int si, sj;
                              if (nt > 0 && copy_corner_x(d, ii, jj, si, sj)) return F3(q, si, sj);
                              return F3(q, ii, jj);
                            };
                            auto qy = [&](int ii, int jj) {
                              int si, sj;
                              if (nt > 0 && copy_corner_y(d, ii, jj, si, sj)) return F3(q, si, sj);
                              return F3(q, ii, jj);
                            };
                            if (j < je + 1 + nt) W3(fx, i, j) = F2(g.del6_v, i, j) * (qx(i - 1, j) - qx(i, j));
                            if (i < e + 1 + nt) W3(fy, i, j) = F2(g.del6_u, i, j) * (qy(i, j - 1) - qy(i, j));
                          }));
    // copy back (q after both corner copies) and update_q
    FV3B_CHECK(launch_box(Box{0, full, 0, full, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
      PT_SETUP(d, t, k);
      int si, sj;
      real qv = (nt > 0 && copy_corner_y(d, i, j, si, sj)) ? F3(q, si, sj) : F3(q, i, j);
      if (i >= s - nt && i < e + 1 + nt && j >= js - nt && j < je + 1 + nt)
        qv = qv + cd * F2(g.rarea, i, j) * (F3(fx, i, j) - F3(fx, i + 1, j) + F3(fy, i, j) - F3(fy, i, j + 1));
      W3(qdel, i, j) = qv;
    }));
  }
  return FV3B_OK;
}

// Adjoint of fv3b_del2cubed (no reference counterpart), in place on the
// cotangent g of the filtered field: the passes transposed in reverse order
// (del2cubed_adjoint.h), each scattering every point's cotangent onto the
// inputs it read (atomic adds) in the workspace, then copied back.
extern "C" int fv3b_del2cubed_adjoint(fv3b_ctx* ctx, real* gq, double cd_in, int nmax, void* stream) {
  FV3B_TILES(ctx);
  const real cd = static_cast<real>(cd_in);
  FV3B_REQUIRE(ctx && gq, "fv3b_del2cubed_adjoint: null argument");
  const Dims d = ctx->d;
  const real *del6_u = ctx->m.del6_u, *del6_v = ctx->m.del6_v, *rarea = ctx->m.rarea;
  cudaStream_t st = (cudaStream_t)stream;
  const int full = d.ni - 1, nz = d.nz;
  real* nxt = ctx->ws[0];
  const int ntimes = nmax < 3 ? nmax : 3;
  for (int n = ntimes - 1; n >= 0; --n) {
    const int nt = ntimes - (n + 1);
    FV3B_CHECK(cudaMemsetAsync(nxt, 0, sizeof(real) * (size_t)d.nt * d.st, st));
    FV3B_CHECK(launch_box(Box{0, d.ni, 0, d.nj, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
      const idx_t o = idx3(d, t, i, j, k);
      if (i == full || j == full) {
        atomicAdd(nxt + o, gq[o]);
        return;
      }
      auto add = [&](idx_t oo, real v) { atomicAdd(nxt + oo, v); };
      adj::d2c_pass_adjoint<real>(d, t, i, j, k, nt, cd, del6_u, del6_v, rarea, gq[o], add);
    }));
    FV3B_CHECK(launch_box(Box{0, d.ni, 0, d.nj, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
      const idx_t o = idx3(d, t, i, j, k);
      gq[o] = nxt[o];
    }));
  }
  return FV3B_OK;
}

// compute_pkz_tempadjust (temperature_adjust.py:8-44) on the compute domain,
// levels [0, nk_heat).
extern "C" int fv3b_pkz_tempadjust(fv3b_ctx* ctx, const real* delp, const real* delz, const real* cappa,
                                   const real* heat_source, real* pt, real* pkz, double delt_time_factor_in,
                                   int nk_heat, void* stream) {
  FV3B_TILES(ctx);
  // the build's precision inside the kernels (the same value in FP64 builds)
  const real delt_time_factor = static_cast<real>(delt_time_factor_in);
  FV3B_REQUIRE(ctx && delp && delz && cappa && heat_source && pt && pkz, "fv3b_pkz_tempadjust: null argument");
  const Dims d = ctx->d;
  FV3B_REQUIRE(nk_heat >= 0 && nk_heat <= d.nz, "fv3b_pkz_tempadjust: nk_heat out of range");
  cudaStream_t st = (cudaStream_t)stream;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  FV3B_CHECK(launch_box(Box{s, e + 1, js, je + 1, 0, nk_heat}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    real cp = F3(cappa, i, j), dp = F3(delp, i, j);
    real p = fm::fm_pow(RDG * dp / F3(delz, i, j) * F3(pt, i, j), cp / (RC(1.0) - cp));
    real dtmp = F3(heat_source, i, j) / (CV_AIR * dp);
    real lim = k == 0 ? delt_time_factor * RC(0.1) : (k == 1 ? delt_time_factor * RC(0.5) : delt_time_factor);
    real a = fabs(dtmp);
    real m = lim < a ? lim : a;
    real deltmin = dtmp > RC(0.0) ? fabs(m) : -fabs(m);
    W3(pkz, i, j) = p;
    W3(pt, i, j) = F3(pt, i, j) + deltmin / p;
  }));
  return FV3B_OK;
}

// Adjoint of fv3b_pkz_tempadjust (no reference counterpart).  delp, delz,
// cappa, heat_source and pt are the forward call's inputs; g_pt and g_pkz
// hold the cotangents of the new pt and pkz on entry and those of the old
// ones on return (pkz's zero where the stage overwrote it); g_delp, g_delz
// and g_heat are overwritten on every point.  cappa is held fixed.
extern "C" int fv3b_pkz_tempadjust_adjoint(fv3b_ctx* ctx, const real* delp, const real* delz, const real* cappa,
                                           const real* heat_source, const real* pt, real* g_pt, real* g_pkz,
                                           real* g_delp, real* g_delz, real* g_heat, double delt_time_factor_in,
                                           int nk_heat, void* stream) {
  FV3B_TILES(ctx);
  const real delt_time_factor = static_cast<real>(delt_time_factor_in);
  FV3B_REQUIRE(ctx && delp && delz && cappa && heat_source && pt && g_pt && g_pkz && g_delp && g_delz && g_heat,
               "fv3b_pkz_tempadjust_adjoint: null argument");
  const Dims d = ctx->d;
  FV3B_REQUIRE(nk_heat >= 0 && nk_heat <= d.nz, "fv3b_pkz_tempadjust_adjoint: nk_heat out of range");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t bytes = sizeof(real) * (size_t)d.nt * d.st;
  FV3B_CHECK(cudaMemsetAsync(g_delp, 0, bytes, st));
  FV3B_CHECK(cudaMemsetAsync(g_delz, 0, bytes, st));
  FV3B_CHECK(cudaMemsetAsync(g_heat, 0, bytes, st));
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  FV3B_CHECK(launch_box(Box{s, e + 1, js, je + 1, 0, nk_heat}, st, [=] __device__(int t, int i, int j, int k) {
    const idx_t o = idx3(d, t, i, j, k);
    const real lim = k == 0 ? delt_time_factor * RC(0.1) : (k == 1 ? delt_time_factor * RC(0.5) : delt_time_factor);
    real a_dp, a_dz, a_pt, a_heat;
    adj::tempadjust_point_adjoint<real>(delp[o], delz[o], pt[o], heat_source[o], cappa[o], lim, RDG, CV_AIR, g_pt[o],
                                        g_pkz[o], a_dp, a_dz, a_pt, a_heat);
    g_pt[o] = a_pt;
    g_pkz[o] = RC(0.0);
    g_delp[o] = a_dp;
    g_delz[o] = a_dz;
    g_heat[o] = a_heat;
  }));
  return FV3B_OK;
}

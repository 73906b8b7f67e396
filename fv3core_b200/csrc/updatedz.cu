// Height updates of the acoustic substep:
//   UpdateGeopotentialHeightOnCGrid (fv3core/stencils/updatedzc.py) — the
//     interface heights advected by the C-grid fluxes over half a step;
//   UpdateHeightOnDGrid (fv3core/stencils/updatedzd.py) — the interface
//     heights advected by the D-grid fluxes (spline-interpolated to
//     interfaces) with PPM transport and del-n damping.
// Both end in a per-column bottom-up pass (surface w and the DZ_MIN floor),
// fused here with the last horizontal update.
#include <math.h>

#include <vector>

#include "corners.cuh"
#include "ctx.cuh"
#include "stencil.cuh"
#include "transport.cuh"

using namespace fv3b;

namespace {
constexpr real DZ_MIN = RC(2.0);

// p_weighted_average_top / _domain / _bottom (updatedzc.py:15-34): C-grid
// flux at interface k from the layer fluxes above and below it.
__device__ __forceinline__ real p_weighted(const real* dp0, int k, int nk, real a_km2, real a_km1,
                                             real a_k, real a_kp1) {
  if (k == 0) {
    real ratio = dp0[0] / (dp0[0] + dp0[1]);
    return a_k + (a_k - a_kp1) * ratio;
  }
  if (k == nk - 1) {
    real ratio = dp0[k - 1] / (dp0[k - 2] + dp0[k - 1]);
    return a_km1 + (a_km1 - a_km2) * ratio;
  }
  real ir = RC(1.0) / (dp0[k - 1] + dp0[k]);
  return (dp0[k] * a_km1 + dp0[k - 1] * a_k) * ir;
}
}  // namespace

// UpdateGeopotentialHeightOnCGrid.__call__ (updatedzc.py:123-163).
extern "C" int fv3b_update_dz_c(fv3b_ctx* ctx, const real* dp_ref, const real* zs, const real* ut,
                                const real* vt, real* gz, real* ws, double dt_in, void* stream) {
  FV3B_TILES(ctx);
  // the build's precision inside the kernels (the same value in FP64 builds)
  const real dt = static_cast<real>(dt_in);
  FV3B_REQUIRE(ctx && dp_ref && zs && ut && vt && gz && ws, "fv3b_update_dz_c: null argument");
  const Dims d = ctx->d;
  const fv3b_metrics g = ctx->m;
  FV3B_REQUIRE(d.nk >= 3, "fv3b_update_dz_c: npz must be at least 2");
  cudaStream_t st = (cudaStream_t)stream;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec, nk = d.nk;
  real* gz_new = ctx->ws[0];
  // advected heights on [is-1, ie+1] x [js-1, je+1], every interface; the
  // reference's corner-filled copies gz_x / gz_y are reads through the
  // two-cell corner rules
  FV3B_CHECK(launch_box(Box{s - 1, e + 2, js - 1, je + 2, 0, nk}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    auto gzx = [&](int ii, int jj) {
      CornerRule r;
      if (corner_x(d, ii, jj, false, RC(1.0), RC(1.0), RC(1.0), RC(1.0), r)) return F3(gz, ii + r.di, jj + r.dj);
      return F3(gz, ii, jj);
    };
    auto gzy = [&](int ii, int jj) {
      CornerRule r;
      if (corner_y(d, ii, jj, false, RC(1.0), RC(1.0), RC(1.0), RC(1.0), r)) return F3(gz, ii + r.di, jj + r.dj);
      return F3(gz, ii, jj);
    };
    auto lev = [&](const real* a, int ii, int jj, int dk) {
      int kk = k + dk;
      return (kk >= 0 && kk < nk) ? F3K(a, ii, jj, dk) : RC(0.0);
    };
    auto xfx = [&](int ii) {
      return p_weighted(dp_ref, k, nk, lev(ut, ii, j, -2), lev(ut, ii, j, -1), lev(ut, ii, j, 0),
                        lev(ut, ii, j, 1));
    };
    auto yfx = [&](int jj) {
      return p_weighted(dp_ref, k, nk, lev(vt, i, jj, -2), lev(vt, i, jj, -1), lev(vt, i, jj, 0),
                        lev(vt, i, jj, 1));
    };
    real xf0 = xfx(i), xf1 = xfx(i + 1), yf0 = yfx(j), yf1 = yfx(j + 1);
    real fx0 = xf0 * (xf0 > RC(0.0) ? gzx(i - 1, j) : gzx(i, j));
    real fx1 = xf1 * (xf1 > RC(0.0) ? gzx(i, j) : gzx(i + 1, j));
    real fy0 = yf0 * (yf0 > RC(0.0) ? gzy(i, j - 1) : gzy(i, j));
    real fy1 = yf1 * (yf1 > RC(0.0) ? gzy(i, j) : gzy(i, j + 1));
    real area = F2(g.area, i, j);
    W3(gz_new, i, j) = (gzy(i, j) * area + fx0 - fx1 + fy0 - fy1) / (area + xf0 - xf1 + yf0 - yf1);
  }));
  // surface w and the DZ_MIN floor, bottom up (updatedzc.py:100-120)
  const real rdt = RC(1.0) / dt;
  FV3B_CHECK(launch_columns(s - 1, e + 2, js - 1, je + 2, st, [=] __device__(int t, int i, int j) {
    idx_t o = idx3(d, t, i, j, nk - 1);
    real below = gz_new[o];
    gz[o] = below;
    ws[idx2(d, t, i, j)] = (zs[idx2(d, t, i, j)] - below) * rdt;
    for (int k = nk - 2; k >= 0; --k) {
      o -= d.sk;
      real v = gz_new[o];
      real kp1 = below + DZ_MIN;
      below = v > kp1 ? v : kp1;
      gz[o] = below;
    }
  }));
  return FV3B_OK;
}

// UpdateHeightOnDGrid.__init__ (updatedzd.py:189-320): the cubic-spline
// constants of cubic_spline_interpolation_constants (121-145) from dp0.
extern "C" int fv3b_update_dz_d_setup(fv3b_ctx* ctx, const double* dp_ref_host, int hord_tm) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && dp_ref_host, "fv3b_update_dz_d_setup: null argument");
  FV3B_REQUIRE(ctx->dsw.ready, "fv3b_update_dz_d_setup: call fv3b_d_sw_setup first (column namelist)");
  const int nk = ctx->d.nk;
  FV3B_REQUIRE(nk > 4 && nk <= MAXLEV, "fv3b_update_dz_d_setup: npz must be in 4..127");
  std::vector<double> c((size_t)4 * MAXLEV, 0.0);
  double *dp = c.data(), *gk = dp + MAXLEV, *beta = gk + MAXLEV, *gamma = beta + MAXLEV;
  for (int k = 0; k < nk; ++k) dp[k] = dp_ref_host[k];
  gk[0] = dp[1] / dp[0];
  beta[0] = gk[0] * (gk[0] + 0.5);
  gamma[0] = (1.0 + gk[0] * (gk[0] + 1.5)) / beta[0];
  for (int k = 1; k < nk - 1; ++k) {
    gk[k] = dp[k - 1] / dp[k];
    beta[k] = 2.0 + 2.0 * gk[k] - gamma[k - 1];
    gamma[k] = gk[k] / beta[k];
  }
  const std::vector<real> c_r(c.begin(), c.end());
  FV3B_CHECK(cudaMemcpy(colp(ctx, COL_DP_REF), c_r.data(), sizeof(real) * c_r.size(), cudaMemcpyHostToDevice));
  ctx->dzd_hord_tm = hord_tm;
  ctx->dzd_ready = true;
  return FV3B_OK;
}

// UpdateHeightOnDGrid.__call__ (updatedzd.py:323-393).
extern "C" int fv3b_update_dz_d(fv3b_ctx* ctx, const real* zs, real* zh, const real* crx, const real* cry,
                                const real* xfx, const real* yfx, real* wsd, double dt_in, void* stream) {
  FV3B_TILES(ctx);
  // the build's precision inside the kernels (the same value in FP64 builds)
  const real dt = static_cast<real>(dt_in);
  FV3B_REQUIRE(ctx && zs && zh && crx && cry && xfx && yfx && wsd, "fv3b_update_dz_d: null argument");
  FV3B_REQUIRE(ctx->dzd_ready, "fv3b_update_dz_d: call fv3b_update_dz_d_setup first");
  const Dims d = ctx->d;
  const fv3b_metrics g = ctx->m;
  cudaStream_t st = (cudaStream_t)stream;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec, nk = d.nk;
  const int full = d.ni - 1;
  real** W = ctx->ws;
  real *crx_i = W[0], *cry_i = W[1], *xfx_i = W[2], *yfx_i = W[3], *fx = W[4], *fy = W[5];
  real *fx_mean = W[7], *fy_mean = W[8], *q_adv_x = W[9], *q_adv_y = W[10];
  real *gzx_diff = W[11], *gzy_diff = W[12], *d2 = W[13];
  const real* gk = colp(ctx, COL_SPLINE_GK);
  const real* beta = colp(ctx, COL_SPLINE_BETA);
  const real* gamma = colp(ctx, COL_SPLINE_GAMMA);
  // cubic_spline_interpolation_from_layer_center_to_interfaces
  // (updatedzd.py:148-186) of the four flux fields over the full domain;
  // one thread per (field, column): the launch's i index runs over the four
  // fields' column rows in turn, f = i / full
  FV3B_CHECK(launch_columns(0, 4 * full, 0, full, st, [=] __device__(int t, int fi, int j) {
    const int f = fi / full, i = fi % full;
    const real* q = (f == 0 ? crx : f == 1 ? xfx : f == 2 ? cry : yfx) + idx3(d, t, i, j, 0);
    real* out = (f == 0 ? crx_i : f == 1 ? xfx_i : f == 2 ? cry_i : yfx_i) + idx3(d, t, i, j, 0);
    const idx_t sk = d.sk;
    {
      real xt1 = RC(2.0) * gk[0] * (gk[0] + RC(1.0));
      real prev = (xt1 * q[0] + q[sk]) / beta[0];
      out[0] = prev;
      for (int k = 1; k < nk - 1; ++k) {
        prev = (RC(3.0) * (q[(k - 1) * sk] + gk[k] * q[k * sk]) - prev) / beta[k];
        out[k * sk] = prev;
      }
      const int k = nk - 1;
      const real a_bot = RC(1.0) + gk[k - 1] * (gk[k - 1] + RC(1.5));
      const real xb1 = RC(2.0) * gk[k - 1] * (gk[k - 1] + RC(1.0));
      const real xb2 = gk[k - 1] * (gk[k - 1] + RC(0.5)) - a_bot * gamma[k - 1];
      real next = (xb1 * q[(k - 1) * sk] + q[(k - 2) * sk] - a_bot * prev) / xb2;
      out[k * sk] = next;
      for (int kk = nk - 2; kk >= 0; --kk) {
        next = out[kk * sk] - gamma[kk] * next;
        out[kk * sk] = next;
      }
    }
  }));
  FV3B_CHECK(copy_corners_x_inplace(d, zh, st));
  FvTp2dArgs a{zh, crx_i, cry_i, xfx_i, yfx_i, xfx_i, yfx_i, fx, fy, ctx->dzd_hord_tm,
               fx_mean, fy_mean, q_adv_x, q_adv_y};
  FV3B_CHECK(fvtp2d(d, g, a, st));
  // DelnFluxNoSG on npz + 1 levels with the raw damp_vt column (range-scaled
  // copy, identical to damp_vt in double builds)
  DelnCol dl{colp(ctx, COL_NORD_V), colp(ctx, COL_DAMP_VT_DZ), static_cast<real>(ctx->dsw.area_scale)};
  FV3B_CHECK(delnflux_nosg(d, g, zh, gzx_diff, gzy_diff, dl, d2, W[WS_DELN_ALT], false, ctx->dsw.nmax_v, st, nk));
  // apply_height_fluxes (updatedzd.py:63-118) fused with the surface w and
  // DZ_MIN floor, bottom up per column of the compute domain
  FV3B_CHECK(launch_columns(s, e + 1, js, je + 1, st, [=] __device__(int t, int i, int j) {
    const real area = g.area[idx2(d, t, i, j)];
    auto new_height = [&](int k) {
      PT_SETUP(d, t, k);
      real aaf = (area + F3(xfx_i, i, j) - F3(xfx_i, i + 1, j)) + (area + F3(yfx_i, i, j) - F3(yfx_i, i, j + 1)) -
                   area;
      real adv = (F3(zh, i, j) * area + F3(fx, i, j) - F3(fx, i + 1, j) + F3(fy, i, j) - F3(fy, i, j + 1)) / aaf;
      real diff =
          (F3(gzx_diff, i, j) - F3(gzx_diff, i + 1, j) + F3(gzy_diff, i, j) - F3(gzy_diff, i, j + 1)) / area;
      return adv + diff;
    };
    idx_t o = idx3(d, t, i, j, nk - 1);
    real below = new_height(nk - 1);
    zh[o] = below;
    wsd[idx2(d, t, i, j)] = (zs[idx2(d, t, i, j)] - below) / dt;
    for (int k = nk - 2; k >= 0; --k) {
      o -= d.sk;
      real v = new_height(k);
      real other = below + DZ_MIN;
      below = v > other ? v : other;
      zh[o] = below;
    }
  }));
  return FV3B_OK;
}

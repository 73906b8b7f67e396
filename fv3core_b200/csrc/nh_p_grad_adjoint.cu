// fv3b_nh_p_grad_adjoint: the adjoint of NonHydrostaticPressureGradient
// (nh_p_grad.py:147-206) from nh_p_grad_adjoint.h and a2b_adjoint.h.  The
// B-grid fields are recomputed with the forward's a2b_ord4, the wind
// update's cotangents are scattered onto them, and each interpolation is
// transposed back onto its A-grid input (three passes, atomic adds: the
// passes' points share inputs).
#include <math.h>

#include "a2b.cuh"
#include "a2b_adjoint.h"
#include "ctx.cuh"
#include "nh_p_grad_adjoint.h"
#include "stencil.cuh"

using namespace fv3b;

namespace {

// gin += (a2b_ord4 on levels [k0, k1))^T gout; gqx, gqy, gedges: scratch
cudaError_t a2b_transpose(const Dims d, const adj::A2BGrid<real> g, const real* gout, real* gin, real* gqx,
                          real* gqy, real* gedges, int k0, int k1, cudaStream_t st) {
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec, n = d.n;
  const size_t bytes = sizeof(real) * (size_t)d.nt * d.st;
  cudaError_t err;
  if ((err = cudaMemsetAsync(gqx, 0, bytes, st)) != cudaSuccess) return err;
  if ((err = cudaMemsetAsync(gqy, 0, bytes, st)) != cudaSuccess) return err;
  if ((err = cudaMemsetAsync(gedges, 0, bytes, st)) != cudaSuccess) return err;
  err = launch_box(Box{s + 1, e + 1, js + 1, je + 1, k0, k1}, st, [=] __device__(int t, int i, int j, int k) {
    real* const out[3] = {gqx, gqy, gedges};
    auto add = [&](int a, idx_t o, real v) { atomicAdd(out[a] + o, v); };
    adj::a2b_interior_adjoint<real>(d, t, i, j, k, gout[idx3(d, t, i, j, k)], add);
  });
  if (err != cudaSuccess) return err;
  err = launch_box(Box{s - 2, e + 3, js - 2, je + 3, k0, k1}, st, [=] __device__(int t, int i, int j, int k) {
    const idx_t o = idx3(d, t, i, j, k);
    auto add = [&](int, idx_t oo, real v) { atomicAdd(gin + oo, v); };
    adj::a2b_volume_mean_adjoint<real>(d, g, t, i, j, k, gqx[o], gqy[o], add);
  });
  if (err != cudaSuccess) return err;
  // the boundary of [is, ie+1] x [js, je+1]: south and north rows (corners
  // included), then the west and east columns
  return launch_box(Box{0, 4 * (n + 1), 0, 1, k0, k1}, st, [=] __device__(int t, int p, int, int k) {
    const int side = p / (n + 1), a = p % (n + 1);
    if (side >= 2 && (a == 0 || a == n)) return;
    const int i = side < 2 ? s + a : (side == 2 ? s : e + 1);
    const int j = side == 0 ? js : (side == 1 ? je + 1 : js + a);
    const idx_t o = idx3(d, t, i, j, k);
    auto add = [&](int, idx_t oo, real v) { atomicAdd(gin + oo, v); };
    adj::a2b_boundary_adjoint<real>(d, g, t, i, j, k, gout[o] + gedges[o], add);
  });
}

}  // namespace

extern "C" int fv3b_nh_p_grad_adjoint(fv3b_ctx* ctx, const real* pp, const real* gz, const real* pk3,
                                      const real* delp, const real* gu, const real* gv, const real* gpp,
                                      const real* ggz, const real* gpk3, real* g_u, real* g_v, real* g_pp,
                                      real* g_gz, real* g_pk3, real* g_delp, double dt_in, double ptop, double akap,
                                      void* stream) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && pp && gz && pk3 && delp && gu && gv && gpp && ggz && gpk3 && g_u && g_v && g_pp && g_gz &&
                   g_pk3 && g_delp,
               "fv3b_nh_p_grad_adjoint: null argument");
  const Dims d = ctx->d;
  const fv3b_metrics m = ctx->m;
  const adj::A2BGrid<real> ag{m.dxa, m.dya, m.edge_w, m.edge_e, m.edge_s, m.edge_n, m.a2b_extrap};
  const real dt = static_cast<real>(dt_in);
  const real ptk = static_cast<real>(pow(ptop, akap));
  cudaStream_t st = (cudaStream_t)stream;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec, nz = d.nz, nk = d.nk;
  real *wk1 = ctx->ws[0], *qx = ctx->ws[1], *qy = ctx->ws[2], *edges = ctx->ws[3];
  real *pp_b = ctx->ws[4], *pk3_b = ctx->ws[5], *gz_b = ctx->ws[6];
  real *gb_pp = ctx->ws[7], *gb_pk3 = ctx->ws[8], *gb_gz = ctx->ws[9], *gb_wk1 = ctx->ws[10];
  // the forward's B-grid fields (a2b_ord4 leaves its input unchanged here)
  FV3B_CHECK(a2b_ord4(d, m, const_cast<real*>(pp), pp_b, qx, qy, edges, 1, nk, st, false));
  FV3B_CHECK(a2b_ord4(d, m, const_cast<real*>(pk3), pk3_b, qx, qy, edges, 1, nk, st, false));
  FV3B_CHECK(a2b_ord4(d, m, const_cast<real*>(gz), gz_b, qx, qy, edges, 0, nk, st, false));
  FV3B_CHECK(a2b_ord4(d, m, const_cast<real*>(delp), wk1, qx, qy, edges, 0, nz, st, false));
  // pass-through outside what the stage writes; the B-grid outputs'
  // cotangents onto the B-grid fields (levels of pp and pk3 above 0)
  FV3B_CHECK(launch_box(Box{0, d.ni, 0, d.nj, 0, nk}, st, [=] __device__(int t, int i, int j, int k) {
    const idx_t o = idx3(d, t, i, j, k);
    const bool box = i >= s && i <= e + 1 && j >= js && j <= je + 1;
    g_u[o] = (k < nz && i >= s && i <= e && j >= js && j <= je + 1) ? RC(0.0) : gu[o];
    g_v[o] = (k < nz && i >= s && i <= e + 1 && j >= js && j <= je) ? RC(0.0) : gv[o];
    g_pp[o] = box ? RC(0.0) : gpp[o];
    g_pk3[o] = box ? RC(0.0) : gpk3[o];
    g_gz[o] = box ? RC(0.0) : ggz[o];
    g_delp[o] = RC(0.0);
    gb_pp[o] = box && k > 0 ? gpp[o] : RC(0.0);
    gb_pk3[o] = box && k > 0 ? gpk3[o] : RC(0.0);
    gb_gz[o] = box ? ggz[o] : RC(0.0);
    gb_wk1[o] = RC(0.0);
  }));
  const real *rdx = m.rdx, *rdy = m.rdy;
  FV3B_CHECK(launch_box(Box{s, e + 2, js, je + 2, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
    real* out[5] = {gb_pp, gb_pk3, gb_gz, gb_wk1, nullptr};
    for (int dir = 0; dir < 2; ++dir) {
      if ((dir == 0 && i > e) || (dir == 1 && j > je)) continue;
      out[4] = dir == 0 ? g_u : g_v;
      auto add = [&](int a, idx_t o, real v) { atomicAdd(out[a] + o, v); };
      adj::nhp_wind_adjoint<real>(d, t, i, j, k, dir, (dir == 0 ? gu : gv)[idx3(d, t, i, j, k)], dt, ptk,
                                  dir == 0 ? rdx : rdy, pp_b, pk3_b, gz_b, wk1, add);
    }
  }));
  real *gqx = ctx->ws[11], *gqy = ctx->ws[12], *gedges = ctx->ws[13];
  FV3B_CHECK(a2b_transpose(d, ag, gb_pp, g_pp, gqx, gqy, gedges, 1, nk, st));
  FV3B_CHECK(a2b_transpose(d, ag, gb_pk3, g_pk3, gqx, gqy, gedges, 1, nk, st));
  FV3B_CHECK(a2b_transpose(d, ag, gb_gz, g_gz, gqx, gqy, gedges, 0, nk, st));
  FV3B_CHECK(a2b_transpose(d, ag, gb_wk1, g_delp, gqx, gqy, gedges, 0, nz, st));
  return FV3B_OK;
}

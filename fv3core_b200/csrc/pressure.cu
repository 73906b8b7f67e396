// Pressure-gradient stages of the acoustic substep:
//   p_grad_c_stencil (fv3core/stencils/dyn_core.py:101-145), nonhydrostatic;
//   NonHydrostaticPressureGradient (fv3core/stencils/nh_p_grad.py);
//   edge_pe (fv3core/stencils/pe_halo.py) and PK3Halo
//   (fv3core/stencils/pk3_halo.py), the hydrostatic pressure on the rings
//   of halo cells around the compute domain.
#include <math.h>

#include "a2b.cuh"
#include "ctx.cuh"
#include "fmath.h"
#include "stencil.cuh"

using namespace fv3b;

// p_grad_c_stencil, nonhydrostatic (wk = delpc), on [is, ie+1] x [js, je+1].
extern "C" int fv3b_p_grad_c(fv3b_ctx* ctx, real* uc, real* vc, const real* delpc, const real* pkc,
                             const real* gz, double dt2_in, void* stream) {
  FV3B_TILES(ctx);
  // the build's precision inside the kernels (the same value in FP64 builds)
  const real dt2 = static_cast<real>(dt2_in);
  FV3B_REQUIRE(ctx && uc && vc && delpc && pkc && gz, "fv3b_p_grad_c: null argument");
  const Dims d = ctx->d;
  const fv3b_metrics g = ctx->m;
  cudaStream_t st = (cudaStream_t)stream;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  FV3B_CHECK(launch_box(Box{s, e + 2, js, je + 2, 0, d.nz}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    real wk = F3(delpc, i, j);
    W3(uc, i, j) = F3(uc, i, j) + dt2 * F2(g.rdxc, i, j) / (F3(delpc, i - 1, j) + wk) *
                                      ((F3K(gz, i - 1, j, 1) - F3(gz, i, j)) * (F3K(pkc, i, j, 1) - F3(pkc, i - 1, j)) +
                                       (F3(gz, i - 1, j) - F3K(gz, i, j, 1)) * (F3K(pkc, i - 1, j, 1) - F3(pkc, i, j)));
    W3(vc, i, j) = F3(vc, i, j) + dt2 * F2(g.rdyc, i, j) / (F3(delpc, i, j - 1) + wk) *
                                      ((F3K(gz, i, j - 1, 1) - F3(gz, i, j)) * (F3K(pkc, i, j, 1) - F3(pkc, i, j - 1)) +
                                       (F3(gz, i, j - 1) - F3K(gz, i, j, 1)) * (F3K(pkc, i, j - 1, 1) - F3(pkc, i, j)));
  }));
  return FV3B_OK;
}

// NonHydrostaticPressureGradient.__call__ (nh_p_grad.py:147-206).  pp, pk3
// and gz are replaced by their B-grid interpolations (levels 1.., 1.., 0..);
// the B-grid delp goes to scratch.  set_k0_and_calc_wk is folded into the
// wind update: level 0 of pp and pk3 is read as its new value (0, ptop^akap).
extern "C" int fv3b_nh_p_grad(fv3b_ctx* ctx, real* u, real* v, real* pp, real* gz, real* pk3,
                              real* delp, double dt_in, double ptop, double akap, void* stream) {
  FV3B_TILES(ctx);
  // the build's precision inside the kernels (the same value in FP64 builds)
  const real dt = static_cast<real>(dt_in);
  FV3B_REQUIRE(ctx && u && v && pp && gz && pk3 && delp, "fv3b_nh_p_grad: null argument");
  const Dims d = ctx->d;
  const fv3b_metrics g = ctx->m;
  cudaStream_t st = (cudaStream_t)stream;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec, nz = d.nz, nk = d.nk;
  // The B-grid values of pp, pk3 and gz go to scratch (the reference
  // interpolates them in place); the wind update reads only the scratch
  // copies and writes them back into pp, pk3, gz, which replaces the
  // reference's copy passes.
  real *wk1 = ctx->ws[0], *qx = ctx->ws[1], *qy = ctx->ws[2], *edges = ctx->ws[3];
  real *pp_b = ctx->ws[4], *pk3_b = ctx->ws[5], *gz_b = ctx->ws[6];
  const real ptk = static_cast<real>(pow(ptop, akap));
  FV3B_CHECK(a2b_ord4(d, g, pp, pp_b, qx, qy, edges, 1, nk, st, false));
  FV3B_CHECK(a2b_ord4(d, g, pk3, pk3_b, qx, qy, edges, 1, nk, st, false));
  FV3B_CHECK(a2b_ord4(d, g, gz, gz_b, qx, qy, edges, 0, nk, st, false));
  FV3B_CHECK(a2b_ord4(d, g, delp, wk1, qx, qy, edges, 0, nz, st, false));
  // calc_u on [is, ie] x [js, je+1], calc_v on [is, ie+1] x [js, je] (levels
  // [0, npz)); every interface of [is, ie+1] x [js, je+1] takes its B-grid
  // pp, pk3, gz, with pp = 0 and pk3 = ptop^akap on top (set_k0_and_calc_wk)
  FV3B_CHECK(launch_box(Box{s, e + 2, js, je + 2, 0, nk}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    auto P = [&](int ii, int jj, int dk) { return k + dk == 0 ? RC(0.0) : F3K(pp_b, ii, jj, dk); };
    auto K3 = [&](int ii, int jj, int dk) { return k + dk == 0 ? ptk : F3K(pk3_b, ii, jj, dk); };
    auto wk = [&](int ii, int jj) { return K3(ii, jj, 1) - K3(ii, jj, 0); };
    if (k < nz && i <= e) {
      real du = dt / (wk(i, j) + wk(i + 1, j)) *
                  ((F3K(gz_b, i, j, 1) - F3(gz_b, i + 1, j)) * (K3(i + 1, j, 1) - K3(i, j, 0)) +
                   (F3(gz_b, i, j) - F3K(gz_b, i + 1, j, 1)) * (K3(i, j, 1) - K3(i + 1, j, 0)));
      W3(u, i, j) = (F3(u, i, j) + du +
                     dt / (F3(wk1, i, j) + F3(wk1, i + 1, j)) *
                         ((F3K(gz_b, i, j, 1) - F3(gz_b, i + 1, j)) * (P(i + 1, j, 1) - P(i, j, 0)) +
                          (F3(gz_b, i, j) - F3K(gz_b, i + 1, j, 1)) * (P(i, j, 1) - P(i + 1, j, 0)))) *
                    F2(g.rdx, i, j);
    }
    if (k < nz && j <= je) {
      real dv = dt / (wk(i, j) + wk(i, j + 1)) *
                  ((F3K(gz_b, i, j, 1) - F3(gz_b, i, j + 1)) * (K3(i, j + 1, 1) - K3(i, j, 0)) +
                   (F3(gz_b, i, j) - F3K(gz_b, i, j + 1, 1)) * (K3(i, j, 1) - K3(i, j + 1, 0)));
      W3(v, i, j) = (F3(v, i, j) + dv +
                     dt / (F3(wk1, i, j) + F3(wk1, i, j + 1)) *
                         ((F3K(gz_b, i, j, 1) - F3(gz_b, i, j + 1)) * (P(i, j + 1, 1) - P(i, j, 0)) +
                          (F3(gz_b, i, j) - F3K(gz_b, i, j + 1, 1)) * (P(i, j, 1) - P(i, j + 1, 0)))) *
                    F2(g.rdy, i, j);
    }
    W3(pp, i, j) = P(i, j, 0);
    W3(pk3, i, j) = K3(i, j, 0);
    W3(gz, i, j) = F3(gz_b, i, j);
  }));
  return FV3B_OK;
}

// edge_pe (pe_halo.py:6-33): interface pressure on the one-cell ring around
// the compute domain, summed from ptop.
extern "C" int fv3b_edge_pe(fv3b_ctx* ctx, real* pe, const real* delp, double ptop, void* stream) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && pe && delp, "fv3b_edge_pe: null argument");
  const Dims d = ctx->d;
  cudaStream_t st = (cudaStream_t)stream;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec, nk = d.nk;
  FV3B_CHECK(launch_columns(s - 1, e + 2, js - 1, je + 2, st, [=] __device__(int t, int i, int j) {
    if (i >= s && i <= e && j >= js && j <= je) return;
    idx_t o = idx3(d, t, i, j, 0);
    double p = ptop;  // column sums of delp in double in every build
    pe[o] = static_cast<real>(p);
    for (int k = 1; k < nk; ++k) {
      p = p + delp[o];
      o += d.sk;
      pe[o] = static_cast<real>(p);
    }
  }));
  return FV3B_OK;
}

// PK3Halo.__call__ (pk3_halo.py:36-68): pk3 = pe^akap on the two-cell ring,
// levels 1..npz.
extern "C" int fv3b_pk3_halo(fv3b_ctx* ctx, real* pk3, const real* delp, double ptop, double akap,
                             void* stream) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && pk3 && delp, "fv3b_pk3_halo: null argument");
  const Dims d = ctx->d;
  cudaStream_t st = (cudaStream_t)stream;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec, nk = d.nk;
  FV3B_CHECK(launch_columns(s - 2, e + 3, js - 2, je + 3, st, [=] __device__(int t, int i, int j) {
    if (i >= s && i <= e && j >= js && j <= je) return;
    idx_t o = idx3(d, t, i, j, 0);
    double p = ptop;  // column sums of delp in double in every build
    for (int k = 1; k < nk; ++k) {
      p = p + delp[o];
      o += d.sk;
      pk3[o] = static_cast<real>(fm::fm_pow(p, akap));
    }
  }));
  return FV3B_OK;
}

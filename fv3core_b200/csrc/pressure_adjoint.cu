// fv3b_edge_pe_adjoint and fv3b_pk3_halo_adjoint: the column adjoints of
// pressure_adjoint.h on the halo rings of the forward stages, one thread
// per column.
#include "ctx.cuh"
#include "pressure_adjoint.h"
#include "stencil.cuh"

using namespace fv3b;

extern "C" int fv3b_edge_pe_adjoint(fv3b_ctx* ctx, real* g_pe, real* g_delp, void* stream) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && g_pe && g_delp, "fv3b_edge_pe_adjoint: null argument");
  const Dims d = ctx->d;
  cudaStream_t st = (cudaStream_t)stream;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec, nk = d.nk;
  FV3B_CHECK(cudaMemsetAsync(g_delp, 0, sizeof(real) * (size_t)d.nt * d.st, st));
  FV3B_CHECK(launch_columns(s - 1, e + 2, js - 1, je + 2, st, [=] __device__(int t, int i, int j) {
    if (i >= s && i <= e && j >= js && j <= je) return;
    const idx_t o = idx3(d, t, i, j, 0);
    adj::edge_pe_column_adjoint<real>(nk, d.sk, g_pe + o, g_delp + o);
  }));
  return FV3B_OK;
}

extern "C" int fv3b_pk3_halo_adjoint(fv3b_ctx* ctx, const real* delp, real* g_pk3, real* g_delp, double ptop,
                                     double akap, void* stream) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && delp && g_pk3 && g_delp, "fv3b_pk3_halo_adjoint: null argument");
  const Dims d = ctx->d;
  FV3B_REQUIRE(d.nk <= 128, "fv3b_pk3_halo_adjoint: npz must be at most 127");
  cudaStream_t st = (cudaStream_t)stream;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec, nk = d.nk;
  FV3B_CHECK(cudaMemsetAsync(g_delp, 0, sizeof(real) * (size_t)d.nt * d.st, st));
  FV3B_CHECK(launch_columns(s - 2, e + 3, js - 2, je + 3, st, [=] __device__(int t, int i, int j) {
    if (i >= s && i <= e && j >= js && j <= je) return;
    const idx_t o = idx3(d, t, i, j, 0);
    adj::pk3_column_adjoint<real>(nk, d.sk, ptop, akap, delp + o, g_pk3 + o, g_delp + o);
  }));
  return FV3B_OK;
}

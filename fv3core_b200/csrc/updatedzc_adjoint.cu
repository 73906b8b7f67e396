// fv3b_update_dz_c_adjoint: the adjoint of UpdateGeopotentialHeightOnCGrid
// (updatedzc.py:123-163) from updatedzc_adjoint.h.  Four launches: the
// gradients start from the pass-through of gz outside the updated box, the
// heights before the floor are recomputed into the workspace, each column
// runs the floor backwards, and every updated point adds its contributions
// to gz, ut and vt (atomically: a point's sources are shared with its
// neighbours').
#include "ctx.cuh"
#include "stencil.cuh"
#include "updatedzc_adjoint.h"

using namespace fv3b;

extern "C" int fv3b_update_dz_c_adjoint(fv3b_ctx* ctx, const real* dp_ref, const real* ut, const real* vt,
                                        const real* gz, const real* g_gz_out, const real* g_ws, real* g_gz,
                                        real* g_ut, real* g_vt, double dt_in, void* stream) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && dp_ref && ut && vt && gz && g_gz_out && g_ws && g_gz && g_ut && g_vt,
               "fv3b_update_dz_c_adjoint: null argument");
  const Dims d = ctx->d;
  FV3B_REQUIRE(d.nk >= 3 && d.nk <= 128, "fv3b_update_dz_c_adjoint: npz must be in 2..127");
  const real rdt = RC(1.0) / static_cast<real>(dt_in);
  const real* area = ctx->m.area;
  real* hnew = ctx->ws[0];
  real* g_new = ctx->ws[1];
  cudaStream_t st = (cudaStream_t)stream;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec, nk = d.nk;
  FV3B_CHECK(launch_box(Box{0, d.ni, 0, d.nj, 0, nk}, st, [=] __device__(int t, int i, int j, int k) {
    const idx_t o = idx3(d, t, i, j, k);
    const bool updated = i >= s - 1 && i <= e + 1 && j >= js - 1 && j <= je + 1;
    g_gz[o] = updated ? RC(0.0) : g_gz_out[o];
    g_ut[o] = RC(0.0);
    g_vt[o] = RC(0.0);
  }));
  FV3B_CHECK(launch_box(Box{s - 1, e + 2, js - 1, je + 2, 0, nk}, st, [=] __device__(int t, int i, int j, int k) {
    hnew[idx3(d, t, i, j, k)] = adj::uzc_new<real>(d, t, i, j, k, dp_ref, area, ut, vt, gz);
  }));
  FV3B_CHECK(launch_columns(s - 1, e + 2, js - 1, je + 2, st, [=] __device__(int t, int i, int j) {
    const idx_t o = idx3(d, t, i, j, 0);
    adj::uzc_column_adjoint<real>(nk, d.sk, hnew + o, g_gz_out + o, g_ws[idx2(d, t, i, j)], rdt, g_new + o);
  }));
  FV3B_CHECK(launch_box(Box{s - 1, e + 2, js - 1, je + 2, 0, nk}, st, [=] __device__(int t, int i, int j, int k) {
    real* const out[3] = {g_gz, g_ut, g_vt};
    auto add = [&](int a, idx_t o, real v) { atomicAdd(out[a] + o, v); };
    adj::uzc_point_adjoint<real>(d, t, i, j, k, g_new[idx3(d, t, i, j, k)], dp_ref, area, ut, vt, gz, add);
  }));
  return FV3B_OK;
}

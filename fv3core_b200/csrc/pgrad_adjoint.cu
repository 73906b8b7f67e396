// fv3b_p_grad_c_adjoint: the adjoint of p_grad_c_stencil
// (dyn_core.py:101-145) from pgrad_adjoint.h, one thread per input point of
// [is-1, ie+1] x [js-1, je+1] x interfaces 0..npz.
#include "ctx.cuh"
#include "pgrad_adjoint.h"
#include "stencil.cuh"

using namespace fv3b;

extern "C" int fv3b_p_grad_c_adjoint(fv3b_ctx* ctx, const real* delpc, const real* pkc, const real* gz,
                                     const real* gu, const real* gv, real* g_delpc, real* g_pkc, real* g_gz,
                                     double dt2_in, void* stream) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && delpc && pkc && gz && gu && gv && g_delpc && g_pkc && g_gz,
               "fv3b_p_grad_c_adjoint: null argument");
  const real dt2 = static_cast<real>(dt2_in);
  const Dims d = ctx->d;
  const real *rdxc = ctx->m.rdxc, *rdyc = ctx->m.rdyc;
  cudaStream_t st = (cudaStream_t)stream;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  FV3B_CHECK(launch_box(Box{s - 1, e + 2, js - 1, je + 2, 0, d.nk}, st, [=] __device__(int t, int i, int j, int k) {
    real a_delp, a_pk, a_gz;
    adj::pgc_point_adjoint<real>(d, t, i, j, k, dt2, rdxc, rdyc, delpc, pkc, gz, gu, gv, a_delp, a_pk, a_gz);
    const idx_t o = idx3(d, t, i, j, k);
    g_delpc[o] = a_delp;
    g_pkc[o] = a_pk;
    g_gz[o] = a_gz;
  }));
  return FV3B_OK;
}

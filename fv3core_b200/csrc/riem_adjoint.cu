// fv3b_riem_solver3_adjoint and fv3b_riem_solver_c_adjoint: the column
// adjoints of riem_adjoint.h over each solver's columns, one thread per
// column.  The per-level forward
// values and adjoints live in the thread's local memory (about 50 arrays of
// the level bucket), so this kernel favours simplicity over speed.
#include "common.cuh"
#include "riem_adjoint.h"

namespace fv3b {
namespace {

struct Riem3AdjArgs {
  double dt, ptop, p_fac;
  const real *cappa, *wsd, *q_con, *delp, *pt, *zh, *w, *gw_out, *gdz_out;
  real *g_w, *g_zh, *g_delp, *g_pt, *g_wsd;
};

template <int NK>
cudaError_t launch_adjoint(const Dims& d, cudaStream_t s, const Riem3AdjArgs a) {
  const Dims dd = d;
  return launch_columns(d.isc, d.iec + 1, d.jsc, d.jec + 1, s, [=] __device__(int t, int i, int j) {
    const idx_t o = idx3(dd, t, i, j, 0);
    adj::riem3_column_adjoint<NK, real, real>(dd.nk, dd.sk, a.dt, a.ptop, a.p_fac, (double)a.wsd[idx2(dd, t, i, j)],
                                              a.w + o, a.zh + o, a.delp + o, a.pt + o, a.cappa + o, a.q_con + o,
                                              a.gw_out + o, a.gdz_out + o, a.g_w + o, a.g_zh + o, a.g_delp + o,
                                              a.g_pt + o, a.g_wsd + idx2(dd, t, i, j));
  }, 64);
}

struct RiemCAdjArgs {
  double dt2, ptop, p_fac;
  const real *cappa, *ws, *q_con, *delpc, *ptc, *gz, *w3, *gpef_out, *ggz_out;
  real *g_w3, *g_gz, *g_delpc, *g_ptc, *g_ws;
};

template <int NK>
cudaError_t launch_adjoint_c(const Dims& d, cudaStream_t s, const RiemCAdjArgs a) {
  const Dims dd = d;
  return launch_columns(d.isc - 1, d.iec + 2, d.jsc - 1, d.jec + 2, s, [=] __device__(int t, int i, int j) {
    const idx_t o = idx3(dd, t, i, j, 0);
    adj::riemc_column_adjoint<NK, real, real>(dd.nk, dd.sk, a.dt2, a.ptop, a.p_fac, (double)a.ws[idx2(dd, t, i, j)],
                                              a.w3 + o, a.gz + o, a.delpc + o, a.ptc + o, a.cappa + o, a.q_con + o,
                                              a.gpef_out + o, a.ggz_out + o, a.g_w3 + o, a.g_gz + o, a.g_delpc + o,
                                              a.g_ptc + o, a.g_ws + idx2(dd, t, i, j));
  }, 64);
}

}  // namespace
}  // namespace fv3b

using namespace fv3b;

extern "C" int fv3b_riem_solver3_adjoint(const fv3b_grid_dims* dims, double dt, double ptop, double p_fac,
                                         const real* cappa, const real* wsd, const real* q_con, const real* delp,
                                         const real* pt, const real* zh, const real* w, const real* gw_out,
                                         const real* gdz_out, real* g_w, real* g_zh, real* g_delp, real* g_pt,
                                         real* g_wsd, void* stream) {
  FV3B_REQUIRE(dims && cappa && wsd && q_con && delp && pt && zh && w && gw_out && gdz_out && g_w && g_zh && g_delp &&
                   g_pt && g_wsd,
               "fv3b_riem_solver3_adjoint: null argument");
  FV3B_REQUIRE(dims_fit(dims), "fv3b_riem_solver3_adjoint: a 3-D field of the six tiles must hold fewer than 2^31 elements");
  const Dims d = make_dims(dims);
  FV3B_REQUIRE(d.nk >= 4 && d.nk <= 128, "fv3b_riem_solver3_adjoint: npz must be in 3..127");
  const Riem3AdjArgs a{dt, ptop, p_fac, cappa, wsd, q_con, delp, pt, zh, w, gw_out, gdz_out, g_w, g_zh, g_delp, g_pt, g_wsd};
  cudaStream_t s = (cudaStream_t)stream;
  if (d.nk <= 16) FV3B_CHECK(launch_adjoint<16>(d, s, a));
  else if (d.nk <= 32) FV3B_CHECK(launch_adjoint<32>(d, s, a));
  else if (d.nk <= 64) FV3B_CHECK(launch_adjoint<64>(d, s, a));
  else if (d.nk <= 80) FV3B_CHECK(launch_adjoint<80>(d, s, a));
  else FV3B_CHECK(launch_adjoint<128>(d, s, a));
  return FV3B_OK;
}

extern "C" int fv3b_riem_solver_c_adjoint(const fv3b_grid_dims* dims, double dt2, double ptop, double p_fac,
                                          const real* cappa, const real* ws, const real* q_con, const real* delpc,
                                          const real* ptc, const real* gz, const real* w3, const real* gpef_out,
                                          const real* ggz_out, real* g_w3, real* g_gz, real* g_delpc, real* g_ptc,
                                          real* g_ws, void* stream) {
  FV3B_REQUIRE(dims && cappa && ws && q_con && delpc && ptc && gz && w3 && gpef_out && ggz_out && g_w3 && g_gz &&
                   g_delpc && g_ptc && g_ws,
               "fv3b_riem_solver_c_adjoint: null argument");
  FV3B_REQUIRE(dims_fit(dims), "fv3b_riem_solver_c_adjoint: a 3-D field of the six tiles must hold fewer than 2^31 elements");
  const Dims d = make_dims(dims);
  FV3B_REQUIRE(d.nk >= 4 && d.nk <= 128, "fv3b_riem_solver_c_adjoint: npz must be in 3..127");
  const RiemCAdjArgs a{dt2, ptop, p_fac, cappa, ws, q_con, delpc, ptc, gz, w3, gpef_out, ggz_out,
                       g_w3, g_gz, g_delpc, g_ptc, g_ws};
  cudaStream_t s = (cudaStream_t)stream;
  if (d.nk <= 16) FV3B_CHECK(launch_adjoint_c<16>(d, s, a));
  else if (d.nk <= 32) FV3B_CHECK(launch_adjoint_c<32>(d, s, a));
  else if (d.nk <= 64) FV3B_CHECK(launch_adjoint_c<64>(d, s, a));
  else if (d.nk <= 80) FV3B_CHECK(launch_adjoint_c<80>(d, s, a));
  else FV3B_CHECK(launch_adjoint_c<128>(d, s, a));
  return FV3B_OK;
}

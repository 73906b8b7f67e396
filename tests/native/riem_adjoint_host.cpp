// Host build of the RiemannSolver3 column adjoint (fv3core_b200/csrc/riem_adjoint.h)
// for the CPU tests: columns are rows of [ncol][K] arrays.
#include "../../fv3core_b200/csrc/riem_adjoint.h"

extern "C" void riem3_adjoint_columns(int ncol, int K, double dt, double ptop, double p_fac, const double* wsr,
                                      const double* w, const double* zh, const double* delp, const double* pt,
                                      const double* cappa, const double* q_con, const double* gw,
                                      const double* gdz, double* g_w, double* g_zh, double* g_delp,
                                      double* g_pt, double* g_wsr) {
  for (int c = 0; c < ncol; ++c) {
    const long long o = (long long)c * K;
    fv3b::adj::riem3_column_adjoint<128, double, double>(K, 1, dt, ptop, p_fac, wsr[c], w + o, zh + o, delp + o,
                                                         pt + o, cappa + o, q_con + o, gw + o, gdz + o, g_w + o,
                                                         g_zh + o, g_delp + o, g_pt + o, g_wsr + c);
  }
}

extern "C" void riemc_adjoint_columns(int ncol, int K, double dt2, double ptop, double p_fac, const double* wsr,
                                      const double* w3, const double* gz, const double* delpc, const double* ptc,
                                      const double* cappa, const double* q_con, const double* gpef,
                                      const double* ggz, double* g_w3, double* g_gz, double* g_delpc,
                                      double* g_ptc, double* g_wsr) {
  for (int c = 0; c < ncol; ++c) {
    const long long o = (long long)c * K;
    fv3b::adj::riemc_column_adjoint<128, double, double>(K, 1, dt2, ptop, p_fac, wsr[c], w3 + o, gz + o,
                                                         delpc + o, ptc + o, cappa + o, q_con + o, gpef + o,
                                                         ggz + o, g_w3 + o, g_gz + o, g_delpc + o, g_ptc + o,
                                                         g_wsr + c);
  }
}

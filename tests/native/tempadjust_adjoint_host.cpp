// Host build of the compute_pkz_tempadjust point adjoint
// (fv3core_b200/csrc/tempadjust_adjoint.h) for the CPU tests, over flat
// arrays of points.
#include "../../fv3core_b200/csrc/tempadjust_adjoint.h"

extern "C" void tempadjust_adjoint_host(int npts, const double* dp, const double* dz, const double* pt,
                                        const double* heat, const double* cappa, const double* lim, double rdg,
                                        double cv, const double* gt, const double* gk, double* a_dp, double* a_dz,
                                        double* a_pt, double* a_heat) {
  for (int q = 0; q < npts; ++q)
    fv3b::adj::tempadjust_point_adjoint<double>(dp[q], dz[q], pt[q], heat[q], cappa[q], lim[q], rdg, cv, gt[q], gk[q],
                                                a_dp[q], a_dz[q], a_pt[q], a_heat[q]);
}

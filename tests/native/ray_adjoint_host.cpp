// Host build of the Rayleigh-damping column adjoint
// (fv3core_b200/csrc/ray_adjoint.h) for the CPU tests, on winds in the
// device layout [6][npz+1][nj][ni].  The damping constants are derived here
// as RayleighDamping derives them (ray_fast.py:130-167).
#include <cmath>
#include <vector>

#include "../../fv3core_b200/csrc/ray_adjoint.h"

extern "C" void ray_adjoint_host(int n, int halo, int npz, const double* dp, const double* pfull, double dt,
                                 double ptop, double rf_cutoff, double tau, double* gu, double* gv, double* gw) {
  fv3b_grid_dims g{n, halo, npz, 0};
  const fv3b::Dims d = fv3b::make_dims(&g);
  const double pi = 3.141592653589793, sday = 86400.0;
  const double nudge = rf_cutoff + std::fmin(100.0, 10.0 * ptop);
  std::vector<double> rf(npz, 1.0), dm(npz, 0.0);
  int k_rf = 0, k_nudge = 0;
  while (k_rf < npz && pfull[k_rf] < rf_cutoff) ++k_rf;
  while (k_nudge < npz && pfull[k_nudge] < nudge) ++k_nudge;
  if (k_rf == 0) return;
  for (int k = 0; k < k_rf; ++k) {
    const double sn = std::sin(0.5 * pi * std::log(rf_cutoff / pfull[k]) / std::log(rf_cutoff / ptop));
    rf[k] = 1.0 / (1.0 + dt / (tau * sday) * sn * sn);
  }
  dm[0] = dp[0];
  for (int k = 1; k < k_nudge; ++k) dm[k] = dm[k - 1] + dp[k];
  for (int k = k_nudge - 2; k >= 0; --k) dm[k] = dm[k + 1];
  for (int t = 0; t < 6; ++t)
    for (int j = d.jsc; j <= d.jec + 1; ++j)
      for (int i = d.isc; i <= d.iec + 1; ++i) {
        const fv3b::idx_t o = fv3b::idx3(d, t, i, j, 0);
        if (i <= d.iec) fv3b::adj::ray_column_adjoint<double>(k_rf, k_nudge, d.sk, rf.data(), dm.data(), dp, gu + o);
        if (j <= d.jec) fv3b::adj::ray_column_adjoint<double>(k_rf, k_nudge, d.sk, rf.data(), dm.data(), dp, gv + o);
        if (i <= d.iec && j <= d.jec) fv3b::adj::ray_w_column_adjoint<double>(k_rf, d.sk, rf.data(), gw + o);
      }
}

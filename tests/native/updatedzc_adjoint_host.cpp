// Host build of the UpdateGeopotentialHeightOnCGrid adjoint
// (fv3core_b200/csrc/updatedzc_adjoint.h) for the CPU tests: fields in the
// device layout [6][npz+1][nj][ni], 2-D fields [6][nj][ni].  The same four
// steps as the device wrapper, run serially.
#include "../../fv3core_b200/csrc/updatedzc_adjoint.h"

namespace {
fv3b::Dims dims_of(int n, int halo, int npz) {
  fv3b_grid_dims g{n, halo, npz, 0};
  return fv3b::make_dims(&g);
}
}  // namespace

// The header's forward: the new gz (floor included) and ws on the updated box.
extern "C" void uzc_forward_host(int n, int halo, int npz, double dt, const double* dp0, const double* area,
                                 const double* zs, const double* ut, const double* vt, const double* gz,
                                 double* gz_out, double* ws) {
  const fv3b::Dims d = dims_of(n, halo, npz);
  for (int t = 0; t < 6; ++t)
    for (int j = d.jsc - 1; j <= d.jec + 1; ++j)
      for (int i = d.isc - 1; i <= d.iec + 1; ++i) {
        double below = fv3b::adj::uzc_new<double>(d, t, i, j, d.nk - 1, dp0, area, ut, vt, gz);
        gz_out[fv3b::idx3(d, t, i, j, d.nk - 1)] = below;
        ws[fv3b::idx2(d, t, i, j)] = (zs[fv3b::idx2(d, t, i, j)] - below) * (1.0 / dt);
        for (int k = d.nk - 2; k >= 0; --k) {
          const double v = fv3b::adj::uzc_new<double>(d, t, i, j, k, dp0, area, ut, vt, gz);
          const double kp1 = below + fv3b::adj::UZC_DZ_MIN;
          below = v > kp1 ? v : kp1;
          gz_out[fv3b::idx3(d, t, i, j, k)] = below;
        }
      }
}

extern "C" void uzc_adjoint_host(int n, int halo, int npz, double dt, const double* dp0, const double* area,
                                 const double* ut, const double* vt, const double* gz, const double* g_gz_out,
                                 const double* g_ws, double* g_gz, double* g_ut, double* g_vt, double* hnew,
                                 double* g_new) {
  const fv3b::Dims d = dims_of(n, halo, npz);
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  for (int t = 0; t < 6; ++t)
    for (int k = 0; k < d.nk; ++k)
      for (int j = 0; j < d.nj; ++j)
        for (int i = 0; i < d.ni; ++i) {
          const fv3b::idx_t o = fv3b::idx3(d, t, i, j, k);
          const bool updated = i >= s - 1 && i <= e + 1 && j >= js - 1 && j <= je + 1;
          g_gz[o] = updated ? 0.0 : g_gz_out[o];
          g_ut[o] = g_vt[o] = 0.0;
          if (updated) hnew[o] = fv3b::adj::uzc_new<double>(d, t, i, j, k, dp0, area, ut, vt, gz);
        }
  for (int t = 0; t < 6; ++t)
    for (int j = js - 1; j <= je + 1; ++j)
      for (int i = s - 1; i <= e + 1; ++i) {
        const fv3b::idx_t o = fv3b::idx3(d, t, i, j, 0);
        fv3b::adj::uzc_column_adjoint<double>(d.nk, d.sk, hnew + o, g_gz_out + o, g_ws[fv3b::idx2(d, t, i, j)],
                                              1.0 / dt, g_new + o);
      }
  double* const out[3] = {g_gz, g_ut, g_vt};
  auto add = [&](int a, fv3b::idx_t o, double v) { out[a][o] += v; };
  for (int t = 0; t < 6; ++t)
    for (int k = 0; k < d.nk; ++k)
      for (int j = js - 1; j <= je + 1; ++j)
        for (int i = s - 1; i <= e + 1; ++i)
          fv3b::adj::uzc_point_adjoint<double>(d, t, i, j, k, g_new[fv3b::idx3(d, t, i, j, k)], dp0, area, ut, vt,
                                               gz, add);
}

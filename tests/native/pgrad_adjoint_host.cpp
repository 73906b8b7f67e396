// Host build of the p_grad_c adjoint (fv3core_b200/csrc/pgrad_adjoint.h) for
// the CPU tests: fields in the device layout [6][npz+1][nj][ni], metrics
// [6][nj][ni]; writes the three gradients on the adjoint's box.
#include "../../fv3core_b200/csrc/pgrad_adjoint.h"

extern "C" void pgc_adjoint_host(int n, int halo, int npz, double dt2, const double* rdxc, const double* rdyc,
                                 const double* delpc, const double* pkc, const double* gz, const double* gu,
                                 const double* gv, double* g_delpc, double* g_pkc, double* g_gz) {
  fv3b_grid_dims g{n, halo, npz, 0};
  const fv3b::Dims d = fv3b::make_dims(&g);
  for (int t = 0; t < 6; ++t)
    for (int k = 0; k < d.nk; ++k)
      for (int j = d.jsc - 1; j <= d.jec + 1; ++j)
        for (int i = d.isc - 1; i <= d.iec + 1; ++i) {
          const fv3b::idx_t o = fv3b::idx3(d, t, i, j, k);
          fv3b::adj::pgc_point_adjoint<double>(d, t, i, j, k, dt2, rdxc, rdyc, delpc, pkc, gz, gu, gv, g_delpc[o],
                                               g_pkc[o], g_gz[o]);
        }
}

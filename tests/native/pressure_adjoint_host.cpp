// Host build of the halo-ring column adjoints
// (fv3core_b200/csrc/pressure_adjoint.h) for the CPU tests, on fields in the
// device layout [6][npz+1][nj][ni]; the same rings as the device wrappers.
#include "../../fv3core_b200/csrc/pressure_adjoint.h"

namespace {
template <class F>
void for_ring(int n, int halo, int npz, int width, F f) {
  fv3b_grid_dims g{n, halo, npz, 0};
  const fv3b::Dims d = fv3b::make_dims(&g);
  for (int t = 0; t < 6; ++t)
    for (int j = d.jsc - width; j <= d.jec + width; ++j)
      for (int i = d.isc - width; i <= d.iec + width; ++i) {
        if (i >= d.isc && i <= d.iec && j >= d.jsc && j <= d.jec) continue;
        f(d, fv3b::idx3(d, t, i, j, 0));
      }
}
}  // namespace

extern "C" void edge_pe_adjoint_host(int n, int halo, int npz, double* g_pe, double* g_delp) {
  for_ring(n, halo, npz, 1, [&](const fv3b::Dims& d, fv3b::idx_t o) {
    fv3b::adj::edge_pe_column_adjoint<double>(d.nk, d.sk, g_pe + o, g_delp + o);
  });
}

extern "C" void pk3_halo_adjoint_host(int n, int halo, int npz, double ptop, double akap, const double* delp,
                                      double* g_pk3, double* g_delp) {
  for_ring(n, halo, npz, 2, [&](const fv3b::Dims& d, fv3b::idx_t o) {
    fv3b::adj::pk3_column_adjoint<double>(d.nk, d.sk, ptop, akap, delp + o, g_pk3 + o, g_delp + o);
  });
}

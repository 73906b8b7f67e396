// Host build of the halo-update transposes (fv3core_b200/csrc/halo_adjoint.h)
// for the CPU tests: the same two passes as the device kernels, run
// serially, on fields in the device layout [6][npz+1][nj][ni].
#include "../../fv3core_b200/csrc/halo_adjoint.h"

namespace {
fv3b::Dims dims_of(int n, int halo, int npz) {
  fv3b_grid_dims g{n, halo, npz, 0};
  return fv3b::make_dims(&g);
}

void transpose(const fv3b::Dims& d, double* gx, double* gy, const int sx[2], const int sy[2], int ncomp,
               int n_halo, int nlev) {
  for (int zero = 0; zero < 2; ++zero)
    for (int t = 0; t < 6; ++t)
      for (int comp = 0; comp < ncomp; ++comp)
        for (int p = 0; p < fv3b::halo_candidates(d, n_halo); ++p) {
          fv3b::HaloCopy c;
          if (!fv3b::halo_copy(d, t, p, comp, sx, sy, n_halo, c)) continue;
          double* gd = comp == 0 ? gx : gy;
          double* gs = c.src_comp == 0 ? gx : gy;
          for (int k = 0; k < nlev; ++k) {
            if (zero) gd[c.dst + k * d.sk] = 0.0;
            else gs[c.src + k * d.sk] += (ncomp == 2 ? c.sign : 1) * gd[c.dst + k * d.sk];
          }
        }
}
}  // namespace

extern "C" void halo_scalar_adjoint_host(int n, int halo, int npz, double* g, int stagger, int n_halo, int nlev) {
  const int s[2] = {stagger, stagger};
  transpose(dims_of(n, halo, npz), g, g, s, s, 1, n_halo, nlev);
}

extern "C" void halo_vector_adjoint_host(int n, int halo, int npz, double* gx, double* gy, int grid, int nlev) {
  const int c = grid == 1;
  const int sx[2] = {c ? 0 : 1, c ? 1 : 0}, sy[2] = {c ? 1 : 0, c ? 0 : 1};
  transpose(dims_of(n, halo, npz), gx, gy, sx, sy, 2, halo, nlev);
}

extern "C" void interface_sync_adjoint_host(int n, int halo, int npz, double* gu, double* gv, int nlev) {
  const fv3b::Dims d = dims_of(n, halo, npz);
  for (int zero = 0; zero < 2; ++zero)
    for (int t = 0; t < 6; ++t)
      for (int comp = 0; comp < 2; ++comp)
        for (int a = 0; a < n; ++a) {
          int dst_comp;
          const fv3b::HaloCopy c = fv3b::interface_sync_copy(d, t, comp, a, dst_comp);
          double* gd = dst_comp == 0 ? gu : gv;
          double* gs = comp == 0 ? gu : gv;
          for (int k = 0; k < nlev; ++k) {
            if (zero) gd[c.dst + k * d.sk] = 0.0;
            else gs[c.src + k * d.sk] += c.sign * gd[c.dst + k * d.sk];
          }
        }
}

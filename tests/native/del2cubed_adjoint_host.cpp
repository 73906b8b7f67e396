// Host build of the del2cubed pass functions and their transposes
// (fv3core_b200/csrc/del2cubed_adjoint.h) for the CPU tests: fields in the
// device layout [6][npz+1][nj][ni], metrics [6][nj][ni].
#include <vector>

#include "../../fv3core_b200/csrc/del2cubed_adjoint.h"

namespace {
fv3b::Dims dims_of(int n, int halo, int npz) {
  fv3b_grid_dims g{n, halo, npz, 0};
  return fv3b::make_dims(&g);
}
}  // namespace

// qdel filtered in place, levels 0..npz-1
extern "C" void del2cubed_forward_host(int n, int halo, int npz, double cd, int nmax, const double* del6_u,
                                       const double* del6_v, const double* rarea, double* qdel) {
  const fv3b::Dims d = dims_of(n, halo, npz);
  const int full = d.ni - 1, ntimes = nmax < 3 ? nmax : 3;
  std::vector<double> in(qdel, qdel + (size_t)6 * d.st);
  for (int p = 0; p < ntimes; ++p) {
    const int nt = ntimes - (p + 1);
    in.assign(qdel, qdel + (size_t)6 * d.st);
    for (int t = 0; t < 6; ++t)
      for (int k = 0; k < d.nz; ++k) {
        auto qd = [&](int ii, int jj) { return in[fv3b::idx3(d, t, ii, jj, k)]; };
        for (int j = 0; j < full; ++j)
          for (int i = 0; i < full; ++i)
            qdel[fv3b::idx3(d, t, i, j, k)] =
                fv3b::adj::d2c_pass_value<double>(d, t, i, j, nt, cd, del6_u, del6_v, rarea, qd);
      }
  }
}

// g (the cotangent of the filtered field) turned in place into that of the
// field before the filter
extern "C" void del2cubed_adjoint_host(int n, int halo, int npz, double cd, int nmax, const double* del6_u,
                                       const double* del6_v, const double* rarea, double* g) {
  const fv3b::Dims d = dims_of(n, halo, npz);
  const int full = d.ni - 1, ntimes = nmax < 3 ? nmax : 3;
  std::vector<double> nxt((size_t)6 * d.st);
  for (int p = ntimes - 1; p >= 0; --p) {
    const int nt = ntimes - (p + 1);
    nxt.assign((size_t)6 * d.st, 0.0);
    auto add = [&](fv3b::idx_t o, double v) { nxt[o] += v; };
    for (int t = 0; t < 6; ++t)
      for (int k = 0; k < d.nz; ++k)
        for (int j = 0; j < d.nj; ++j)
          for (int i = 0; i < d.ni; ++i) {
            const fv3b::idx_t o = fv3b::idx3(d, t, i, j, k);
            if (i == full || j == full) nxt[o] += g[o];
            else fv3b::adj::d2c_pass_adjoint<double>(d, t, i, j, k, nt, cd, del6_u, del6_v, rarea, g[o], add);
          }
    for (int t = 0; t < 6; ++t)
      for (int k = 0; k < d.nz; ++k)
        for (int j = 0; j < d.nj; ++j)
          for (int i = 0; i < d.ni; ++i) g[fv3b::idx3(d, t, i, j, k)] = nxt[fv3b::idx3(d, t, i, j, k)];
  }
}

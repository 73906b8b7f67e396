// Host build of the a2b_ord4 point functions and their transposes
// (fv3core_b200/csrc/a2b_adjoint.h) for the CPU tests: 3-D fields in the
// device layout [6][npz+1][nj][ni], dxa/dya [6][nj][ni], edge factors
// [6][n+1], corner ratios [6][4][3].
#include <vector>

#include "../../fv3core_b200/csrc/a2b_adjoint.h"

namespace {
using fv3b::Dims;
using fv3b::idx3;

Dims dims_of(int n, int halo, int npz) {
  fv3b_grid_dims g{n, halo, npz, 0};
  return fv3b::make_dims(&g);
}

template <class F>
void for_boundary(const Dims& d, F f) {
  for (int i = d.isc; i <= d.iec + 1; ++i) {
    f(i, d.jsc);
    f(i, d.jec + 1);
  }
  for (int j = d.jsc + 1; j <= d.jec; ++j) {
    f(d.isc, j);
    f(d.iec + 1, j);
  }
}
}  // namespace

// qout on [is, ie+1] x [js, je+1], levels [k0, k1), from qin
extern "C" void a2b_forward_host(int n, int halo, int npz, int k0, int k1, const double* dxa, const double* dya,
                                 const double* ew, const double* ee, const double* es, const double* en,
                                 const double* extrap, const double* qin, double* qout) {
  const Dims d = dims_of(n, halo, npz);
  const fv3b::adj::A2BGrid<double> g{dxa, dya, ew, ee, es, en, extrap};
  const size_t size = (size_t)6 * d.st;
  std::vector<double> qx(size, 0.0), qy(size, 0.0), edges(size, 0.0);
  for (int t = 0; t < 6; ++t)
    for (int k = k0; k < k1; ++k) {
      for_boundary(d, [&](int i, int j) {
        auto q = [&](int di, int dj) { return qin[idx3(d, t, i + di, j + dj, k)]; };
        const double v = fv3b::adj::a2b_boundary_value<double>(d, t, i, j, g, q);
        qout[idx3(d, t, i, j, k)] = v;
        edges[idx3(d, t, i, j, k)] = v;
      });
      for (int j = d.jsc - 2; j <= d.jec + 2; ++j)
        for (int i = d.isc - 2; i <= d.iec + 2; ++i) {
          const fv3b::idx_t o = idx3(d, t, i, j, k), b2 = fv3b::idx2(d, t, i, j);
          if (i >= d.isc && i <= d.iec + 1) {
            auto q = [&](int m) { return qin[o + m]; };
            auto sp = [&](int m) { return dxa[b2 + m]; };
            qx[o] = fv3b::adj::a2b_volume_mean<double>(q, sp, i, d.isc, d.iec);
          }
          if (j >= d.jsc && j <= d.jec + 1) {
            auto q = [&](int m) { return qin[o + m * d.sj]; };
            auto sp = [&](int m) { return dya[b2 + m * d.ni]; };
            qy[o] = fv3b::adj::a2b_volume_mean<double>(q, sp, j, d.jsc, d.jec);
          }
        }
      for (int j = d.jsc + 1; j <= d.jec; ++j)
        for (int i = d.isc + 1; i <= d.iec; ++i) {
          const double* arr[3] = {qx.data(), qy.data(), edges.data()};
          auto q = [&](int a, int di, int dj) { return arr[a][idx3(d, t, i + di, j + dj, k)]; };
          qout[idx3(d, t, i, j, k)] = fv3b::adj::a2b_interior_value<double>(d, i, j, q);
        }
    }
}

// gin += the transpose applied to gout (read on [is, ie+1] x [js, je+1],
// levels [k0, k1))
extern "C" void a2b_adjoint_host(int n, int halo, int npz, int k0, int k1, const double* dxa, const double* dya,
                                 const double* ew, const double* ee, const double* es, const double* en,
                                 const double* extrap, const double* gout, double* gin) {
  const Dims d = dims_of(n, halo, npz);
  const fv3b::adj::A2BGrid<double> g{dxa, dya, ew, ee, es, en, extrap};
  const size_t size = (size_t)6 * d.st;
  std::vector<double> gqx(size, 0.0), gqy(size, 0.0), gedges(size, 0.0);
  double* const out[4] = {gqx.data(), gqy.data(), gedges.data(), gin};
  auto add = [&](int a, fv3b::idx_t o, double v) { out[a][o] += v; };
  for (int t = 0; t < 6; ++t)
    for (int k = k0; k < k1; ++k) {
      for (int j = d.jsc + 1; j <= d.jec; ++j)
        for (int i = d.isc + 1; i <= d.iec; ++i)
          fv3b::adj::a2b_interior_adjoint<double>(d, t, i, j, k, gout[idx3(d, t, i, j, k)], add);
      for (int j = d.jsc - 2; j <= d.jec + 2; ++j)
        for (int i = d.isc - 2; i <= d.iec + 2; ++i) {
          const fv3b::idx_t o = idx3(d, t, i, j, k);
          fv3b::adj::a2b_volume_mean_adjoint<double>(d, g, t, i, j, k, gqx[o], gqy[o], add);
        }
      for_boundary(d, [&](int i, int j) {
        const fv3b::idx_t o = idx3(d, t, i, j, k);
        fv3b::adj::a2b_boundary_adjoint<double>(d, g, t, i, j, k, gout[o] + gedges[o], add);
      });
    }
}

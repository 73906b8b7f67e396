// Host build of the a2b_ord4 point functions and their transposes
// (fv3core_b200/csrc/a2b_adjoint.h), and of the nh_p_grad adjoint built on
// them (fv3core_b200/csrc/nh_p_grad_adjoint.h), for the CPU tests: 3-D
// fields in the device layout [6][npz+1][nj][ni], 2-D fields [6][nj][ni],
// edge factors [6][n+1], corner ratios [6][4][3].
#include <cmath>
#include <vector>

#include "../../fv3core_b200/csrc/a2b_adjoint.h"
#include "../../fv3core_b200/csrc/nh_p_grad_adjoint.h"

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

// The gradients of <gu, u'> + <gv, v'> + <gpp, pp'> + <gpk3, pk3'> +
// <ggz, gz'> of NonHydrostaticPressureGradient with respect to its inputs
// u, v, pp, pk3, gz (pass-through included) and delp; ptk = ptop^akap.
extern "C" void nhp_adjoint_host(int n, int halo, int npz, double dt, double ptk, const double* dxa,
                                 const double* dya, const double* ew, const double* ee, const double* es,
                                 const double* en, const double* extrap, const double* rdx, const double* rdy,
                                 const double* pp, const double* pk3, const double* gz, const double* delp,
                                 const double* gu, const double* gv, const double* gpp, const double* gpk3,
                                 const double* ggz, double* g_u, double* g_v, double* g_pp, double* g_pk3,
                                 double* g_gz, double* g_delp) {
  const Dims d = dims_of(n, halo, npz);
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec, nk = d.nk, nz = d.nz;
  const size_t size = (size_t)6 * d.st;
  std::vector<double> b[4] = {std::vector<double>(size, 0.0), std::vector<double>(size, 0.0),
                              std::vector<double>(size, 0.0), std::vector<double>(size, 0.0)};
  std::vector<double> gb[4] = {std::vector<double>(size, 0.0), std::vector<double>(size, 0.0),
                               std::vector<double>(size, 0.0), std::vector<double>(size, 0.0)};
  a2b_forward_host(n, halo, npz, 1, nk, dxa, dya, ew, ee, es, en, extrap, pp, b[0].data());
  a2b_forward_host(n, halo, npz, 1, nk, dxa, dya, ew, ee, es, en, extrap, pk3, b[1].data());
  a2b_forward_host(n, halo, npz, 0, nk, dxa, dya, ew, ee, es, en, extrap, gz, b[2].data());
  a2b_forward_host(n, halo, npz, 0, nz, dxa, dya, ew, ee, es, en, extrap, delp, b[3].data());
  for (int t = 0; t < 6; ++t)
    for (int k = 0; k < nk; ++k)
      for (int j = 0; j < d.nj; ++j)
        for (int i = 0; i < d.ni; ++i) {
          const fv3b::idx_t o = idx3(d, t, i, j, k);
          const bool box = i >= s && i <= e + 1 && j >= js && j <= je + 1;
          g_u[o] = (k < nz && i >= s && i <= e && j >= js && j <= je + 1) ? 0.0 : gu[o];
          g_v[o] = (k < nz && i >= s && i <= e + 1 && j >= js && j <= je) ? 0.0 : gv[o];
          g_pp[o] = box ? 0.0 : gpp[o];
          g_pk3[o] = box ? 0.0 : gpk3[o];
          g_gz[o] = box ? 0.0 : ggz[o];
          g_delp[o] = 0.0;
          if (box) {
            if (k > 0) {
              gb[0][o] += gpp[o];
              gb[1][o] += gpk3[o];
            }
            gb[2][o] += ggz[o];
          }
        }
  for (int dir = 0; dir < 2; ++dir) {
    double* gw = dir == 0 ? g_u : g_v;
    const double* G = dir == 0 ? gu : gv;
    auto add = [&](int a, fv3b::idx_t o, double v) {
      if (a == 4) gw[o] += v;
      else gb[a][o] += v;
    };
    for (int t = 0; t < 6; ++t)
      for (int k = 0; k < nz; ++k)
        for (int j = js; j <= je + (dir == 0 ? 1 : 0); ++j)
          for (int i = s; i <= e + (dir == 1 ? 1 : 0); ++i)
            fv3b::adj::nhp_wind_adjoint<double>(d, t, i, j, k, dir, G[idx3(d, t, i, j, k)], dt, ptk,
                                                dir == 0 ? rdx : rdy, b[0].data(), b[1].data(), b[2].data(),
                                                b[3].data(), add);
  }
  a2b_adjoint_host(n, halo, npz, 1, nk, dxa, dya, ew, ee, es, en, extrap, gb[0].data(), g_pp);
  a2b_adjoint_host(n, halo, npz, 1, nk, dxa, dya, ew, ee, es, en, extrap, gb[1].data(), g_pk3);
  a2b_adjoint_host(n, halo, npz, 0, nk, dxa, dya, ew, ee, es, en, extrap, gb[2].data(), g_gz);
  a2b_adjoint_host(n, halo, npz, 0, nz, dxa, dya, ew, ee, es, en, extrap, gb[3].data(), g_delp);
}

// Host build of the device grid generator's point functions
// (fv3core_b200/csrc/grid_gen.h), for a CPU test against the numpy
// generator fv3core_b200/grid.py.  Fields come out in the numpy layout
// [f][t][i][j].
#include <math.h>

#include "../../fv3core_b200/csrc/grid_gen.h"

extern "C" void grid_gen_host(int n, int h, int lattice, double radius, double omega, double* fields, double* edges,
                              double* a2b, double* scalars) {
  using namespace fv3b;
  fv3b_grid_dims gd{n, h, 1, 0};
  gg::Grid g;
  g.d = make_dims(&gd);
  g.n = n;
  g.h = h;
  g.m = n + 2 * h + 1;
  g.lattice = lattice;
  g.radius = radius;
  g.omega = omega;
  const long long mm = (long long)g.m * g.m;
  for (int f = 0; f < gg::GF_COUNT; ++f)
    for (int t = 0; t < 6; ++t)
      for (int i = 0; i < g.m; ++i)
        for (int j = 0; j < g.m; ++j) fields[(f * 6LL + t) * mm + (long long)i * g.m + j] = gg::field_at(g, f, t, i, j);
  for (int e = 0; e < 4; ++e)
    for (int t = 0; t < 6; ++t)
      for (int j = 0; j <= n; ++j) edges[(e * 6 + t) * (n + 1) + j] = gg::edge_factor(g, e, t, j);
  for (int r = 0; r < 72; ++r) a2b[r] = gg::a2b_extrap_at(g, r / 12, (r / 3) % 4, r % 3);
  double amin = 1e300, amax = -1e300, cmin = 1e300, cmax = -1e300;
  for (int t = 0; t < 6; ++t) {
    for (int i = h; i < h + n; ++i)
      for (int j = h; j < h + n; ++j) {
        const double a = gg::area_at(g, t, i, j);
        amin = fmin(amin, a);
        amax = fmax(amax, a);
      }
    for (int i = h; i <= h + n; ++i)
      for (int j = h; j <= h + n; ++j) {
        const double a = gg::area_c_at(g, t, i, j);
        cmin = fmin(cmin, a);
        cmax = fmax(cmax, a);
      }
  }
  scalars[0] = amin;
  scalars[1] = amax;
  scalars[2] = cmin;
  scalars[3] = cmax;
}

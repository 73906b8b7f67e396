// The transpose of the fourth-order A-grid to B-grid interpolation
// (a2b_ord4.py, AGrid2BGridFourthOrder.__call__ 606-676), for the adjoints
// of the stages that interpolate with it.  Written for both the device and
// the host (the tests build it with g++, check its forward against the
// oracle and its transpose by the dot-product identity).
//
// a2b_ord4 is linear in its input and runs in three passes: the values on
// the boundary of [is, ie+1] x [js, je+1] (cube-corner extrapolations and
// edge-weighted means), the PPM volume means qx, qy, and the interior
// interpolation from qx, qy and the boundary values.  Each pass is written
// here once, as a point function of an accessor; its transpose evaluates the
// same point function on unit inputs to get the weight of every input the
// point reads, and adds the point's cotangent times that weight there.  So
// the transpose is exact to rounding and follows the forward's statement
// order (the edge rows override the general formulas) without restating it.
#pragma once

#include "dims.h"

namespace fv3b {
namespace adj {

// the grid terms the interpolation reads (kernel layout; edge factors
// [6][n+1], corner ratios [6][4][3] as in fv3b_metrics)
template <class R>
struct A2BGrid {
  const R *dxa, *dya, *edge_w, *edge_e, *edge_s, *edge_n, *extrap;
};

// pass 1: the value at a boundary point (i, j) of [is, ie+1] x [js, je+1];
// q(di, dj) reads the input at (i + di, j + dj)
template <class R, class Q>
__device__ inline R a2b_boundary_value(const Dims& d, int t, int i, int j, const A2BGrid<R>& g, const Q& q) {
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec, h = d.h, n = d.n;
  const bool wcol = i == s, ecol = i == e + 1, srow = j == js, nrow = j == je + 1;
  if ((wcol || ecol) && (srow || nrow)) {
    // offsets (near, far) of the three extrapolations (a2b_ord4.py:60-235)
    const int O[4][3][4] = {{{0, 0, 1, 1}, {-1, 0, -2, 1}, {0, -1, 1, -2}},
                            {{-1, 0, -2, 1}, {-1, -1, -2, -2}, {0, 0, 1, 1}},
                            {{-1, -1, -2, -2}, {0, -1, 1, -2}, {-1, 0, -2, 1}},
                            {{0, -1, 1, -2}, {-1, -1, -2, -2}, {0, 0, 1, 1}}};
    const int c = (wcol && srow) ? 0 : (ecol && srow) ? 1 : (ecol && nrow) ? 2 : 3;
    const R* ratio = g.extrap + (t * 4 + c) * 3;
    R sum = R(0);
    for (int m = 0; m < 3; ++m) {
      const R qa = q(O[c][m][0], O[c][m][1]), qb = q(O[c][m][2], O[c][m][3]);
      sum += qa + ratio[m] * (qa - qb);
    }
    return sum * (R(1) / R(3));
  }
  if (wcol || ecol) {
    const R w = (wcol ? g.edge_w : g.edge_e)[t * (n + 1) + (j - h)];
    auto q2 = [&](int dj) {
      const R a0 = g.dxa[idx2(d, t, i - 1, j + dj)], a1 = g.dxa[idx2(d, t, i, j + dj)];
      return (q(-1, dj) * a1 + q(0, dj) * a0) / (a0 + a1);
    };
    return w * q2(-1) + (R(1) - w) * q2(0);
  }
  const R w = (srow ? g.edge_s : g.edge_n)[t * (n + 1) + (i - h)];
  auto q1 = [&](int di) {
    const R a0 = g.dya[idx2(d, t, i + di, j - 1)], a1 = g.dya[idx2(d, t, i + di, j)];
    return (q(di, -1) * a1 + q(di, 0) * a0) / (a0 + a1);
  };
  return w * q1(-1) + (R(1) - w) * q1(0);
}

// pass 2: ppm_volume_mean (a2b_ord4.py:340-451) at position pos of one
// axis; q(o) reads the input at offset o along it, sp(o) the spacing
template <class R, class Q, class S>
__device__ inline R a2b_volume_mean(const Q& q, const S& sp, int pos, int s, int e) {
  const R B1 = R(7) / R(12), B2 = -R(1) / R(12);
  auto side = [&](int a, int b, R gr) { return ((R(2) + gr) * q(a) - q(b)) / (R(1) + gr); };
  if (pos == e) {
    const R g_in = sp(-1) / sp(0), g_ou = sp(2) / sp(1);
    const R right = R(0.5) * (side(0, -1, g_in) + side(1, 2, g_ou));
    const R left = B2 * (q(-3) + q(0)) + B1 * (q(-2) + q(-1));
    return (R(3) * (q(-1) + g_in * q(0)) - (g_in * right + left)) / (R(2) + R(2) * g_in);
  }
  if (pos == e + 1) {
    const R g_in = sp(-2) / sp(-1), g_ou = sp(1) / sp(0);
    return R(0.5) * (side(-1, -2, g_in) + side(0, 1, g_ou));
  }
  if (pos == s + 1) {
    const R g_in = sp(0) / sp(-1), g_ou = sp(-3) / sp(-2);
    const R left = R(0.5) * (side(-1, 0, g_in) + side(-2, -3, g_ou));
    const R right = B2 * (q(-1) + q(2)) + B1 * (q(0) + q(1));
    return (R(3) * (g_in * q(-1) + q(0)) - (g_in * left + right)) / (R(2) + R(2) * g_in);
  }
  if (pos == s) {
    const R g_in = sp(1) / sp(0), g_ou = sp(-2) / sp(-1);
    return R(0.5) * (side(0, 1, g_in) + side(-1, -2, g_ou));
  }
  return B2 * (q(-2) + q(1)) + B1 * (q(-1) + q(0));
}

// pass 3: a2b_interpolation (a2b_ord4.py:286-310) at an interior corner
// (i, j); q(a, di, dj) reads array a (0 = qx, 1 = qy, 2 = boundary values)
// at (i + di, j + dj)
template <class R, class Q>
__device__ inline R a2b_interior_value(const Dims& d, int i, int j, const Q& q) {
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  const R C1 = R(2) / R(3), C2 = -R(1) / R(6), A1 = R(9) / R(16), A2 = -R(1) / R(16);
  R qxx = A2 * (q(0, 0, -2) + q(0, 0, 1)) + A1 * (q(0, 0, -1) + q(0, 0, 0));
  R qyy = A2 * (q(1, -2, 0) + q(1, 1, 0)) + A1 * (q(1, -1, 0) + q(1, 0, 0));
  if (j == js + 1) {
    const R up = A2 * (q(0, 0, -1) + q(0, 0, 2)) + A1 * (q(0, 0, 0) + q(0, 0, 1));
    qxx = C1 * (q(0, 0, -1) + q(0, 0, 0)) + C2 * (q(2, 0, -1) + up);
  }
  if (j == je) {
    const R lo = A2 * (q(0, 0, -3) + q(0, 0, 0)) + A1 * (q(0, 0, -2) + q(0, 0, -1));
    qxx = C1 * (q(0, 0, -1) + q(0, 0, 0)) + C2 * (q(2, 0, 1) + lo);
  }
  if (i == s + 1) {
    const R right = A2 * (q(1, -1, 0) + q(1, 2, 0)) + A1 * (q(1, 0, 0) + q(1, 1, 0));
    qyy = C1 * (q(1, -1, 0) + q(1, 0, 0)) + C2 * (q(2, -1, 0) + right);
  }
  if (i == e) {
    const R left = A2 * (q(1, -3, 0) + q(1, 0, 0)) + A1 * (q(1, -2, 0) + q(1, -1, 0));
    qyy = C1 * (q(1, -1, 0) + q(1, 0, 0)) + C2 * (q(2, 1, 0) + left);
  }
  return R(0.5) * (qxx + qyy);
}

// ---------------------------------------------------------------- transposes
// add(a, o, v) adds v to element o (a 3-D offset) of array a.

// pass 3 transposed at interior corner (t, i, j, k) with cotangent G: into
// the cotangents of qx (a = 0), qy (1) and the boundary values (2)
template <class R, class Add>
__device__ inline void a2b_interior_adjoint(const Dims& d, int t, int i, int j, int k, R G, Add add) {
  // the inputs a point can read: qx along j, qy along i, the four neighbours
  // of the boundary values
  for (int a = 0; a < 3; ++a) {
    const int lo = a == 2 ? -1 : -3, hi = a == 2 ? 1 : 2;
    for (int o = lo; o <= hi; ++o) {
      if (a == 2 && o == 0) continue;
      for (int dir = 0; dir < (a == 2 ? 2 : 1); ++dir) {
        // qx: offsets along j; qy: along i; boundary values: both
        const int di = (a == 1 || (a == 2 && dir == 0)) ? o : 0;
        const int dj = (a == 0 || (a == 2 && dir == 1)) ? o : 0;
        auto unit = [&](int b, int ei, int ej) { return (b == a && ei == di && ej == dj) ? R(1) : R(0); };
        const R w = a2b_interior_value<R>(d, i, j, unit);
        if (w != R(0)) add(a, idx3(d, t, i + di, j + dj, k), G * w);
      }
    }
  }
}

// pass 2 transposed: the cotangents gx of qx at (t, i, j, k) (when i is in
// [is, ie+1]) and gy of qy (when j is in [js, je+1]) into the input (a = 3)
template <class R, class Add>
__device__ inline void a2b_volume_mean_adjoint(const Dims& d, const A2BGrid<R>& g, int t, int i, int j, int k,
                                               R gx, R gy, Add add) {
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  const idx_t b2 = idx2(d, t, i, j);
  for (int o = -3; o <= 2; ++o) {
    if (i >= s && i < e + 2 && gx != R(0)) {
      auto unit = [&](int m) { return m == o ? R(1) : R(0); };
      auto sp = [&](int m) { return g.dxa[b2 + m]; };
      const R w = a2b_volume_mean<R>(unit, sp, i, s, e);
      if (w != R(0)) add(3, idx3(d, t, i + o, j, k), gx * w);
    }
    if (j >= js && j < je + 2 && gy != R(0)) {
      auto unit = [&](int m) { return m == o ? R(1) : R(0); };
      auto sp = [&](int m) { return g.dya[b2 + m * d.ni]; };
      const R w = a2b_volume_mean<R>(unit, sp, j, js, je);
      if (w != R(0)) add(3, idx3(d, t, i, j + o, k), gy * w);
    }
  }
}

// pass 1 transposed at boundary point (t, i, j, k) with cotangent G (of the
// output there plus that of the boundary value pass 3 read) into the input
// (a = 3)
template <class R, class Add>
__device__ inline void a2b_boundary_adjoint(const Dims& d, const A2BGrid<R>& g, int t, int i, int j, int k, R G,
                                            Add add) {
  for (int di = -2; di <= 1; ++di)
    for (int dj = -2; dj <= 1; ++dj) {
      auto unit = [&](int ei, int ej) { return (ei == di && ej == dj) ? R(1) : R(0); };
      const R w = a2b_boundary_value<R>(d, t, i, j, g, unit);
      if (w != R(0)) add(3, idx3(d, t, i + di, j + dj, k), G * w);
    }
}

}  // namespace adj
}  // namespace fv3b

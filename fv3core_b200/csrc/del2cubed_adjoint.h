// The transpose of HyperdiffusionDamping (del2cubed.py:152-181), for the
// adjoint of the heat-source filter; device and host.  Each of its passes is
// linear in the filtered field: the corner fill of the cube corners
// (del2cubed.py:41-75), the zonal and meridional fluxes of the filled field
// read through the corner copies, and the update on the compute domain
// plus nt halo rows, the rest of the field taking the filled copy.  The
// pass is written here as a point function of an accessor, and its transpose
// evaluates it on unit inputs at every point within reach to get that
// input's weight (the corner copies reach at most seven points away, the
// plain stencil one).
#pragma once

#include "corners.cuh"

namespace fv3b {
namespace adj {

constexpr int D2C_REACH = 7;

// One pass's output at (t, i, j) (i, j below ni - 1, the last row and column
// being left alone) from the accessor qd(ii, jj) of its input.
template <class R, class In>
__device__ inline R d2c_pass_value(const Dims& d, int t, int i, int j, int nt, R cd, const R* del6_u,
                                   const R* del6_v, const R* rarea, const In& qd) {
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  const R third = R(1) / R(3);
  // corner_fill at (ii, jj)
  auto cf = [&](int ii, int jj) {
    auto Q = [&](int di, int dj) { return qd(ii + di, jj + dj); };
    if (jj == js) {
      if (ii == s) return (Q(0, 0) + Q(-1, 0) + Q(0, -1)) * third;
      if (ii == s - 1) return (Q(1, 0) + Q(0, 0) + Q(1, -1)) * third;
      if (ii == e) return (Q(0, 0) + Q(1, 0) + Q(0, -1)) * third;
      if (ii == e + 1) return (Q(-1, 0) + Q(0, 0) + Q(-1, -1)) * third;
    } else if (jj == js - 1) {
      if (ii == s) return (Q(0, 1) + Q(-1, 1) + Q(0, 0)) * third;
      if (ii == e) return (Q(0, 1) + Q(1, 1) + Q(0, 0)) * third;
    } else if (jj == je) {
      if (ii == e) return (Q(0, 0) + Q(1, 0) + Q(0, 1)) * third;
      if (ii == e + 1) return (Q(-1, 0) + Q(0, 0) + Q(-1, 1)) * third;
      if (ii == s) return (Q(0, 0) + Q(-1, 0) + Q(0, 1)) * third;
      if (ii == s - 1) return (Q(1, 0) + Q(0, 0) + Q(1, 1)) * third;
    } else if (jj == je + 1) {
      if (ii == e) return (Q(0, -1) + Q(1, -1) + Q(0, 0)) * third;
      if (ii == s) return (Q(0, -1) + Q(-1, -1) + Q(0, 0)) * third;
    }
    return Q(0, 0);
  };
  auto qx = [&](int ii, int jj) {
    int si, sj;
    if (nt > 0 && copy_corner_x(d, ii, jj, si, sj)) return cf(si, sj);
    return cf(ii, jj);
  };
  auto qy = [&](int ii, int jj) {
    int si, sj;
    if (nt > 0 && copy_corner_y(d, ii, jj, si, sj)) return cf(si, sj);
    return cf(ii, jj);
  };
  R out = qy(i, j);
  if (i >= s - nt && i < e + 1 + nt && j >= js - nt && j < je + 1 + nt) {
    auto fx = [&](int ii, int jj) { return del6_v[idx2(d, t, ii, jj)] * (qx(ii - 1, jj) - qx(ii, jj)); };
    auto fy = [&](int ii, int jj) { return del6_u[idx2(d, t, ii, jj)] * (qy(ii, jj - 1) - qy(ii, jj)); };
    out = out + cd * rarea[idx2(d, t, i, j)] * (fx(i, j) - fx(i + 1, j) + fy(i, j) - fy(i, j + 1));
  }
  return out;
}

// One pass transposed at output (t, i, j, k) with cotangent G: add(o, v)
// adds v to the input's cotangent at 3-D offset o.
template <class R, class Add>
__device__ inline void d2c_pass_adjoint(const Dims& d, int t, int i, int j, int k, int nt, R cd, const R* del6_u,
                                        const R* del6_v, const R* rarea, R G, Add add) {
  if (G == R(0)) return;
  // away from the cube corners neither the corner fill nor the corner copies
  // act, and a point reads only its four neighbours
  const bool near_corner = (i <= d.isc + 2 || i >= d.iec - 2) && (j <= d.jsc + 2 || j >= d.jec - 2);
  const int reach = near_corner ? D2C_REACH : 2;
  for (int di = -reach; di <= reach; ++di)
    for (int dj = -reach; dj <= reach; ++dj) {
      const int ci = i + di, cj = j + dj;
      if (ci < 0 || ci >= d.ni || cj < 0 || cj >= d.nj) continue;
      auto unit = [&](int ii, int jj) { return (ii == ci && jj == cj) ? R(1) : R(0); };
      const R w = d2c_pass_value<R>(d, t, i, j, nt, cd, del6_u, del6_v, rarea, unit);
      if (w != R(0)) add(idx3(d, t, ci, cj, k), G * w);
    }
}

}  // namespace adj
}  // namespace fv3b

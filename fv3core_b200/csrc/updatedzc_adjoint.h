// Hand-written adjoint (reverse mode) of UpdateGeopotentialHeightOnCGrid
// (updatedzc.py:123-163), written for both the device and the host (the
// tests build it with g++ and compare with torch autograd of a PyTorch-ops
// restatement).  dp_ref, zs and the cell areas are held fixed; gradients
// flow to gz, ut and vt.
//
// The forward, on the points p of [is-1, ie+1] x [js-1, je+1] and every
// interface k:
//   xf0, xf1 = the interface fluxes of ut at i and i+1 (p_weighted over the
//              layers k-2..k+1), yf0, yf1 those of vt at j and j+1;
//   sx0 = gzx(i-1) if xf0 > 0 else gzx(i), sx1 = gzx(i) if xf1 > 0 else
//   gzx(i+1), likewise sy0, sy1 from gzy (gzx, gzy: gz read through the
//   two-cell corner rules);
//   new = (gzy(p) area + xf0 sx0 - xf1 sx1 + yf0 sy0 - yf1 sy1)
//         / (area + xf0 - xf1 + yf0 - yf1);
// then per column, bottom up: gz = new at the surface, ws = (zs - new) / dt
// there, and gz[k] = max(new[k], gz[k+1] + DZ_MIN) above.  Upwind choices
// and the floor are taken as the forward took them.
#pragma once

#include "corners.cuh"

namespace fv3b {
namespace adj {

constexpr double UZC_DZ_MIN = 2.0;

// p_weighted_average_top / _domain / _bottom (updatedzc.py:15-34) as
// weights of the layers k-2, k-1, k, k+1.
template <class R>
__device__ inline void uzc_weights(const R* dp0, int k, int nk, R w[4]) {
  w[0] = w[1] = w[2] = w[3] = R(0);
  if (k == 0) {
    const R ratio = dp0[0] / (dp0[0] + dp0[1]);
    w[2] = R(1) + ratio;
    w[3] = -ratio;
  } else if (k == nk - 1) {
    const R ratio = dp0[k - 1] / (dp0[k - 2] + dp0[k - 1]);
    w[1] = R(1) + ratio;
    w[0] = -ratio;
  } else {
    const R ir = R(1) / (dp0[k - 1] + dp0[k]);
    w[1] = dp0[k] * ir;
    w[2] = dp0[k - 1] * ir;
  }
}

// The interface flux at offset o (level k) of a layer field a.
template <class R>
__device__ inline R uzc_flux(const Dims& d, const R* a, const R w[4], idx_t o, int k) {
  R f = R(0);
  for (int m = 0; m < 4; ++m) {
    const int kk = k - 2 + m;
    if (w[m] != R(0) && kk >= 0 && kk < d.nk) f += w[m] * a[o + (kk - k) * d.sk];
  }
  return f;
}

// Offset of the point gz is read from at (i, j), level k, through the
// two-cell corner rules of the x (xdir) or y sweep.
__device__ inline idx_t uzc_source(const Dims& d, int t, int i, int j, int k, bool xdir) {
  CornerRule r;
  const bool hit = xdir ? corner_x(d, i, j, false, 1.0, 1.0, 1.0, 1.0, r) : corner_y(d, i, j, false, 1.0, 1.0, 1.0, 1.0, r);
  return hit ? idx3(d, t, i + r.di, j + r.dj, k) : idx3(d, t, i, j, k);
}

// The advected height at (t, i, j, k), before the floor.
template <class R>
__device__ inline R uzc_new(const Dims& d, int t, int i, int j, int k, const R* dp0, const R* area, const R* ut,
                            const R* vt, const R* gz) {
  R w[4];
  uzc_weights<R>(dp0, k, d.nk, w);
  const R xf0 = uzc_flux<R>(d, ut, w, idx3(d, t, i, j, k), k), xf1 = uzc_flux<R>(d, ut, w, idx3(d, t, i + 1, j, k), k);
  const R yf0 = uzc_flux<R>(d, vt, w, idx3(d, t, i, j, k), k), yf1 = uzc_flux<R>(d, vt, w, idx3(d, t, i, j + 1, k), k);
  const R sx0 = gz[uzc_source(d, t, xf0 > R(0) ? i - 1 : i, j, k, true)];
  const R sx1 = gz[uzc_source(d, t, xf1 > R(0) ? i : i + 1, j, k, true)];
  const R sy0 = gz[uzc_source(d, t, i, yf0 > R(0) ? j - 1 : j, k, false)];
  const R sy1 = gz[uzc_source(d, t, i, yf1 > R(0) ? j : j + 1, k, false)];
  const R a = area[idx2(d, t, i, j)];
  return (gz[uzc_source(d, t, i, j, k, false)] * a + xf0 * sx0 - xf1 * sx1 + yf0 * sy0 - yf1 * sy1) /
         (a + xf0 - xf1 + yf0 - yf1);
}

// Adds the contributions of the cotangent G of new(t, i, j, k) to the
// cotangents of gz, ut and vt through add(array, offset, value), array 0 =
// gz, 1 = ut, 2 = vt.
template <class R, class Add>
__device__ inline void uzc_point_adjoint(const Dims& d, int t, int i, int j, int k, R G, const R* dp0, const R* area,
                                         const R* ut, const R* vt, const R* gz, Add add) {
  R w[4];
  uzc_weights<R>(dp0, k, d.nk, w);
  const idx_t ox0 = idx3(d, t, i, j, k), ox1 = idx3(d, t, i + 1, j, k), oy1 = idx3(d, t, i, j + 1, k);
  const R xf0 = uzc_flux<R>(d, ut, w, ox0, k), xf1 = uzc_flux<R>(d, ut, w, ox1, k);
  const R yf0 = uzc_flux<R>(d, vt, w, ox0, k), yf1 = uzc_flux<R>(d, vt, w, oy1, k);
  const idx_t qx0 = uzc_source(d, t, xf0 > R(0) ? i - 1 : i, j, k, true);
  const idx_t qx1 = uzc_source(d, t, xf1 > R(0) ? i : i + 1, j, k, true);
  const idx_t qy0 = uzc_source(d, t, i, yf0 > R(0) ? j - 1 : j, k, false);
  const idx_t qy1 = uzc_source(d, t, i, yf1 > R(0) ? j : j + 1, k, false);
  const idx_t qc = uzc_source(d, t, i, j, k, false);
  const R sx0 = gz[qx0], sx1 = gz[qx1], sy0 = gz[qy0], sy1 = gz[qy1];
  const R a = area[idx2(d, t, i, j)];
  const R num = gz[qc] * a + xf0 * sx0 - xf1 * sx1 + yf0 * sy0 - yf1 * sy1;
  const R den = a + xf0 - xf1 + yf0 - yf1;
  const R aN = G / den;
  const R aD = -aN * (num / den);
  add(0, qc, aN * a);
  add(0, qx0, aN * xf0);
  add(0, qx1, -aN * xf1);
  add(0, qy0, aN * yf0);
  add(0, qy1, -aN * yf1);
  const R a_xf0 = aN * sx0 + aD, a_xf1 = -aN * sx1 - aD;
  const R a_yf0 = aN * sy0 + aD, a_yf1 = -aN * sy1 - aD;
  for (int m = 0; m < 4; ++m) {
    const int kk = k - 2 + m;
    if (w[m] == R(0) || kk < 0 || kk >= d.nk) continue;
    const idx_t dk = (kk - k) * d.sk;
    add(1, ox0 + dk, w[m] * a_xf0);
    add(1, ox1 + dk, w[m] * a_xf1);
    add(2, ox0 + dk, w[m] * a_yf0);
    add(2, oy1 + dk, w[m] * a_yf1);
  }
}

// The floor and the surface w of one column, backwards: from the
// cotangents g_out of the new gz (levels 0..nk-1, stride sk) and g_ws of
// ws, the cotangents g_new of the heights before the floor.  new_col holds
// those heights (the forward's values).
template <class R>
__device__ inline void uzc_column_adjoint(int nk, idx_t sk, const R* new_col, const R* g_out, R g_ws, R rdt,
                                          R* g_new) {
  // the forward's choices: floor[k] when gz[k] took gz[k+1] + DZ_MIN
  unsigned long long floor_bits[2] = {0ull, 0ull};
  R below = new_col[(nk - 1) * sk];
  for (int k = nk - 2; k >= 0; --k) {
    const R v = new_col[k * sk];
    const R kp1 = below + R(UZC_DZ_MIN);
    if (!(v > kp1)) floor_bits[k >> 6] |= 1ull << (k & 63);
    below = v > kp1 ? v : kp1;
  }
  R carry = R(0);
  for (int k = 0; k < nk - 1; ++k) {
    const R tot = g_out[k * sk] + carry;
    const bool fl = (floor_bits[k >> 6] >> (k & 63)) & 1ull;
    g_new[k * sk] = fl ? R(0) : tot;
    carry = fl ? tot : R(0);
  }
  g_new[(nk - 1) * sk] = g_out[(nk - 1) * sk] + carry - g_ws * rdt;
}

}  // namespace adj
}  // namespace fv3b

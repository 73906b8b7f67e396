// Hand-written adjoint (reverse mode) of the wind update of
// NonHydrostaticPressureGradient (nh_p_grad.py:21-83, 147-206), written for
// both the device and the host.  The B-grid interpolations that feed it are
// a2b_ord4, whose transpose is in a2b_adjoint.h.
//
// With the B-grid fields pp_b, pk3_b, gz_b and wk1 (= a2b of delp), and at
// level 0 pp = 0 and pk3 = ptop^akap (set_k0_and_calc_wk), the forward sets
// at u points ([is, ie] x [js, je+1], layers 0..npz-1; q = (i+1, j)) and v
// points ([is, ie+1] x [js, je], q = (i, j+1)):
//   X1 = gz_b(p, k+1) - gz_b(q, k),  X2 = gz_b(p, k) - gz_b(q, k+1)
//   du = dt / (wk(p) + wk(q)) * (X1 (pk3(q, k+1) - pk3(p, k)) + X2 (pk3(p, k+1) - pk3(q, k)))
//   dp = dt / (wk1(p) + wk1(q)) * (X1 (pp(q, k+1) - pp(p, k)) + X2 (pp(p, k+1) - pp(q, k)))
//   u  = (u + du + dp) * rdx (v: rdy)
// with wk = pk3(k+1) - pk3(k).
#pragma once

#include "dims.h"

namespace fv3b {
namespace adj {

// Adds the contributions of the cotangent G of the new wind at (t, i, j,
// k), direction dir (0 = u, 1 = v), through add(a, o, v): a = 0 pp_b,
// 1 pk3_b, 2 gz_b, 3 wk1, 4 the old wind.  Level-0 values of pp and pk3 are
// constants and take nothing.
template <class R, class Add>
__device__ inline void nhp_wind_adjoint(const Dims& d, int t, int i, int j, int k, int dir, R G, R dt, R ptk,
                                        const R* rd, const R* pp_b, const R* pk3_b, const R* gz_b, const R* wk1,
                                        Add add) {
  const idx_t sk = d.sk;
  const idx_t o = idx3(d, t, i, j, k), on = o + (dir == 0 ? 1 : d.sj);
  auto P = [&](idx_t x, int dk) { return k + dk == 0 ? R(0) : pp_b[x + dk * sk]; };
  auto K3 = [&](idx_t x, int dk) { return k + dk == 0 ? ptk : pk3_b[x + dk * sk]; };
  const R X1 = gz_b[o + sk] - gz_b[on], X2 = gz_b[o] - gz_b[on + sk];
  const R Yk1 = K3(on, 1) - K3(o, 0), Yk2 = K3(o, 1) - K3(on, 0);
  const R Dk = (K3(o, 1) - K3(o, 0)) + (K3(on, 1) - K3(on, 0));
  const R cdu = dt / Dk;
  const R du = cdu * (X1 * Yk1 + X2 * Yk2);
  const R D1 = wk1[o] + wk1[on];
  const R cdp = dt / D1;
  const R Yp1 = P(on, 1) - P(o, 0), Yp2 = P(o, 1) - P(on, 0);
  const R dp = cdp * (X1 * Yp1 + X2 * Yp2);
  const R Gr = G * rd[idx2(d, t, i, j)];
  add(4, o, Gr);
  const R aX1 = Gr * (cdu * Yk1 + cdp * Yp1), aX2 = Gr * (cdu * Yk2 + cdp * Yp2);
  add(2, o + sk, aX1);
  add(2, on, -aX1);
  add(2, o, aX2);
  add(2, on + sk, -aX2);
  const R aYk1 = Gr * cdu * X1, aYk2 = Gr * cdu * X2, aDk = -Gr * du / Dk;
  const R aYp1 = Gr * cdp * X1, aYp2 = Gr * cdp * X2, aD1 = -Gr * dp / D1;
  // pk3: through Yk1, Yk2 and both wk
  add(1, o + sk, aYk2 + aDk);
  add(1, on + sk, aYk1 + aDk);
  if (k > 0) {
    add(1, o, -aYk1 - aDk);
    add(1, on, -aYk2 - aDk);
  }
  add(0, on + sk, aYp1);
  add(0, o + sk, aYp2);
  if (k > 0) {
    add(0, o, -aYp1);
    add(0, on, -aYp2);
  }
  add(3, o, aD1);
  add(3, on, aD1);
}

}  // namespace adj
}  // namespace fv3b

// Hand-written adjoint of RayleighDamping's wind damping
// (ray_fast.py:48-128, 169-192), for one column, device and host.  The
// forward is linear in the winds: on the damped levels k < k_rf,
// q[k] -> rf[k] q[k], and the momentum removed there,
// total = sum (1 - rf[k]) dp[k] q[k], is given back as total / dm[k] on the
// levels k < k_nudge.  Its adjoint, in place on the cotangent g of the new
// wind: s = sum_{k < k_nudge} g[k] / dm[k], then on the damped levels
// g[k] -> rf[k] g[k] + (1 - rf[k]) dp[k] s.  w is only scaled by rf.
#pragma once

#include "dims.h"

namespace fv3b {
namespace adj {

template <class R>
__device__ inline void ray_column_adjoint(int k_rf, int k_nudge, idx_t sk, const R* rf, const R* dm, const R* dp,
                                          R* g) {
  double s = 0.0;
  for (int k = 0; k < k_nudge; ++k) s += (double)g[k * sk] / (double)dm[k];
  for (int k = 0; k < k_rf; ++k) {
    const double back = (1.0 - (double)rf[k]) * (double)dp[k] * s;
    g[k * sk] = static_cast<R>((double)g[k * sk] * (double)rf[k] + back);
  }
}

template <class R>
__device__ inline void ray_w_column_adjoint(int k_rf, idx_t sk, const R* rf, R* g) {
  for (int k = 0; k < k_rf; ++k) g[k * sk] = g[k * sk] * rf[k];
}

}  // namespace adj
}  // namespace fv3b

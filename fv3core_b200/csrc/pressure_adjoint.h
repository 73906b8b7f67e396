// Hand-written adjoints of the two column sums on halo rings: edge_pe
// (pe_halo.py:6-33; pe[k] = ptop + sum of delp above k on the one-cell
// ring) and PK3Halo (pk3_halo.py:36-68; pk3[k] = pe[k]^akap on the two-cell
// ring, levels 1..npz).  One column each; written for the device and the
// host.  The cotangent of the new field is turned, in place, into that of
// the old one (zero where the stage overwrote it); g_delp is overwritten.
#pragma once

#include <math.h>

#include "dims.h"

namespace fv3b {
namespace adj {

template <class R>
__device__ inline void edge_pe_column_adjoint(int nk, idx_t sk, R* g_pe, R* g_delp) {
  // delp[m] enters every pe[k] with k > m
  double acc = 0.0;
  g_delp[(nk - 1) * sk] = R(0);
  for (int m = nk - 2; m >= 0; --m) {
    acc += (double)g_pe[(m + 1) * sk];
    g_delp[m * sk] = static_cast<R>(acc);
  }
  for (int k = 0; k < nk; ++k) g_pe[k * sk] = R(0);
}

template <class R>
__device__ inline void pk3_column_adjoint(int nk, idx_t sk, double ptop, double akap, const R* delp, R* g_pk3,
                                          R* g_delp) {
  // pe at every interface, as the forward sums it
  double pe[128];
  pe[0] = ptop;
  for (int k = 1; k < nk; ++k) pe[k] = pe[k - 1] + (double)delp[(k - 1) * sk];
  double acc = 0.0;
  g_delp[(nk - 1) * sk] = R(0);
  for (int m = nk - 2; m >= 0; --m) {
    const int k = m + 1;
    acc += (double)g_pk3[k * sk] * akap * pow(pe[k], akap - 1.0);
    g_delp[m * sk] = static_cast<R>(acc);
  }
  // level 0 of pk3 is not written by the stage: its cotangent passes through
  for (int k = 1; k < nk; ++k) g_pk3[k * sk] = R(0);
}

}  // namespace adj
}  // namespace fv3b

// Hand-written adjoint of compute_pkz_tempadjust (temperature_adjust.py:
// 8-44) at one point; device and host.  The forward:
//   X = rdg dp / dz pt,  pkz = X^c (c = cappa / (1 - cappa)),
//   dtmp = heat / (cv dp),  delt = dtmp unless lim < |dtmp|, then +-lim,
//   pt' = pt + delt / pkz.
// Cotangents Gt of pt' and Gk of pkz' give those of dp, dz, pt and heat
// (cappa held fixed; the clipping branch is the forward's).
#pragma once

#include <math.h>

#include "dims.h"

namespace fv3b {
namespace adj {

template <class R>
__device__ inline void tempadjust_point_adjoint(R dp, R dz, R pt, R heat, R cappa, R lim, R rdg, R cv, R Gt, R Gk,
                                                R& a_dp, R& a_dz, R& a_pt, R& a_heat) {
  const double c = (double)cappa / (1.0 - (double)cappa);
  const double X = (double)rdg * dp / dz * pt;
  const double p = pow(X, c);
  const double dtmp = (double)heat / ((double)cv * dp);
  const bool clipped = (double)lim < fabs(dtmp);
  const double delt = clipped ? (dtmp > 0.0 ? (double)lim : -(double)lim) : dtmp;
  const double a_p = Gk - Gt * delt / (p * p);
  const double a_delt = clipped ? 0.0 : Gt / p;
  const double a_X = a_p * c * p / X;
  a_pt = static_cast<R>(Gt + a_X * rdg * dp / dz);
  a_dp = static_cast<R>(a_X * rdg * pt / dz - a_delt * dtmp / dp);
  a_dz = static_cast<R>(-a_X * X / dz);
  a_heat = static_cast<R>(a_delt / (cv * (double)dp));
}

}  // namespace adj
}  // namespace fv3b

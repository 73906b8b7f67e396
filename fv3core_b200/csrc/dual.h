// Forward-mode dual numbers for the adjoints of small nonlinear stencils;
// device and host.  A stage's point function written once over a scalar
// type T gives, evaluated with Dual<R> inputs seeded at one input point, the
// exact derivative of its output with respect to that input; the point's
// adjoint then scatters its cotangent times each such derivative (the
// scheme the linear transposes use with unit inputs, extended to nonlinear
// point functions).  Branches follow the values, as the forward took them.
#pragma once

#include <math.h>

#include "dims.h"
#include "fmath.h"

namespace fv3b {
namespace adj {

template <class R>
struct Dual {
  R v, d;
  __host__ __device__ Dual() : v(R(0)), d(R(0)) {}
  // constants promote to duals with no derivative
  __host__ __device__ Dual(R value) : v(value), d(R(0)) {}
  __host__ __device__ Dual(R value, R deriv) : v(value), d(deriv) {}
};

template <class R>
__host__ __device__ inline Dual<R> operator+(Dual<R> a, Dual<R> b) { return {a.v + b.v, a.d + b.d}; }
template <class R>
__host__ __device__ inline Dual<R> operator-(Dual<R> a, Dual<R> b) { return {a.v - b.v, a.d - b.d}; }
template <class R>
__host__ __device__ inline Dual<R> operator-(Dual<R> a) { return {-a.v, -a.d}; }
template <class R>
__host__ __device__ inline Dual<R> operator*(Dual<R> a, Dual<R> b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
template <class R>
__host__ __device__ inline Dual<R> operator/(Dual<R> a, Dual<R> b) {
  const R q = a.v / b.v;
  return {q, (a.d - q * b.d) / b.v};
}
template <class R>
__host__ __device__ inline Dual<R> operator+(Dual<R> a, R b) { return {a.v + b, a.d}; }
template <class R>
__host__ __device__ inline Dual<R> operator+(R a, Dual<R> b) { return {a + b.v, b.d}; }
template <class R>
__host__ __device__ inline Dual<R> operator-(Dual<R> a, R b) { return {a.v - b, a.d}; }
template <class R>
__host__ __device__ inline Dual<R> operator-(R a, Dual<R> b) { return {a - b.v, -b.d}; }
template <class R>
__host__ __device__ inline Dual<R> operator*(Dual<R> a, R b) { return {a.v * b, a.d * b}; }
template <class R>
__host__ __device__ inline Dual<R> operator*(R a, Dual<R> b) { return {a * b.v, a * b.d}; }
template <class R>
__host__ __device__ inline Dual<R> operator/(Dual<R> a, R b) { return {a.v / b, a.d / b}; }
template <class R>
__host__ __device__ inline Dual<R> operator/(R a, Dual<R> b) {
  const R q = a / b.v;
  return {q, -q * b.d / b.v};
}
template <class R>
__host__ __device__ inline bool operator>(Dual<R> a, Dual<R> b) { return a.v > b.v; }
template <class R>
__host__ __device__ inline bool operator<(Dual<R> a, Dual<R> b) { return a.v < b.v; }
template <class R>
__host__ __device__ inline bool operator>(Dual<R> a, R b) { return a.v > b; }
template <class R>
__host__ __device__ inline bool operator<(Dual<R> a, R b) { return a.v < b; }

template <class R>
__host__ __device__ inline Dual<R> dabs(Dual<R> a) { return a.v < R(0) ? -a : a; }
// exp, log and pow are the library's own (fmath.h), the functions the
// forward kernels evaluate, so value-driven branches and derivatives are
// taken at the forward's values
template <class R>
__host__ __device__ inline Dual<R> dexp(Dual<R> a) {
  const R e = static_cast<R>(fm::fm_exp(static_cast<double>(a.v)));
  return {e, e * a.d};
}
template <class R>
__host__ __device__ inline Dual<R> dlog(Dual<R> a) {
  return {static_cast<R>(fm::fm_log(static_cast<double>(a.v))), a.d / a.v};
}
// a^b for a constant exponent b
template <class R>
__host__ __device__ inline Dual<R> dpow(Dual<R> a, R b) {
  const R p = static_cast<R>(fm::fm_pow(static_cast<double>(a.v), static_cast<double>(b)));
  return {p, b * p / a.v * a.d};
}

// The derivative of a point function f(seeded) -> Dual<R> with respect to
// one input: seeded(x) is an accessor factory that marks the input x.
// Adds, for every candidate input c of the point (cands(n, c) enumerates
// them, returning false past the last), G * d out / d c through add(c, v).
template <class R, class F, class Cands, class Add>
__host__ __device__ inline void dual_point_adjoint(const F& f, const Cands& cands, R G, Add add) {
  if (G == R(0)) return;
  idx_t c;
  for (int n = 0; cands(n, c); ++n) {
    const Dual<R> out = f(c);
    if (out.d != R(0)) add(c, G * out.d);
  }
}

}  // namespace adj
}  // namespace fv3b

// exp, log and pow for the FP64 kernels, written from the mathematics so
// that the same source compiles for the device and for the host (the
// oracle's C helper includes this header).  Built without implicit a*b+c
// contraction on both sides (nvcc --fmad=false, gcc -ffp-contract=off) and
// with every fused multiply-add written out as fma() (exactly rounded in
// IEEE 754 on both the GPU and the host), the host and device results are
// bit-identical.  That lets the kernels be checked against the oracle to
// the last bit even where the substep amplifies last-place differences of
// these functions (the Riemann solvers subtract the hydrostatic pressure
// from exp(...) of the full pressure).
//
// Methods:
//   exp: Cody-Waite reduction x = k ln2 + r (ln2 split into a 32-bit head
//        and a tail, both derived from ln2 to 60 digits), |r| <= ln2/2, r
//        kept as a double-double; Taylor polynomial of degree 13 with the
//        leading terms 1 + r + r^2 q summed in double-double; exact scaling
//        by 2^k.
//   log: x = 2^e m with m in [sqrt(1/2), sqrt(2)), f = m - 1,
//        s = f / (2 + f), log(1 + f) = 2 atanh(s) written as
//        f - f^2/2 + s (f^2/2 + R), R = sum_k 2 s^(2k) / (2k + 1), k <= 11
//        (the identity f - 2s = s f gives this form); e ln2 + f - f^2/2
//        summed in double-double.
//   pow: exp(y log x) with log x and y log x in double-double.
// Double-double steps use Knuth's TwoSum and the fma-based exact product.
// Accuracy (tested on the host against correctly rounded values): all
// three within 1 ulp, correctly rounded in all but a small fraction of
// cases on the ranges the substep uses.
#pragma once

#include <stdint.h>
#include <string.h>

#ifndef __CUDACC__
#include <math.h>
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif
#ifndef __forceinline__
#define __forceinline__ inline
#endif
#endif

namespace fv3b {
namespace fm {

constexpr double LN2_HI = 0x1.62e42ff000000p-1;   // ln2 rounded to 32 bits
constexpr double LN2_LO = -0x1.718432a1b0e26p-35;  // ln2 - LN2_HI
constexpr double LOG2E = 0x1.71547652b82fep+0;
constexpr double SQRT2 = 0x1.6a09e667f3bcdp+0;

__host__ __device__ __forceinline__ uint64_t bits_of(double x) {
  uint64_t u;
  memcpy(&u, &x, sizeof u);
  return u;
}
__host__ __device__ __forceinline__ double from_bits(uint64_t u) {
  double x;
  memcpy(&x, &u, sizeof x);
  return x;
}
// 2^k for -1022 <= k <= 1023
__host__ __device__ __forceinline__ double pow2i(int k) { return from_bits((uint64_t)(k + 1023) << 52); }

__host__ __device__ __forceinline__ double round_half_even(double x) {
#ifdef __CUDA_ARCH__
  return rint(x);
#else
  return nearbyint(x);
#endif
}

// Error-free transformations: a + b = s + e (Knuth's TwoSum) and
// a * b = p + e (the exact product from one fused multiply-add).
__host__ __device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}
__host__ __device__ __forceinline__ void two_prod(double a, double b, double& p, double& e) {
  p = a * b;
  e = fma(a, b, -p);
}

// exp(rh + rl) for |rh| <= ln2/2 + tiny, |rl| << ulp(rh):
// 1 + r + r^2/2 + r^3 q(r), q the Taylor tail 1/3! + r/4! + ... + r^10/13!;
// 1 + r + r^2/2 is summed in double-double (r^2 from the exact product), so
// the only rounding of size ~ulp left is the last one.
__host__ __device__ __forceinline__ double exp_reduced(double rh, double rl) {
  double q = 1.0 / 6227020800.0;
  q = fma(q, rh, 1.0 / 479001600.0);
  q = fma(q, rh, 1.0 / 39916800.0);
  q = fma(q, rh, 1.0 / 3628800.0);
  q = fma(q, rh, 1.0 / 362880.0);
  q = fma(q, rh, 1.0 / 40320.0);
  q = fma(q, rh, 1.0 / 5040.0);
  q = fma(q, rh, 1.0 / 720.0);
  q = fma(q, rh, 1.0 / 120.0);
  q = fma(q, rh, 1.0 / 24.0);
  q = fma(q, rh, 1.0 / 6.0);
  double r2h, r2l;
  two_prod(rh, rh, r2h, r2l);
  const double small = fma(r2h * rh, q, fma(rl, 1.0 + rh, 0.5 * r2l));  // + exp'(r) rl
  double s1, e1, sh, sl;
  two_sum(rh, 0.5 * r2h, s1, e1);
  two_sum(s1, e1 + small, sh, sl);
  double h, l;
  two_sum(1.0, sh, h, l);
  return h + (l + sl);
}

__host__ __device__ __forceinline__ double scale2(double p, int k) {
  if (k > 1023) return p * pow2i(1023) * pow2i(k - 1023);
  if (k < -1022) return p * pow2i(-1022) * pow2i(k + 1022);
  return p * pow2i(k);
}

// exp(xh + xl), |xl| <= ulp(xh)
__host__ __device__ __forceinline__ double exp_dd(double xh, double xl) {
  if (xh != xh) return xh;
  if (xh > 709.782712893384) return from_bits(0x7ff0000000000000ull);
  if (xh < -745.1332191019412) return 0.0;
  const double kd = round_half_even(xh * LOG2E);
  const int k = (int)kd;
  const double t = xh - kd * LN2_HI;  // exact: kd * LN2_HI has <= 43 bits and is close to xh
  const double c = fma(kd, LN2_LO, -xl);
  double rh = t - c;
  double rl = (t - rh) - c;
  return scale2(exp_reduced(rh, rl), k);
}

// The mixed-precision library is compiled with FV3B_FAST_TRANSCENDENTALS:
// it has no last-bit parity target, so its device code calls CUDA's FP64
// exp, log and pow, which take a fraction of the instructions of the
// double-double forms below.
#if defined(FV3B_FAST_TRANSCENDENTALS) && defined(__CUDA_ARCH__)
#define FV3B_FM_FAST 1
#else
#define FV3B_FM_FAST 0
#endif

__host__ __device__ __forceinline__ double fm_exp(double x) {
#if FV3B_FM_FAST
  return ::exp(x);
#else
  return exp_dd(x, 0.0);
#endif
}

// log(x) as hi + lo (x positive, finite, normal or subnormal)
__host__ __device__ __forceinline__ void log_dd(double x, double& hi, double& lo) {
  uint64_t u = bits_of(x);
  int e = (int)((u >> 52) & 0x7ff);
  if (e == 0) {  // subnormal: scale into the normal range
    x = x * 0x1p54;
    u = bits_of(x);
    e = (int)((u >> 52) & 0x7ff) - 54;
  }
  e -= 1023;
  double m = from_bits((u & 0x000fffffffffffffull) | 0x3ff0000000000000ull);  // [1, 2)
  if (m > SQRT2) {
    m = m * 0.5;
    e += 1;
  }
  const double f = m - 1.0;  // exact (Sterbenz)
  const double s = f / (2.0 + f);
  const double z = s * s;
  // R = sum_{k=1..11} 2 z^k / (2k + 1)
  double R = 2.0 / 23.0;
  R = fma(R, z, 2.0 / 21.0);
  R = fma(R, z, 2.0 / 19.0);
  R = fma(R, z, 2.0 / 17.0);
  R = fma(R, z, 2.0 / 15.0);
  R = fma(R, z, 2.0 / 13.0);
  R = fma(R, z, 2.0 / 11.0);
  R = fma(R, z, 2.0 / 9.0);
  R = fma(R, z, 2.0 / 7.0);
  R = fma(R, z, 2.0 / 5.0);
  R = fma(R, z, 2.0 / 3.0);
  R = R * z;
  // log x = e ln2 + f - f^2/2 + s (f^2/2 + R); e*LN2_HI, f and f^2/2 (from
  // the exact square) are carried without rounding, the small rest rounded
  double sqh, sql;
  two_prod(f, f, sqh, sql);
  const double hfh = 0.5 * sqh, hfl = 0.5 * sql;  // exact halving
  const double dk = (double)e;
  const double small = fma(s, hfh + R, fma(dk, LN2_LO, -hfl));
  double a, ae, b, be;
  two_sum(dk * LN2_HI, f, a, ae);
  two_sum(a, -hfh, b, be);
  double l = ae + be + small;
  two_sum(b, l, hi, lo);
}

__host__ __device__ __forceinline__ double fm_log(double x) {
#if FV3B_FM_FAST
  return ::log(x);
#endif
  if (x != x) return x;
  if (x < 0.0) return from_bits(0x7ff8000000000000ull);
  if (x == 0.0) return -from_bits(0x7ff0000000000000ull);
  if (x == from_bits(0x7ff0000000000000ull)) return x;
  double hi, lo;
  log_dd(x, hi, lo);
  return hi + lo;
}

// x^y = exp(y log x) with log x and the product carried in double-double
// (x > 0; x == 0 gives 0 for y > 0, 1 for y == 0, inf for y < 0; x < 0 NaN)
__host__ __device__ __forceinline__ double fm_pow(double x, double y) {
#if FV3B_FM_FAST
  return ::pow(x, y);
#endif
  if (x != x || y != y) return x + y;
  if (x == 0.0) return y > 0.0 ? 0.0 : (y == 0.0 ? 1.0 : from_bits(0x7ff0000000000000ull));
  if (x < 0.0) return from_bits(0x7ff8000000000000ull);
  if (x == from_bits(0x7ff0000000000000ull)) return y > 0.0 ? x : (y == 0.0 ? 1.0 : 0.0);
  double lh, ll;
  log_dd(x, lh, ll);
  double ph, pl;
  two_prod(y, lh, ph, pl);
  pl = fma(y, ll, pl);
  double zh, zl;
  two_sum(ph, pl, zh, zl);
  return exp_dd(zh, zl);
}

}  // namespace fm
}  // namespace fv3b

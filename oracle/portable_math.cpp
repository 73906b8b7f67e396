// Host build of the kernels' exp / log / pow (fv3core_b200/csrc/fmath.h)
// for the oracle's "device math" mode -- TEST INFRASTRUCTURE ONLY.
// Compiled by oracle/_math.py with g++ -O2 -ffp-contract=off.
#include "../fv3core_b200/csrc/fmath.h"

extern "C" {
void pm_exp(const double* x, double* y, long n) {
  for (long i = 0; i < n; ++i) y[i] = fv3b::fm::fm_exp(x[i]);
}
void pm_log(const double* x, double* y, long n) {
  for (long i = 0; i < n; ++i) y[i] = fv3b::fm::fm_log(x[i]);
}
void pm_pow(const double* x, const double* p, double* y, long n) {
  for (long i = 0; i < n; ++i) y[i] = fv3b::fm::fm_pow(x[i], p[i]);
}
}

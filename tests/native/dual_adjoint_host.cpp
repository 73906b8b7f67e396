// Host check of the dual-number adjoint scheme (fv3core_b200/csrc/dual.h):
// p_grad_c's increments written once over a scalar type and differentiated
// with duals, for comparison with the hand-written adjoint
// (fv3core_b200/csrc/pgrad_adjoint.h).  Fields in the device layout.
#include "../../fv3core_b200/csrc/dual.h"

namespace {
using fv3b::idx_t;
using D = fv3b::adj::Dual<double>;

// the increment of p_grad_c at offset o with neighbour o - off, over T
template <class T, class A>
T pgc_increment(const A& at, idx_t o, idx_t off, idx_t sk, double dt2, double rdc) {
  const idx_t q = o - off;
  const T Dn = at(0, q) + at(0, o);
  const T a = at(2, q + sk) - at(2, o), b = at(1, o + sk) - at(1, q);
  const T cc = at(2, q) - at(2, o + sk), e = at(1, q + sk) - at(1, o);
  return dt2 * rdc / Dn * (a * b + cc * e);
}
}  // namespace

// the gradients of <gu, uc_new> + <gv, vc_new> with respect to delpc, pkc
// and gz (same arguments as pgc_adjoint_host); the outputs are accumulated
extern "C" void pgc_dual_adjoint_host(int n, int halo, int npz, double dt2, const double* rdxc, const double* rdyc,
                                      const double* delpc, const double* pkc, const double* gz, const double* gu,
                                      const double* gv, double* g_delpc, double* g_pkc, double* g_gz) {
  fv3b_grid_dims g{n, halo, npz, 0};
  const fv3b::Dims d = fv3b::make_dims(&g);
  const double* arr[3] = {delpc, pkc, gz};
  double* out[3] = {g_delpc, g_pkc, g_gz};
  const idx_t S = (idx_t)6 * d.st;  // candidate c = array * S + offset
  for (int t = 0; t < 6; ++t)
    for (int k = 0; k < d.nz; ++k)
      for (int j = d.jsc; j <= d.jec + 1; ++j)
        for (int i = d.isc; i <= d.iec + 1; ++i)
          for (int face = 0; face < 2; ++face) {
            const idx_t o = fv3b::idx3(d, t, i, j, k), off = face == 0 ? 1 : d.sj, q = o - off;
            const double rdc = (face == 0 ? rdxc : rdyc)[fv3b::idx2(d, t, i, j)];
            const double G = (face == 0 ? gu : gv)[o];
            const idx_t cand[10] = {q, o, S + o + d.sk, S + q, S + q + d.sk, S + o,
                                    2 * S + q + d.sk, 2 * S + o, 2 * S + q, 2 * S + o + d.sk};
            auto cands = [&](int m, idx_t& c) {
              if (m >= 10) return false;
              c = cand[m];
              return true;
            };
            auto f = [&](idx_t c) {
              auto at = [&](int a, idx_t x) { return D(arr[a][x], a * S + x == c ? 1.0 : 0.0); };
              return pgc_increment<D>(at, o, off, d.sk, dt2, rdc);
            };
            auto add = [&](idx_t c, double v) { out[c / S][c % S] += v; };
            fv3b::adj::dual_point_adjoint<double>(f, cands, G, add);
          }
}

// The scheme on a branchy stage: UpdateGeopotentialHeightOnCGrid's
// advected height (upwind choices, corner copies) over T, differentiated
// with duals; for comparison with the scatter of uzc_point_adjoint
// (fv3core_b200/csrc/updatedzc_adjoint.h).  g_new: the cotangents of the
// heights before the floor; the results are accumulated into g_gz, g_ut,
// g_vt.
#include "../../fv3core_b200/csrc/updatedzc_adjoint.h"

namespace {
template <class T, class A>
T uzc_value(const fv3b::Dims& d, int t, int i, int j, int k, const double* dp0, const double* area, const A& at) {
  double w[4];
  fv3b::adj::uzc_weights<double>(dp0, k, d.nk, w);
  auto flux = [&](int a, int ii, int jj) {
    T f(0.0);
    for (int m = 0; m < 4; ++m) {
      const int kk = k - 2 + m;
      if (w[m] != 0.0 && kk >= 0 && kk < d.nk) f = f + w[m] * at(a, fv3b::idx3(d, t, ii, jj, kk));
    }
    return f;
  };
  const T xf0 = flux(1, i, j), xf1 = flux(1, i + 1, j), yf0 = flux(2, i, j), yf1 = flux(2, i, j + 1);
  auto gzs = [&](int ii, int jj, bool xdir) { return at(0, fv3b::adj::uzc_source(d, t, ii, jj, k, xdir)); };
  const T sx0 = gzs(xf0 > 0.0 ? i - 1 : i, j, true), sx1 = gzs(xf1 > 0.0 ? i : i + 1, j, true);
  const T sy0 = gzs(i, yf0 > 0.0 ? j - 1 : j, false), sy1 = gzs(i, yf1 > 0.0 ? j : j + 1, false);
  const double a = area[fv3b::idx2(d, t, i, j)];
  return (gzs(i, j, false) * a + xf0 * sx0 - xf1 * sx1 + yf0 * sy0 - yf1 * sy1) / (a + xf0 - xf1 + yf0 - yf1);
}
}  // namespace

extern "C" void uzc_dual_scatter_host(int n, int halo, int npz, const double* dp0, const double* area,
                                      const double* ut, const double* vt, const double* gz, const double* g_new,
                                      double* g_gz, double* g_ut, double* g_vt) {
  fv3b_grid_dims g{n, halo, npz, 0};
  const fv3b::Dims d = fv3b::make_dims(&g);
  const double* arr[3] = {gz, ut, vt};
  double* out[3] = {g_gz, g_ut, g_vt};
  const idx_t S = (idx_t)6 * d.st;
  for (int t = 0; t < 6; ++t)
    for (int k = 0; k < d.nk; ++k)
      for (int j = d.jsc - 1; j <= d.jec + 1; ++j)
        for (int i = d.isc - 1; i <= d.iec + 1; ++i) {
          // candidates, the stencil's read set: gz within two points of the
          // point's own level (corner copies included), the fluxes' four
          // layers at i, i+1 (ut) and j, j+1 (vt)
          auto cands = [&](int m, idx_t& c) {
            if (m < 25) {
              c = fv3b::idx3(d, t, i - 2 + m % 5, j - 2 + m / 5, k);
              return true;
            }
            m -= 25;
            if (m >= 16) return false;
            const int a = 1 + m / 8, side = (m / 4) % 2, kk = k - 2 + m % 4;
            if (kk < 0 || kk >= d.nk) {
              c = -1;
              return true;
            }
            c = a * S + fv3b::idx3(d, t, a == 1 ? i + side : i, a == 2 ? j + side : j, kk);
            return true;
          };
          auto f = [&](idx_t c) {
            if (c < 0) return D(0.0);
            auto at = [&](int a, idx_t x) { return D(arr[a][x], a * S + x == c ? 1.0 : 0.0); };
            return uzc_value<D>(d, t, i, j, k, dp0, area, at);
          };
          auto add = [&](idx_t c, double v) { out[c / S][c % S] += v; };
          fv3b::adj::dual_point_adjoint<double>(f, cands, g_new[fv3b::idx3(d, t, i, j, k)], add);
        }
}

// A nonlinear column function with the transcendentals the column solvers
// use: f(x) = pow(exp(0.3 log x) + x, 1.7) / log(1 + x), value and
// derivative by duals at x[m], for a comparison with finite differences of
// the same fmath functions.
extern "C" void dual_transcendental_host(int n, const double* x, double* value, double* deriv) {
  using fv3b::adj::dexp;
  using fv3b::adj::dlog;
  using fv3b::adj::dpow;
  for (int m = 0; m < n; ++m) {
    const D a(x[m], 1.0);
    const D f = dpow(dexp(dlog(a) * D(0.3)) + a, 1.7) / dlog(a + D(1.0));
    value[m] = f.v;
    deriv[m] = f.d;
  }
}

// The same function on plain doubles with the fmath functions.
extern "C" void plain_transcendental_host(int n, const double* x, double* value) {
  using namespace fv3b::fm;
  for (int m = 0; m < n; ++m)
    value[m] = fm_pow(fm_exp(fm_log(x[m]) * 0.3) + x[m], 1.7) / fm_log(x[m] + 1.0);
}

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

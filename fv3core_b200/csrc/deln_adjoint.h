// The transpose of DelnFluxNoSG (delnflux.py:1156-1207), the del-n
// diffusive fluxes of d_sw's and updatedzd's damping, for the adjoints of
// those stages; host build checked by the dot-product identity against the
// oracle's forward.  The operator is linear in q: pass 0 differences
// d2 = damp q (q for mass-weighted fluxes) into fluxes, each later pass
// differences d2 = (fx - fx(+1, 0) + fy - fy(0, +1)) rarea of the previous
// fluxes into fluxes of the opposite sign, and every pass writes only its
// own region (its lo rows beyond the final faces; levels with nord = 0 take
// pass 0 alone, on the compute-domain faces).  Reads of d2 at the points of
// a cube-corner block map to their copy sources (copy_corners_x/y_nord),
// on levels with nord > 0.  The transpose runs the passes backwards,
// scattering each flux cotangent to the two d2 values it differences and
// each d2 cotangent to the four fluxes it sums.
//
// One level of one tile at a time; 2-D arrays are indexed i * si + j * sj
// (the caller's layout), of the tile's full storage extent.
#pragma once

#include "corners.cuh"

namespace fv3b {
namespace adj {

// Cotangent of q (added into gq) from the cotangents gfx, gfy of the final
// fluxes on their region.  nk_ is the level's nord (0 or nmax), damp its
// coefficient, rscale the range scale of the later passes (1 in FP64).
// wx, wy, wd are work planes of the full extent.
template <class R>
__host__ __device__ inline void delnflux_nosg_adjoint_level(const Dims& d, int nmax, int nk_, R damp, R rscale,
                                                            bool mass_weighted, const R* del6_u, const R* del6_v,
                                                            const R* rarea, int si, int sj, const R* gfx,
                                                            const R* gfy, R* gq, R* wx, R* wy, R* wd) {
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec, ni = d.ni, nj = d.nj;
  auto at = [&](int i, int j) { return i * si + j * sj; };
  const int P = nk_ > 0 ? nmax : 0;
  for (int i = 0; i < ni; ++i)
    for (int j = 0; j < nj; ++j) {
      wx[at(i, j)] = gfx[at(i, j)];
      wy[at(i, j)] = gfy[at(i, j)];
    }
  for (int p = P; p >= 0; --p) {
    const int lo = P - p;
    const R sign = p == 0 ? R(1) : R(-1);
    for (int i = 0; i < ni; ++i)
      for (int j = 0; j < nj; ++j) wd[at(i, j)] = R(0);
    for (int i = 0; i < ni; ++i)
      for (int j = 0; j < nj; ++j) {
        const bool corners = nk_ > 0 && (i <= s || i >= e + 1) && (j <= js || j >= je + 1);
        const bool fx_in = i >= s - lo && i < e + 2 + lo && j >= js - lo && j < je + 1 + lo;
        const bool fy_in = i >= s - lo && i < e + 1 + lo && j >= js - lo && j < je + 2 + lo;
        int si2, sj2;
        if (fx_in && wx[at(i, j)] != R(0)) {
          const R G = sign * wx[at(i, j)] * del6_v[at(i, j)];
          int ai = i - 1, aj = j, bi = i, bj = j;
          if (corners && copy_corner_x(d, ai, aj, si2, sj2)) ai = si2, aj = sj2;
          if (corners && copy_corner_x(d, bi, bj, si2, sj2)) bi = si2, bj = sj2;
          wd[at(ai, aj)] += G;
          wd[at(bi, bj)] -= G;
        }
        if (fy_in && wy[at(i, j)] != R(0)) {
          const R G = sign * wy[at(i, j)] * del6_u[at(i, j)];
          int ai = i, aj = j - 1, bi = i, bj = j;
          if (corners && copy_corner_y(d, ai, aj, si2, sj2)) ai = si2, aj = sj2;
          if (corners && copy_corner_y(d, bi, bj, si2, sj2)) bi = si2, bj = sj2;
          wd[at(ai, aj)] += G;
          wd[at(bi, bj)] -= G;
        }
      }
    if (p == 0) {
      for (int i = 0; i < ni; ++i)
        for (int j = 0; j < nj; ++j) gq[at(i, j)] += (mass_weighted ? R(1) : damp) * wd[at(i, j)];
      break;
    }
    // d2 of pass p from the fluxes of pass p - 1
    for (int i = 0; i < ni; ++i)
      for (int j = 0; j < nj; ++j) {
        wx[at(i, j)] = R(0);
        wy[at(i, j)] = R(0);
      }
    for (int i = 0; i + 1 < ni; ++i)
      for (int j = 0; j + 1 < nj; ++j) {
        const R v = wd[at(i, j)];
        if (v == R(0)) continue;
        const R g = v * rarea[at(i, j)] * rscale;
        wx[at(i, j)] += g;
        wx[at(i + 1, j)] -= g;
        wy[at(i, j)] += g;
        wy[at(i, j + 1)] -= g;
      }
  }
}

}  // namespace adj
}  // namespace fv3b

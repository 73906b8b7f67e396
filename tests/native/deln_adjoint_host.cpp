// Host build of the DelnFluxNoSG transpose (fv3core_b200/csrc/deln_adjoint.h)
// for one tile, arrays in the numpy layout of the oracle: 2-D [i][j], 3-D
// [i][j][k].
#include <vector>

#include "../../fv3core_b200/csrc/deln_adjoint.h"

extern "C" void deln_nosg_adjoint_host(int n, int h, int nk, int nmax, const double* nord_bands, const double* damp,
                                       int mass_weighted, const double* del6_u, const double* del6_v,
                                       const double* rarea, const double* gfx, const double* gfy, double* gq) {
  fv3b_grid_dims g{n, h, nk, 0};
  const fv3b::Dims d = fv3b::make_dims(&g);
  const int m = d.ni;
  std::vector<double> px(m * m), py(m * m), pq(m * m), wx(m * m), wy(m * m), wd(m * m);
  for (int k = 0; k < nk; ++k) {
    for (int p = 0; p < m * m; ++p) {
      px[p] = gfx[(long)p * nk + k];
      py[p] = gfy[(long)p * nk + k];
      pq[p] = 0.0;
    }
    const int nk_ = (int)nord_bands[k < 3 ? k : 3];
    fv3b::adj::delnflux_nosg_adjoint_level<double>(d, nmax, nk_, damp[k], 1.0, mass_weighted != 0, del6_u, del6_v,
                                                   rarea, m, 1, px.data(), py.data(), pq.data(), wx.data(), wy.data(),
                                                   wd.data());
    for (int p = 0; p < m * m; ++p) gq[(long)p * nk + k] += pq[p];
  }
}

// D-grid shallow water (d_sw) for all six tiles: flux preparation,
// finite-volume transport of delp, w, q_con, pt and vorticity, kinetic
// energy, divergence damping and the heat source.
//
// Reference: fv3core/stencils/d_sw.py (DGridShallowWaterLagrangianDynamics),
// fxadv.py, fvtp2d.py, delnflux.py, xtp_u.py/ytp_v.py, divergence_damping.py,
// a2b_ord4.py.  Launch order follows the data dependencies of the reference
// stencils; work within a launch is per point with the reference's
// statement order.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "a2b.cuh"
#include "transport.cuh"

using namespace fv3b;

namespace {

constexpr double DCON_THRESHOLD = 1e-5;

// ---------------------------------------------------------------- fxadv
// FiniteVolumeFluxPrep.__call__ (fxadv.py:488-585)
cudaError_t fxadv(const Dims d, const fv3b_metrics g, const real* uc, const real* vc, real* crx, real* cry,
                  real* xfx, real* yfx, real* ucc, real* vcc, real dt, cudaStream_t st) {
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec, nz = d.nz;
  const int full = d.ni - 1;
  cudaError_t err;
  // main_uc_contra + uc_contra_y_edge (fxadv.py:11-39, 61-71); main_vc_contra (42-58)
  err = launch_box(Box{0, full, 0, full, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    real u_old = F3(ucc, i, j), v_old = F3(vcc, i, j);
    real un = u_old;
    if (i >= s - 1 && i < e + 3) {
      real vv = RC(0.25) * (F3(vc, i - 1, j) + F3(vc, i, j) + F3(vc, i - 1, j + 1) + F3(vc, i, j + 1));
      un = (F3(uc, i, j) - vv * F2(g.cosa_u, i, j)) * F2(g.rsin_u, i, j);
    }
    if ((j >= js - 1 && j < js + 1) || (j >= je && j < je + 2)) un = u_old;
    if (i == s || i == e + 1) {
      real x = F3(uc, i, j);
      un = x > 0 ? x / F2(g.sin_sg3, i - 1, j) : x / F2(g.sin_sg1, i, j);
    }
    W3(ucc, i, j) = un;
    real vn = v_old;
    if (j >= js - 1 && j < je + 3) {
      real uu = RC(0.25) * (F3(uc, i, j - 1) + F3(uc, i + 1, j - 1) + F3(uc, i, j) + F3(uc, i + 1, j));
      vn = (F3(vc, i, j) - uu * F2(g.cosa_v, i, j)) * F2(g.rsin_v, i, j);
    }
    if (j == js || j == je + 1) vn = v_old;
    W3(vcc, i, j) = vn;
  });
  if (err != cudaSuccess) return err;
  // vc_contra_y_edge + vc_contra_x_edge (fxadv.py:97-150).  Only two kinds of
  // points change: the rows js and je+1 (every i) and, on the columns
  // is-1, is, ie, ie+1, the rows js+2 .. je-1; the two sets are disjoint
  // and each point reads only ucc and vc, so two small launches replace a
  // pass over the whole domain.
  err = launch_box(Box{0, full, 0, 2, 0, nz}, st, [=] __device__(int t, int i, int y, int k) {
    PT_SETUP(d, t, k);
    const int j = y == 0 ? js : je + 1;
    real vy = F3(vc, i, j);
    W3(vcc, i, j) = vy > 0 ? vy / F2(g.sin_sg4, i, j - 1) : vy / F2(g.sin_sg2, i, j);
  });
  if (err != cudaSuccess) return err;
  err = launch_box(Box{0, 4, js + 2, je, 0, nz}, st, [=] __device__(int t, int x, int j, int k) {
    PT_SETUP(d, t, k);
    const int i = x < 2 ? s - 1 + x : e + x - 2;
    real uu = RC(0.25) * (F3(ucc, i, j - 1) + F3(ucc, i + 1, j - 1) + F3(ucc, i, j) + F3(ucc, i + 1, j));
    W3(vcc, i, j) = (F3(vc, i, j) - uu * F2(g.cosa_v, i, j)) * RC(1.0);
  });
  if (err != cudaSuccess) return err;
  // uc_contra_x_edge (fxadv.py:74-94): rows js-1, js, je, je+1, columns
  // is+2 .. ie-1
  err = launch_box(Box{s + 2, e, 0, 4, 0, nz}, st, [=] __device__(int t, int i, int y, int k) {
    PT_SETUP(d, t, k);
    const int j = y < 2 ? js - 1 + y : je + y - 2;
    real vv = RC(0.25) * (F3(vcc, i - 1, j) + F3(vcc, i, j) + F3(vcc, i - 1, j + 1) + F3(vcc, i, j + 1));
    W3(ucc, i, j) = (F3(uc, i, j) - vv * F2(g.cosa_u, i, j)) * RC(1.0);
  });
  if (err != cudaSuccess) return err;
  // uc_contra_corners (fxadv.py:156-260): 8 points, none reads another's target
  err = launch_box(Box{0, 8, 0, 1, 0, nz}, st, [=] __device__(int t, int p, int, int k) {
    PT_SETUP(d, t, k);
    int i, j, kind;
    switch (p) {
      case 0: i = s + 1; j = js - 1; kind = 0; break;
      case 1: i = s + 1; j = je; kind = 0; break;
      case 2: i = s + 1; j = js; kind = 1; break;
      case 3: i = s + 1; j = je + 1; kind = 1; break;
      case 4: i = e; j = js - 1; kind = 2; break;
      case 5: i = e; j = je; kind = 2; break;
      case 6: i = e; j = js; kind = 3; break;
      default: i = e; j = je + 1; kind = 3; break;
    }
    real cu = F2(g.cosa_u, i, j), val;
    if (kind == 0) {
      real cv = F2(g.cosa_v, i - 1, j);
      real damp = RC(1.0) / (RC(1.0) - RC(0.0625) * cu * cv);
      val = (F3(uc, i, j) - RC(0.25) * cu *
                                (F3(vcc, i - 1, j + 1) + F3(vcc, i, j + 1) + F3(vcc, i, j) + F3(vc, i - 1, j) -
                                 RC(0.25) * cv * (F3(ucc, i - 1, j) + F3(ucc, i - 1, j - 1) + F3(ucc, i, j - 1)))) *
            damp;
    } else if (kind == 1) {
      real cv = F2(g.cosa_v, i - 1, j + 1);
      real damp = RC(1.0) / (RC(1.0) - RC(0.0625) * cu * cv);
      val = (F3(uc, i, j) - RC(0.25) * cu *
                                (F3(vcc, i - 1, j) + F3(vcc, i, j) + F3(vcc, i, j + 1) + F3(vc, i - 1, j + 1) -
                                 RC(0.25) * cv * (F3(ucc, i - 1, j) + F3(ucc, i - 1, j + 1) + F3(ucc, i, j + 1)))) *
            damp;
    } else if (kind == 2) {
      real cv = F2(g.cosa_v, i, j);
      real damp = RC(1.0) / (RC(1.0) - RC(0.0625) * cu * cv);
      val = (F3(uc, i, j) - RC(0.25) * cu *
                                (F3(vcc, i, j + 1) + F3(vcc, i - 1, j + 1) + F3(vcc, i - 1, j) + F3(vc, i, j) -
                                 RC(0.25) * cv * (F3(ucc, i + 1, j) + F3(ucc, i + 1, j - 1) + F3(ucc, i, j - 1)))) *
            damp;
    } else {
      real cv = F2(g.cosa_v, i, j + 1);
      real damp = RC(1.0) / (RC(1.0) - RC(0.0625) * cu * cv);
      val = (F3(uc, i, j) - RC(0.25) * cu *
                                (F3(vcc, i, j) + F3(vcc, i - 1, j) + F3(vcc, i - 1, j + 1) + F3(vc, i, j + 1) -
                                 RC(0.25) * cv * (F3(ucc, i + 1, j) + F3(ucc, i + 1, j + 1) + F3(ucc, i, j + 1)))) *
            damp;
    }
    W3(ucc, i, j) = val;
  });
  if (err != cudaSuccess) return err;
  // vc_contra_corners (fxadv.py:263-383)
  err = launch_box(Box{0, 8, 0, 1, 0, nz}, st, [=] __device__(int t, int p, int, int k) {
    PT_SETUP(d, t, k);
    int i, j, kind;
    switch (p) {
      case 0: i = s - 1; j = js + 1; kind = 0; break;
      case 1: i = e; j = js + 1; kind = 0; break;
      case 2: i = s; j = js + 1; kind = 1; break;
      case 3: i = e + 1; j = js + 1; kind = 1; break;
      case 4: i = e + 1; j = je; kind = 2; break;
      case 5: i = s; j = je; kind = 2; break;
      case 6: i = e; j = je; kind = 3; break;
      default: i = s - 1; j = je; kind = 3; break;
    }
    real cv = F2(g.cosa_v, i, j), val;
    const real* ut = ucc;
    if (kind == 0) {
      real cu = F2(g.cosa_u, i, j - 1);
      real damp = RC(1.0) / (RC(1.0) - RC(0.0625) * cu * cv);
      val = (F3(vc, i, j) - RC(0.25) * cv *
                                (F3(ut, i + 1, j - 1) + F3(ut, i + 1, j) + F3(ut, i, j) + F3(uc, i, j - 1) -
                                 RC(0.25) * cu * (F3(vcc, i, j - 1) + F3(vcc, i - 1, j - 1) + F3(vcc, i - 1, j)))) *
            damp;
    } else if (kind == 1) {
      real cu = F2(g.cosa_u, i + 1, j - 1);
      real damp = RC(1.0) / (RC(1.0) - RC(0.0625) * cu * cv);
      val = (F3(vc, i, j) - RC(0.25) * cv *
                                (F3(ut, i, j - 1) + F3(ut, i, j) + F3(ut, i + 1, j) + F3(uc, i + 1, j - 1) -
                                 RC(0.25) * cu * (F3(vcc, i, j - 1) + F3(vcc, i + 1, j - 1) + F3(vcc, i + 1, j)))) *
            damp;
    } else if (kind == 2) {
      real cu = F2(g.cosa_u, i + 1, j);
      real damp = RC(1.0) / (RC(1.0) - RC(0.0625) * cu * cv);
      val = (F3(vc, i, j) - RC(0.25) * cv *
                                (F3(ut, i, j) + F3(ut, i, j - 1) + F3(ut, i + 1, j - 1) + F3(uc, i + 1, j) -
                                 RC(0.25) * cu * (F3(vcc, i, j + 1) + F3(vcc, i + 1, j + 1) + F3(vcc, i + 1, j)))) *
            damp;
    } else {
      real cu = F2(g.cosa_u, i, j);
      real damp = RC(1.0) / (RC(1.0) - RC(0.0625) * cu * cv);
      val = (F3(vc, i, j) - RC(0.25) * cv *
                                (F3(ut, i + 1, j) + F3(ut, i + 1, j - 1) + F3(ut, i, j - 1) + F3(uc, i, j) -
                                 RC(0.25) * cu * (F3(vcc, i, j + 1) + F3(vcc, i - 1, j + 1) + F3(vcc, i - 1, j)))) *
            damp;
    }
    W3(vcc, i, j) = val;
  });
  if (err != cudaSuccess) return err;
  // fxadv_fluxes_stencil (fxadv.py:386-421)
  return launch_box(Box{0, full, 0, full, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    if (i >= s && i < e + 2) {
      real prod = dt * F3(ucc, i, j);
      if (prod > 0) {
        W3(crx, i, j) = prod * F2(g.rdxa, i - 1, j);
        W3(xfx, i, j) = F2(g.dy, i, j) * prod * F2(g.sin_sg3, i - 1, j);
      } else {
        W3(crx, i, j) = prod * F2(g.rdxa, i, j);
        W3(xfx, i, j) = F2(g.dy, i, j) * prod * F2(g.sin_sg1, i, j);
      }
    }
    if (j >= js && j < je + 2) {
      real prod = dt * F3(vcc, i, j);
      if (prod > 0) {
        W3(cry, i, j) = prod * F2(g.rdya, i, j - 1);
        W3(yfx, i, j) = F2(g.dx, i, j) * prod * F2(g.sin_sg4, i, j - 1);
      } else {
        W3(cry, i, j) = prod * F2(g.rdya, i, j);
        W3(yfx, i, j) = F2(g.dx, i, j) * prod * F2(g.sin_sg2, i, j);
      }
    }
  });
}

// ---------------------------------------------------------------- corner fills, sequential per level
// fill_corners_bgrid_{x,y} (corners.py:598-722) on levels [k0, k1).  The
// rules only touch the four 3 x 3 blocks i in [s-3, s-1] or [e+2, e+4],
// j in [js-3, js-1] or [je+2, je+4], so the launch covers those 36 points
// (x = block * 3 + column, y = row).
cudaError_t fill_bgrid(const Dims d, real* q, bool xdir, int k0, int k1, cudaStream_t st) {
  return launch_box(Box{0, 12, 0, 3, k0, k1}, st, [=] __device__(int t, int x, int y, int k) {
    PT_SETUP(d, t, k);
    const int c = x / 3, a = x % 3;
    const int i = (c == 0 || c == 2) ? d.isc - 3 + a : d.iec + 2 + a;
    const int j = c < 2 ? d.jsc - 3 + y : d.jec + 2 + y;
    int si, sj;
    bool hit = xdir ? bgrid_corner_x(d, i, j, si, sj) : bgrid_corner_y(d, i, j, si, sj);
    if (hit) W3(q, i, j) = F3(q, si, sj);
  });
}

// fill_corners_dgrid_defn (corners.py:993-1150) with x_in == x_out and
// y_in == y_out: the rules run in the reference's order, one thread per
// (tile, level), so reads see earlier rules' writes exactly as there.
cudaError_t fill_dgrid(const Dims d, real* x, real* y, real mysign, int k0, int k1, cudaStream_t st) {
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  return launch_box(Box{0, 1, 0, 1, k0, k1}, st, [=] __device__(int t, int, int, int k) {
    PT_SETUP(d, t, k);
    auto X = [&](int i, int j) -> real& { return x[_b3 + j * _sj + i]; };
    auto Y = [&](int i, int j) -> real& { return y[_b3 + j * _sj + i]; };
    const real m = mysign;
    // sw corner
    X(s - 1, js - 1) = m * Y(s - 1, js);
    Y(s - 1, js - 1) = m * X(s, js - 1);
    X(s - 1, js - 2) = m * Y(s - 2, js);
    Y(s - 1, js - 2) = m * X(s + 1, js - 1);
    X(s - 1, js - 3) = m * Y(s - 3, js);
    Y(s - 1, js - 3) = m * X(s + 2, js - 1);
    X(s - 2, js - 1) = m * Y(s - 1, js + 1);
    Y(s - 2, js - 1) = m * X(s, js - 2);
    X(s - 2, js - 2) = m * Y(s - 2, js + 1);
    Y(s - 2, js - 2) = m * X(s + 1, js - 2);
    X(s - 2, js - 3) = m * Y(s - 3, js + 1);
    Y(s - 2, js - 3) = m * X(s + 2, js - 2);
    X(s - 3, js - 1) = m * Y(s - 1, js + 2);
    Y(s - 3, js - 1) = m * X(s, js - 3);
    X(s - 3, js - 2) = m * Y(s - 2, js + 2);
    Y(s - 3, js - 2) = m * X(s + 1, js - 3);
    X(s - 3, js - 3) = m * Y(s - 3, js + 2);
    Y(s - 3, js - 3) = m * X(s + 2, js - 3);
    // ne corner
    X(e + 1, je + 2) = m * Y(e + 2, je);
    Y(e + 2, je + 1) = m * X(e, je + 2);
    X(e + 1, je + 3) = m * Y(e + 3, je);
    Y(e + 2, je + 2) = m * X(e - 1, je + 2);
    X(e + 1, je + 4) = m * Y(e + 4, je);
    Y(e + 2, je + 3) = m * X(e - 2, je + 2);
    X(e + 2, je + 2) = m * Y(e + 2, je - 1);
    Y(e + 3, je + 1) = m * X(e, je + 3);
    X(e + 2, je + 3) = m * Y(e + 3, je - 1);
    Y(e + 3, je + 2) = m * X(e - 1, je + 3);
    X(e + 2, je + 4) = m * Y(e + 4, je - 1);
    Y(e + 3, je + 3) = m * X(e - 2, je + 3);
    X(e + 3, je + 2) = m * Y(e + 2, je - 2);
    Y(e + 4, je + 1) = m * X(e, je + 4);
    X(e + 3, je + 3) = m * Y(e + 3, je - 2);
    Y(e + 4, je + 2) = m * X(e - 1, je + 4);
    X(e + 3, je + 4) = m * Y(e + 4, je - 2);
    Y(e + 4, je + 3) = m * X(e - 2, je + 4);
    // nw corner
    X(s - 1, je + 2) = Y(s - 1, je);
    Y(s - 1, je + 1) = X(s, je + 2);
    X(s - 1, je + 3) = Y(s - 2, je);
    Y(s - 1, je + 2) = X(s + 1, je + 2);
    X(s - 1, je + 4) = Y(s - 3, je);
    Y(s - 1, je + 3) = X(s + 2, je + 2);
    X(s - 2, je + 2) = Y(s - 1, je - 1);
    Y(s - 2, je + 1) = X(s, je + 3);
    X(s - 2, je + 3) = Y(s - 2, je - 1);
    Y(s - 2, je + 2) = X(s + 1, je + 3);
    X(s - 2, je + 4) = Y(s - 3, je - 1);
    Y(s - 2, je + 3) = X(s + 2, je + 3);
    X(s - 3, je + 2) = Y(s - 1, je - 2);
    Y(s - 3, je + 1) = X(s, je + 4);
    X(s - 3, je + 3) = Y(s - 2, je - 2);
    Y(s - 3, je + 2) = X(s + 1, je + 4);
    X(s - 3, je + 4) = Y(s - 3, je - 2);
    Y(s - 3, je + 3) = X(s + 2, je + 4);
    // se corner
    X(e + 1, js - 1) = Y(e + 2, js);
    Y(e + 2, js - 1) = X(e, js - 1);
    X(e + 1, js - 2) = Y(e + 3, js);
    Y(e + 2, js - 2) = X(e - 1, js - 1);
    X(e + 1, js - 3) = Y(e + 4, js);
    Y(e + 2, js - 3) = X(e - 2, js - 1);
    X(e + 2, js - 1) = Y(e + 2, js + 1);
    Y(e + 3, js - 1) = X(e, js - 2);
    X(e + 2, js - 2) = Y(e + 3, js + 1);
    Y(e + 3, js - 2) = X(e - 1, js - 2);
    X(e + 2, js - 3) = Y(e + 4, js + 1);
    Y(e + 3, js - 3) = X(e - 2, js - 2);
    X(e + 3, js - 1) = Y(e + 2, js + 2);
    Y(e + 4, js - 1) = X(e, js - 3);
    X(e + 3, js - 2) = Y(e + 3, js + 2);
    Y(e + 4, js - 2) = X(e - 1, js - 3);
    X(e + 3, js - 3) = Y(e + 4, js + 2);
    Y(e + 4, js - 3) = X(e - 2, js - 3);
  });
}

inline double min_(double a, double b) { return a < b ? a : b; }
inline double max_(double a, double b) { return a > b ? a : b; }

}  // namespace

extern "C" int fv3b_d_sw_setup(fv3b_ctx* ctx, const fv3b_dsw_config* cfg) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && cfg, "fv3b_d_sw_setup: null argument");
  if (cfg->grid_type >= 3 || cfg->inline_q || cfg->d_ext > 0.0) {
    set_last_error_msg("fv3b_d_sw_setup: grid_type >= 3, inline_q and d_ext > 0 are not implemented");
    return FV3B_ERR_UNSUPPORTED;
  }
  const int npz = ctx->d.nz;
  const int n = npz + 1;
  std::vector<double> cols((size_t)NCOL * MAXLEV, 0.0);
  auto C = [&](int id) { return cols.data() + (size_t)id * MAXLEV; };
  // get_column_namelist (d_sw.py:512-563)
  for (int k = 0; k < n; ++k) {
    C(COL_KE_BG)[k] = cfg->ke_bg;
    C(COL_D_CON)[k] = cfg->d_con;
    C(COL_NORD)[k] = cfg->nord;
    C(COL_D2_DIVG)[k] = min_(0.2, cfg->d2_bg);
  }
  for (int k = 0; k < n; ++k) {
    C(COL_NORD_V)[k] = min_(2.0, C(COL_NORD)[0]);
    C(COL_NORD_W)[k] = C(COL_NORD_V)[0];
    C(COL_NORD_T)[k] = C(COL_NORD_V)[0];
    C(COL_DAMP_VT)[k] = cfg->do_vort_damp ? cfg->vtdm4 : 0.0;
  }
  for (int k = 0; k < n; ++k) {
    C(COL_DAMP_W)[k] = C(COL_DAMP_VT)[0];
    C(COL_DAMP_T)[k] = C(COL_DAMP_VT)[0];
  }
  auto set_low = [&](int k) {
    C(COL_NORD)[k] = 0;
    C(COL_NORD_W)[k] = 0;
    C(COL_D_CON)[k] = 0;
    C(COL_DAMP_W)[k] = C(COL_D2_DIVG)[k];
  };
  auto vort_opt = [&](int k) {
    if (cfg->do_vort_damp) {
      C(COL_NORD_V)[k] = 0;
      C(COL_DAMP_VT)[k] = 0.5 * C(COL_D2_DIVG)[k];
    }
  };
  if (npz == 1 || cfg->n_sponge < 0) {
    C(COL_D2_DIVG)[0] = cfg->d2_bg;
  } else {
    C(COL_D2_DIVG)[0] = max_(0.01, max_(cfg->d2_bg, cfg->d2_bg_k1));
    set_low(0);
    vort_opt(0);
    if (cfg->d2_bg_k2 > 0.01) {
      C(COL_D2_DIVG)[1] = max_(cfg->d2_bg, cfg->d2_bg_k2);
      set_low(1);
      vort_opt(1);
    }
    if (cfg->d2_bg_k2 > 0.05) {
      C(COL_D2_DIVG)[2] = max_(cfg->d2_bg, 0.2 * cfg->d2_bg_k2);
      set_low(2);
    }
  }
  // DGridShallowWaterLagrangianDynamics.__init__ assertions (d_sw.py:624-634)
  for (int k = 0; k < n; ++k) {
    if (!(C(COL_DAMP_VT)[k] > DCON_THRESHOLD) || !(C(COL_DAMP_W)[k] > DCON_THRESHOLD)) {
      set_last_error_msg("fv3b_d_sw_setup: damp_vt and damp_w must exceed 1e-5 on every level");
      return FV3B_ERR_UNSUPPORTED;
    }
  }
  // calc_damp (delnflux.py:24-26): d_sw's own damping uses da_min_c, the
  // transport damping (DelnFlux) uses da_min
  for (int k = 0; k < npz; ++k) {
    C(COL_DAMP4_VT_C)[k] = pow(C(COL_DAMP_VT)[k] * ctx->m.da_min_c, C(COL_NORD_V)[k] + 1);
    C(COL_DAMP4_W_C)[k] = pow(C(COL_DAMP_W)[k] * ctx->m.da_min_c, C(COL_NORD_W)[k] + 1);
    C(COL_DAMP4_VT)[k] = pow(C(COL_DAMP_VT)[k] * ctx->m.da_min, C(COL_NORD_V)[k] + 1);
    C(COL_DAMP4_T)[k] = pow(C(COL_DAMP_T)[k] * ctx->m.da_min, C(COL_NORD_T)[k] + 1);
  }
  DswSetup& sp = ctx->dsw;
  sp.cfg = *cfg;
  auto nmax = [&](int id) {
    double m = 0;
    for (int k = 0; k < n; ++k) m = max_(m, C(id)[k]);
    return (int)m;
  };
  sp.nmax_v = nmax(COL_NORD_V);
  sp.nmax_w = nmax(COL_NORD_W);
  sp.nmax_t = nmax(COL_NORD_T);
  if (sp.nmax_v > 3 || sp.nmax_w > 3 || sp.nmax_t > 3) {
    set_last_error_msg("fv3b_d_sw_setup: nord must be less than 3");
    return FV3B_ERR_ARGUMENT;
  }
  // DivergenceDamping.__init__ (divergence_damping.py:203-218)
  sp.nonzero_nord_k = 0;
  sp.nonzero_nord = cfg->nord;
  for (int k = 0; k < n; ++k) {
    if (C(COL_NORD)[k] > 0) {
      sp.nonzero_nord_k = k;
      sp.nonzero_nord = (int)C(COL_NORD)[k];
      break;
    }
  }
  sp.dd8 = pow(ctx->m.da_min_c * cfg->d4_bg, sp.nonzero_nord + 1);
  // Range scaling of the del-n iterations.  Each pass of a del-n operator
  // divides by a cell area (1e8..1e12 m^2) and the damping coefficient
  // carries one area per pass, so at nord = 3 the coefficients
  // (damp * da_min)^4 reach 1e40 and the iterated differences 1e-40: outside
  // the single-precision range.  With fields in single precision every pass
  // multiplies by S, a power of two near the smallest area, and the
  // coefficient of a level that takes nmax passes is divided by S^nmax.  S is
  // a power of two, so both scalings are exact and the fluxes are the same
  // numbers the unscaled formula gives; double builds use S = 1.
  const bool scale_range = sizeof(fv3b::real) < sizeof(double);
  sp.area_scale = scale_range ? std::ldexp(1.0, std::ilogb(ctx->m.da_min)) : 1.0;
  sp.area_scale_c = scale_range ? std::ldexp(1.0, std::ilogb(ctx->m.da_min_c)) : 1.0;
  auto scale_levels = [&](int damp_id, int nord_id, int nmax, double scale) {
    if (nmax == 0) return;
    const double f = std::pow(scale, -nmax);
    for (int k = 0; k < MAXLEV; ++k)
      if (C(nord_id)[k < 3 ? k : 3] > 0) C(damp_id)[k] *= f;
  };
  // UpdateHeightOnDGrid damps with the raw damp_vt column over npz + 1 levels
  for (int k = 0; k < MAXLEV; ++k) C(COL_DAMP_VT_DZ)[k] = C(COL_DAMP_VT)[k];
  scale_levels(COL_DAMP_VT_DZ, COL_NORD_V, sp.nmax_v, sp.area_scale);
  scale_levels(COL_DAMP4_VT, COL_NORD_V, sp.nmax_v, sp.area_scale);
  scale_levels(COL_DAMP4_T, COL_NORD_T, sp.nmax_t, sp.area_scale);
  scale_levels(COL_DAMP4_W_C, COL_NORD_W, sp.nmax_w, sp.area_scale);
  scale_levels(COL_DAMP4_VT_C, COL_NORD_V, sp.nmax_v, sp.area_scale);
  sp.dd8_scaled = sp.dd8 * std::pow(sp.area_scale_c, -sp.nonzero_nord);
  // the D-grid columns only; the driver's columns (from COL_DP_REF on) are its own
  const std::vector<real> cols_r(cols.begin(), cols.begin() + (size_t)COL_DP_REF * MAXLEV);
  FV3B_CHECK(cudaMemcpy(ctx->col, cols_r.data(), sizeof(real) * cols_r.size(), cudaMemcpyHostToDevice));
  sp.ready = true;
  return FV3B_OK;
}

extern "C" int fv3b_d_sw(fv3b_ctx* ctx, real* delpc, real* delp, real* ptc, real* pt, real* u, real* v,
                         real* w, real* uc, real* vc, const real* ua, const real* va, real* divgd,
                         real* mfx, real* mfy, real* cx, real* cy, real* crx, real* cry, real* xfx,
                         real* yfx, real* q_con, const real* zh, real* heat_source, real* diss_est,
                         double dt_in, void* stream) {
  FV3B_TILES(ctx);
  // the build's precision inside the kernels (the same value in FP64 builds)
  const real dt = static_cast<real>(dt_in);
  FV3B_REQUIRE(ctx && delpc && delp && ptc && pt && u && v && w && uc && vc && ua && va && divgd && mfx && mfy &&
                   cx && cy && crx && cry && xfx && yfx && q_con && zh && heat_source && diss_est,
               "fv3b_d_sw: null argument");
  FV3B_REQUIRE(ctx->dsw.ready, "fv3b_d_sw: call fv3b_d_sw_setup first");
  const Dims d = ctx->d;
  const fv3b_metrics g = ctx->m;
  const DswSetup sp = ctx->dsw;
  const fv3b_dsw_config cfg = sp.cfg;
  cudaStream_t st = (cudaStream_t)stream;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec, nz = d.nz;
  const int full = d.ni - 1;
  real** W = ctx->ws;
  real *tmp_fx = W[0], *tmp_fy = W[1], *tmp_gx = W[2], *tmp_gy = W[3], *tmp_fx2 = W[4], *tmp_fy2 = W[5];
  real *tmp_dw = W[6], *tmp_wk = W[7], *tmp_vort = W[8], *tmp_ke = W[9], *tmp_heat_s = W[10];
  real *tmp_ut = W[11], *tmp_vt = W[12], *vort_x_delta = W[13], *vort_y_delta = W[14];
  real *fx_mean = W[16], *fy_mean = W[17], *q_adv_x = W[18], *q_adv_y = W[19];
  real *dl_fx2 = W[20], *dl_fy2 = W[21], *dl_d2 = W[22];
  real *a2b_qx = W[23], *a2b_qy = W[24], *a2b_edges = W[25];
  real* deln_alt = W[WS_DELN_ALT];
  real *ucc = W[WS_UC_CONTRA], *vcc = W[WS_VC_CONTRA];
  const real* col_nord = colp(ctx, COL_NORD);
  const real* col_d2_divg = colp(ctx, COL_D2_DIVG);
  const real* col_d_con = colp(ctx, COL_D_CON);
  const real* col_ke_bg = colp(ctx, COL_KE_BG);
  const real* col_damp_w = colp(ctx, COL_DAMP_W);
  const real* col_damp_vt = colp(ctx, COL_DAMP_VT);
  const real area_scale = static_cast<real>(sp.area_scale);
  DelnCol dl_v{colp(ctx, COL_NORD_V), colp(ctx, COL_DAMP4_VT), area_scale};
  DelnCol dl_t{colp(ctx, COL_NORD_T), colp(ctx, COL_DAMP4_T), area_scale};
  DelnCol nosg_w{colp(ctx, COL_NORD_W), colp(ctx, COL_DAMP4_W_C), area_scale};
  DelnCol nosg_v{colp(ctx, COL_NORD_V), colp(ctx, COL_DAMP4_VT_C), area_scale};

  FV3B_CHECK(fxadv(d, g, uc, vc, crx, cry, xfx, yfx, ucc, vcc, dt, st));

  auto transport = [&](real* q, real* fx, real* fy, int hord, const real* xmf, const real* ymf,
                       const real* mass, const DelnCol* dl, int nmax) -> cudaError_t {
    cudaError_t err = copy_corners_x_inplace(d, q, st);
    if (err != cudaSuccess) return err;
    FvTp2dArgs a{q, crx, cry, xfx, yfx, xmf ? xmf : xfx, ymf ? ymf : yfx, fx, fy, hord,
                 fx_mean, fy_mean, q_adv_x, q_adv_y};
    err = fvtp2d(d, g, a, st);
    if (err != cudaSuccess) return err;
    if (dl) err = delnflux(d, g, q, fx, fy, *dl, mass, dl_fx2, dl_fy2, dl_d2, deln_alt, nmax, st);
    return err;
  };
  // delp transport (d_sw.py:910-918) and flux_capacitor (90-117)
  FV3B_CHECK(transport(delp, tmp_fx, tmp_fy, cfg.hord_dp, nullptr, nullptr, nullptr, &dl_v, sp.nmax_v));
  FV3B_CHECK(launch_box(Box{0, full, 0, full, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    W3(cx, i, j) = F3(cx, i, j) + F3(crx, i, j);
    W3(cy, i, j) = F3(cy, i, j) + F3(cry, i, j);
    W3(mfx, i, j) = F3(mfx, i, j) + F3(tmp_fx, i, j);
    W3(mfy, i, j) = F3(mfy, i, j) + F3(tmp_fy, i, j);
  }));
  if (!cfg.hydrostatic) {
    FV3B_CHECK(delnflux_nosg(d, g, w, tmp_fx2, tmp_fy2, nosg_w, tmp_wk, deln_alt, false, sp.nmax_w, st));
    // heat_diss (d_sw.py:347-365)
    const real adt = fabs(dt);
    FV3B_CHECK(launch_box(Box{s, e + 1, js, je + 1, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
      PT_SETUP(d, t, k);
      real diss_e = F3(diss_est, i, j);
      if (col_damp_w[k] > RC(1e-5)) {
        real dd8 = col_ke_bg[k] * adt;
        real dw = (F3(tmp_fx2, i, j) - F3(tmp_fx2, i + 1, j) + F3(tmp_fy2, i, j) - F3(tmp_fy2, i, j + 1)) *
                    F2(g.rarea, i, j);
        W3(tmp_dw, i, j) = dw;
        real hs = dd8 - dw * (F3(w, i, j) + RC(0.5) * dw);
        W3(tmp_heat_s, i, j) = hs;
        W3(diss_est, i, j) = diss_e + hs;
      }
    }));
    FV3B_CHECK(transport(w, tmp_gx, tmp_gy, cfg.hord_vt, tmp_fx, tmp_fy, nullptr, nullptr, 0));
    // flux_adjust on w (d_sw.py:67-87)
    FV3B_CHECK(launch_box(Box{s, e + 1, js, je + 1, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
      PT_SETUP(d, t, k);
      W3(w, i, j) = F3(w, i, j) * F3(delp, i, j) +
                    (F3(tmp_gx, i, j) - F3(tmp_gx, i + 1, j) + F3(tmp_gy, i, j) - F3(tmp_gy, i, j + 1)) *
                        F2(g.rarea, i, j);
    }));
  }
  // q_con transport and flux_adjust (d_sw.py:967-982)
  FV3B_CHECK(transport(q_con, tmp_gx, tmp_gy, cfg.hord_dp, tmp_fx, tmp_fy, delp, &dl_t, sp.nmax_t));
  FV3B_CHECK(launch_box(Box{s, e + 1, js, je + 1, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    W3(q_con, i, j) = F3(q_con, i, j) * F3(delp, i, j) +
                      (F3(tmp_gx, i, j) - F3(tmp_gx, i + 1, j) + F3(tmp_gy, i, j) - F3(tmp_gy, i, j + 1)) *
                          F2(g.rarea, i, j);
  }));
  // pt transport and apply_pt_delp_fluxes (d_sw.py:163-195, 985-1005)
  FV3B_CHECK(transport(pt, tmp_gx, tmp_gy, cfg.hord_tm, tmp_fx, tmp_fy, delp, &dl_v, sp.nmax_v));
  FV3B_CHECK(launch_box(Box{s, e + 1, js, je + 1, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    real ra = F2(g.rarea, i, j);
    real dp = F3(delp, i, j);
    real ptn = F3(pt, i, j) * dp + (F3(tmp_gx, i, j) - F3(tmp_gx, i + 1, j) + F3(tmp_gy, i, j) - F3(tmp_gy, i, j + 1)) * ra;
    real dpn = dp + (F3(tmp_fx, i, j) - F3(tmp_fx, i + 1, j) + F3(tmp_fy, i, j) - F3(tmp_fy, i, j + 1)) * ra;
    W3(pt, i, j) = ptn / dpn;
    W3(delp, i, j) = dpn;
  }));
  // kinetic_energy_update_part_1 + part_2 (d_sw.py:198-246, 566-603; xtp_u.py, ytp_v.py)
  {
    const int mord = cfg.hord_mt < 0 ? -cfg.hord_mt : cfg.hord_mt;
    // the columns whose x-advection takes the interior PPM path in warps of their own
    FV3B_CHECK(launch_box_split(Box{s, e + 2, js, je + 2, 0, nz}, s + 3, e - 1, st,
                                [=] __device__(int t, int i, int j, int k) {
      PT_SETUP(d, t, k);
      real ub_cov = RC(0.5) * (F3(uc, i, j - 1) + F3(uc, i, j));
      real vb_cov = RC(0.5) * (F3(vc, i - 1, j) + F3(vc, i, j));
      real ca = F2(g.cosa, i, j), rs = F2(g.rsina, i, j);
      real ubc = (ub_cov - vb_cov * ca) * rs;
      real vbc = (vb_cov - ub_cov * ca) * rs;
      bool ns = (j == js || j == je + 1), ew = (i == s || i == e + 1);
      if (ns) ubc = RC(0.25) * (-F3(ucc, i, j - 2) + RC(3.0) * (F3(ucc, i, j - 1) + F3(ucc, i, j)) - F3(ucc, i, j + 1));
      if (ew) ubc = RC(0.5) * (F3(ucc, i, j - 1) + F3(ucc, i, j));
      if (ew) vbc = RC(0.25) * (-F3(vcc, i - 2, j) + RC(3.0) * (F3(vcc, i - 1, j) + F3(vcc, i, j)) - F3(vcc, i + 1, j));
      if (ns) vbc = RC(0.5) * (F3(vcc, i - 1, j) + F3(vcc, i, j));
      // advect_v_along_y and advect_u_along_x: PPM of the D-grid wind with
      // cell-edge spacing dx/dy, corner-zeroed edge perturbations
      auto advect = [&](auto qline, auto dxline, real rdx_m, real rdx_0, real ub, int pos, int sA, int eA,
                        bool zero_m, bool zero_0) {
        real alm, al0, alp;
        ppm_al3(qline, dxline, pos, sA, eA, alm, al0, alp);
        real qm = qline(-1), q0 = qline(0);
        real blm = alm - qm, brm = al0 - qm;
        real bl0 = al0 - q0, br0 = alp - q0;
        if (zero_m) { blm = RC(0.0); brm = RC(0.0); }
        if (zero_0) { bl0 = RC(0.0); br0 = RC(0.0); }
        real b0m = blm + brm, b00 = bl0 + br0;
        real cfl = ub > 0 ? ub * dt * rdx_m : ub * dt * rdx_0;
        real fx0 = cfl > RC(0.0) ? (RC(1.0) - cfl) * (brm - cfl * b0m) : (RC(1.0) + cfl) * (bl0 + cfl * b00);
        real mask = (ppm_smooth(blm, b0m, brm, mord) || ppm_smooth(bl0, b00, br0, mord)) ? RC(1.0) : RC(0.0);
        return ub > RC(0.0) ? qm + fx0 * mask : q0 + fx0 * mask;
      };
      // zero-corner regions of get_bl_br (xtp_u.py:40-46 / ytp_v.py)
      auto zc_x = [&](int ii, int jj) {
        return ((ii >= s - 1 && ii < s + 1) || (ii >= e && ii < e + 2)) && (jj == js || jj == je + 1);
      };
      auto zc_y = [&](int ii, int jj) {
        return (ii == s || ii == e + 1) && ((jj >= js - 1 && jj < js + 1) || (jj >= je && jj < je + 2));
      };
      real adv_v = advect(line3<1>(d, v, t, i, j, k), line2<1>(d, g.dy, t, i, j), F2(g.rdy, i, j - 1),
                            F2(g.rdy, i, j), vbc, j, js, je, zc_y(i, j - 1), zc_y(i, j));
      real adv_u = advect(line3<0>(d, u, t, i, j, k), line2<0>(d, g.dx, t, i, j), F2(g.rdx, i - 1, j),
                            F2(g.rdx, i, j), ubc, i, s, e, zc_x(i - 1, j), zc_x(i, j));
      real ke = RC(0.5) * dt * (ubc * adv_u + vbc * adv_v);
      // all_corners_ke (d_sw.py:121-160)
      auto corner_ke = [&](int io1, int jo1, int io2, int vsign) {
        real dt6 = dt / RC(6.0);
        real ut0 = F3(ucc, i, j), utm = F3(ucc, i, j - 1);
        real vt0 = F3(vcc, i, j), vtm = F3(vcc, i - 1, j);
        real u0 = F3(u, i, j), um = F3(u, i - 1, j), v0 = F3(v, i, j), vm = F3(v, i, j - 1);
        return dt6 * ((ut0 + utm) * ((io1 + 1) * u0 - (io1 * um)) + (vt0 + vtm) * ((jo1 + 1) * v0 - (jo1 * vm)) +
                      (((jo1 + 1) * ut0 - (jo1 * utm)) + vsign * ((io1 + 1) * vt0 - (io1 * vtm))) *
                          ((io2 + 1) * u0 - (io2 * um)));
      };
      if (i == s && j == js) ke = corner_ke(0, 0, -1, 1);
      if (i == e + 1 && j == js) ke = corner_ke(-1, 0, 0, -1);
      if (i == e + 1 && j == je + 1) ke = corner_ke(-1, -1, 0, 1);
      if (i == s && j == je + 1) ke = corner_ke(0, -1, -1, -1);
      W3(tmp_ke, i, j) = ke;
    }));
  }
  // compute_vorticity (d_sw.py:468-490), full halo domain
  FV3B_CHECK(launch_box(Box{0, full, 0, full, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    real ra = F2(g.rarea, i, j);
    real dxv = F2(g.dx, i, j), dyv = F2(g.dy, i, j);
    real rdy_tmp = ra * dxv, rdx_tmp = ra * dyv;
    W3(tmp_wk, i, j) = (F3(u, i, j) - F3(u, i, j + 1) * F2(g.dx, i, j + 1) / dxv) * rdy_tmp +
                       (F3(v, i + 1, j) * F2(g.dy, i + 1, j) / dyv - F3(v, i, j)) * rdx_tmp;
  }));
  // adjust_w_and_qcon (d_sw.py:324-335)
  FV3B_CHECK(launch_box(Box{s, e + 1, js, je + 1, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    real dp = F3(delp, i, j);
    real wn = F3(w, i, j) / dp;
    if (col_damp_w[k] > RC(1e-5)) wn = wn + F3(tmp_dw, i, j);
    W3(w, i, j) = wn;
    W3(q_con, i, j) = F3(q_con, i, j) / dp;
  }));
  // ---------------- DivergenceDamping.__call__ (divergence_damping.py:329-413)
  {
    const int kz = sp.nonzero_nord_k;
    const int nn = sp.nonzero_nord;
    const real dddmp = cfg.dddmp, da_min_c = g.da_min_c, dd8 = sp.dd8_scaled;
    const real rscale_c = static_cast<real>(sp.area_scale_c);
    real* u_contra_dyc = ptc;
    real* v_contra_dxc = tmp_vort;
    if (kz > 0) {
      // get_delpc, first computation, on the extent its second one reads
      FV3B_CHECK(launch_box(Box{s - 1, e + 2, js - 1, je + 2, 0, kz}, st, [=] __device__(int t, int i, int j, int k) {
        PT_SETUP(d, t, k);
        if (j >= js) {
          real vfv = RC(0.5) * (F3(va, i, j - 1) + F3(va, i, j));
          real uct = (F3(u, i, j) - vfv * F2(g.cosa_v, i, j)) * F2(g.sina_v, i, j);
          if (j == js || j == je + 1)
            uct = F3(vc, i, j) > 0 ? F3(u, i, j) * F2(g.sin_sg4, i, j - 1) : F3(u, i, j) * F2(g.sin_sg2, i, j);
          W3(u_contra_dyc, i, j) = uct * F2(g.dyc, i, j);
        }
        if (i >= s) {
          real ufu = RC(0.5) * (F3(ua, i - 1, j) + F3(ua, i, j));
          real vct = (F3(v, i, j) - ufu * F2(g.cosa_u, i, j)) * F2(g.sina_u, i, j);
          if (i == s || i == e + 1)
            vct = F3(uc, i, j) > 0 ? F3(v, i, j) * F2(g.sin_sg3, i - 1, j) : F3(v, i, j) * F2(g.sin_sg1, i, j);
          real vcd = vct * F2(g.dxc, i, j);
          if ((i == s || i == e + 1) && (j == je + 1 || j == js - 1)) vcd = RC(0.0);
          W3(v_contra_dxc, i, j) = vcd;
        }
      }));
    }
    // get_delpc second computation (k < kz); copy_computeplus (k >= kz)
    FV3B_CHECK(launch_box(Box{s, e + 2, js, je + 2, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
      PT_SETUP(d, t, k);
      if (k < kz) {
        real dpc = F3(v_contra_dxc, i, j - 1) - F3(v_contra_dxc, i, j) + F3(u_contra_dyc, i - 1, j) -
                     F3(u_contra_dyc, i, j);
        W3(delpc, i, j) = F2(g.rarea_c, i, j) * dpc;
      } else {
        W3(delpc, i, j) = F3(divgd, i, j);
      }
    }));
    // damping (divergence_damping.py:94-107) on k < kz.  It overwrites
    // v_contra_dxc, which the launch above reads one row down, so it is a
    // launch of its own: in one launch a block could read a row another
    // block has already overwritten.
    if (kz > 0) {
      FV3B_CHECK(launch_box(Box{s, e + 2, js, je + 2, 0, kz}, st, [=] __device__(int t, int i, int j, int k) {
        PT_SETUP(d, t, k);
        const real dpc = F3(delpc, i, j);
        real delpcdt = dpc * dt;
        real mintmp = fmin(RC(0.2), dddmp * fabs(delpcdt));
        real damp = da_min_c * fmax(col_d2_divg[k], mintmp);
        real vort = damp * dpc;
        W3(v_contra_dxc, i, j) = vort;
        W3(tmp_ke, i, j) = F3(tmp_ke, i, j) + vort;
      }));
    }
    for (int n = 0; n < nn; ++n) {
      const int nt = nn - n - 1;
      const bool fillc = n + 1 != nn;
      if (fillc) FV3B_CHECK(fill_bgrid(d, divgd, true, kz, nz + 1, st));
      // vc_from_divg (divergence_damping.py:126-128)
      FV3B_CHECK(launch_box(Box{s - nt - 1, e + nt + 2, js - nt, je + nt + 2, kz, nz}, st,
                            [=] __device__(int t, int i, int j, int k) {
                              PT_SETUP(d, t, k);
                              W3(vc, i, j) = (F3(divgd, i + 1, j) - F3(divgd, i, j)) * F2(g.divg_u, i, j);
                            }));
      if (fillc) FV3B_CHECK(fill_bgrid(d, divgd, false, kz, nz + 1, st));
      FV3B_CHECK(launch_box(Box{s - nt, e + nt + 2, js - nt - 1, je + nt + 2, kz, nz}, st,
                            [=] __device__(int t, int i, int j, int k) {
                              PT_SETUP(d, t, k);
                              W3(uc, i, j) = (F3(divgd, i, j + 1) - F3(divgd, i, j)) * F2(g.divg_v, i, j);
                            }));
      if (fillc) FV3B_CHECK(fill_dgrid(d, vc, uc, -RC(1.0), kz, nz, st));
      // redo_divg_d (divergence_damping.py:136-151)
      FV3B_CHECK(launch_box(Box{s - nt, e + nt + 2, js - nt, je + nt + 2, kz, nz}, st,
                            [=] __device__(int t, int i, int j, int k) {
                              PT_SETUP(d, t, k);
                              real dd = F3(uc, i, j - 1) - F3(uc, i, j) + F3(vc, i - 1, j) - F3(vc, i, j);
                              bool ci = (i == s || i == e + 1);
                              if (ci && j == js) dd = F3(vc, i - 1, j) - F3(vc, i, j) - F3(uc, i, j);
                              if (ci && j == je + 1) dd = F3(uc, i, j - 1) + F3(vc, i - 1, j) - F3(vc, i, j);
                              W3(divgd, i, j) = dd * F2(g.rarea_c, i, j) * rscale_c;
                            }));
    }
    // _vorticity_calc: a2b_ord4(wk -> vort) then smagorinsky, on k >= kz
    if (dddmp < RC(1e-5)) {
      FV3B_CHECK(launch_box(Box{s - 3, e + 5, js - 3, je + 5, kz, nz}, st, [=] __device__(int t, int i, int j, int k) {
        PT_SETUP(d, t, k);
        W3(v_contra_dxc, i, j) = RC(0.0);
      }));
    } else {
      FV3B_CHECK(a2b_ord4(d, g, tmp_wk, v_contra_dxc, a2b_qx, a2b_qy, a2b_edges, kz, nz, st));
    }
    // smagorinsky_diffusion_approx + damping_nord_highorder (110-123, 154-156)
    const real adt = fabs(dt);
    const bool smag = !(dddmp < RC(1e-5));
    FV3B_CHECK(launch_box(Box{s, e + 2, js, je + 2, kz, nz}, st, [=] __device__(int t, int i, int j, int k) {
      PT_SETUP(d, t, k);
      real dpc = F3(delpc, i, j);
      real vort = F3(v_contra_dxc, i, j);
      if (smag) vort = adt * sqrt(dpc * dpc + vort * vort);
      real mintmp = fmin(RC(0.2), dddmp * fabs(vort));
      real damp = da_min_c * fmax(col_d2_divg[k], mintmp);
      vort = damp * dpc + dd8 * F3(divgd, i, j);
      W3(v_contra_dxc, i, j) = vort;
      W3(tmp_ke, i, j) = F3(tmp_ke, i, j) + vort;
    }));
  }
  // vort_differencing (d_sw.py:249-265)
  FV3B_CHECK(launch_box(Box{s, e + 2, js, je + 2, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    if (!(col_d_con[k] > DCON_THRESHOLD)) return;
    if (i <= e) W3(vort_x_delta, i, j) = F3(tmp_vort, i, j) - F3(tmp_vort, i + 1, j);
    if (j <= je) W3(vort_y_delta, i, j) = F3(tmp_vort, i, j) - F3(tmp_vort, i, j + 1);
  }));
  // compute_vort (d_sw.py:307-321)
  if (cfg.do_f3d && !cfg.hydrostatic) {
    set_last_error_msg("fv3b_d_sw: do_f3d is not implemented");
    return FV3B_ERR_UNSUPPORTED;
  }
  FV3B_CHECK(launch_box(Box{0, full, 0, full, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    W3(tmp_vort, i, j) = F3(tmp_wk, i, j) + F2(g.f0, i, j);
  }));
  FV3B_CHECK(transport(tmp_vort, tmp_fx, tmp_fy, cfg.hord_vt, nullptr, nullptr, nullptr, nullptr, 0));
  // u_and_v_from_ke (d_sw.py:278-299)
  FV3B_CHECK(launch_box(Box{s, e + 2, js, je + 2, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    if (i <= e) W3(u, i, j) = F3(u, i, j) * F2(g.dx, i, j) + F3(tmp_ke, i, j) - F3(tmp_ke, i + 1, j) + F3(tmp_fy, i, j);
    if (j <= je) W3(v, i, j) = F3(v, i, j) * F2(g.dy, i, j) + F3(tmp_ke, i, j) - F3(tmp_ke, i, j + 1) - F3(tmp_fx, i, j);
  }));
  FV3B_CHECK(delnflux_nosg(d, g, tmp_wk, tmp_ut, tmp_vt, nosg_v, tmp_vort, deln_alt, false, sp.nmax_v, st));
  // heat_source_from_vorticity_damping (d_sw.py:368-438)
  {
    const bool add_total = cfg.d_con > DCON_THRESHOLD || cfg.do_skeb;
    FV3B_CHECK(launch_box(Box{s, e + 2, js, je + 2, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
      PT_SETUP(d, t, k);
      real kf = col_d_con[k];
      if (kf > DCON_THRESHOLD) {
        auto ubt = [&](int ii, int jj) { return (F3(vort_x_delta, ii, jj) + F3(tmp_vt, ii, jj)) * F2(g.rdx, ii, jj); };
        auto vbt = [&](int ii, int jj) { return (F3(vort_y_delta, ii, jj) - F3(tmp_ut, ii, jj)) * F2(g.rdy, ii, jj); };
        auto fyf = [&](int ii, int jj) { return F3(u, ii, jj) * F2(g.rdx, ii, jj); };
        auto fxf = [&](int ii, int jj) { return F3(v, ii, jj) * F2(g.rdy, ii, jj); };
        real ub0 = ubt(i, j), ub1 = ubt(i, j + 1), vb0 = vbt(i, j), vb1 = vbt(i + 1, j);
        real fy0 = fyf(i, j), fy1 = fyf(i, j + 1), fx0 = fxf(i, j), fx1 = fxf(i + 1, j);
        real gy0 = fy0 * ub0, gy1 = fy1 * ub1, gx0 = fx0 * vb0, gx1 = fx1 * vb1;
        real u2 = fy0 + fy1, du2 = ub0 + ub1, v2 = fx0 + fx1, dv2 = vb0 + vb1;
        real dampterm = F2(g.rsin2, i, j) * ((ub0 * ub0 + ub1 * ub1 + vb0 * vb0 + vb1 * vb1) +
                                               RC(2.0) * (gy0 + gy1 + gx0 + gx1) -
                                               F2(g.cosa_s, i, j) * (u2 * dv2 + v2 * du2 + du2 * dv2));
        real hs = F3(delp, i, j) * (F3(tmp_heat_s, i, j) - RC(0.25) * kf * dampterm);
        W3(tmp_heat_s, i, j) = hs;
        if (add_total && i <= e && j <= je) W3(heat_source, i, j) = F3(heat_source, i, j) + hs;
      } else if (add_total && i <= e && j <= je) {
        W3(heat_source, i, j) = F3(heat_source, i, j) + F3(tmp_heat_s, i, j);
      }
    }));
  }
  // update_u_and_v (d_sw.py:441-465)
  FV3B_CHECK(launch_box(Box{s, e + 2, js, je + 2, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    if (!(col_damp_vt[k] > RC(1e-5))) return;
    if (i <= e) W3(u, i, j) = F3(u, i, j) + F3(tmp_vt, i, j);
    if (j <= je) W3(v, i, j) = F3(v, i, j) - F3(tmp_ut, i, j);
  }));
  return FV3B_OK;
}

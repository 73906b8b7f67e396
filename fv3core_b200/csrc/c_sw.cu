// C-grid shallow water (c_sw) with the D->A->C wind interpolation (d2a2c).
//
// Each launch below is one pass over a box of (tile, i, j, k) points; the
// sequence follows the data dependencies of the reference stencils
// (fv3core/stencils/c_sw.py, d2a2c_vect.py): a pass that reads a value at a
// horizontal offset starts only after the pass that wrote it.  Point work is
// written with the reference's statement order so that FP64 results agree
// to rounding.
#include "corners.cuh"
#include "ctx.cuh"
#include "stencil.cuh"

using namespace fv3b;

namespace {

constexpr real C1 = -RC(2.0) / RC(14.0), C2 = RC(11.0) / RC(14.0), C3 = RC(5.0) / RC(14.0);
constexpr real A1 = RC(9.0) / RC(16.0), A2 = -RC(1.0) / RC(16.0);
constexpr real BIG = RC(1e30);

// The only points corner_x can fill: i in {s-3, s-2, s-1, e+1, e+2, e+3}
// (x = 0..5) and j in {js-1, je+1} (y = 0, 1); corner_y swaps the roles.
// The corner passes launch over these 12 points per level and tile.
__device__ __forceinline__ int corner_i6(const Dims& d, int x) { return x < 3 ? d.isc - 3 + x : d.iec + x - 2; }
__device__ __forceinline__ int corner_j6(const Dims& d, int x) { return x < 3 ? d.jsc - 3 + x : d.jec + x - 2; }

}  // namespace

extern "C" int fv3b_c_sw(fv3b_ctx* ctx, real* delp, real* pt, const real* u, const real* v, real* w,
                         real* uc, real* vc, real* ua, real* va, real* ut, real* vt, real* divgd,
                         real* omga, double dt2_in, int nord, real* delpc, real* ptc, void* stream) {
  FV3B_TILES(ctx);
  // the build's precision inside the kernels (the same value in FP64 builds)
  const real dt2 = static_cast<real>(dt2_in);
  FV3B_REQUIRE(ctx && delp && pt && u && v && w && uc && vc && ua && va && ut && vt && divgd && omga && delpc && ptc,
               "fv3b_c_sw: null argument");
  const Dims d = ctx->d;
  const fv3b_metrics g = ctx->m;
  cudaStream_t st = (cudaStream_t)stream;
  real* utmp = ctx->ws[0];
  real* vtmp = ctx->ws[1];
  real* tfx = ctx->ws[2];
  real* tfx1 = ctx->ws[3];
  real* tfx2 = ctx->ws[4];
  real* tke = ctx->ws[5];
  real* tvort = ctx->ws[6];
  const int nz = d.nz;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  const int full = d.ni - 1;  // halo domain is [0, n+2h)
  int npt = 4;
  if (npt > d.n - 1) npt = 0;
  const int lo = npt + 2, hi = e + 1 - npt;  // lagrange p1 box (inclusive)
  const int off = npt == 0 ? -1 : 3;

  // ---- d2a2c: utmp/vtmp (set_tmps, lagrange p1, avg_box) and ua/va
  // (d2a2c_vect.py:18-21, 141-182, 248-260)
  FV3B_CHECK(launch_box(Box{0, full, 0, full, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    real ut_ = BIG, vt_ = BIG;
    if (i >= lo && i <= hi && j >= lo && j <= hi) {
      ut_ = A2 * (F3(u, i, j - 1) + F3(u, i, j + 2)) + A1 * (F3(u, i, j) + F3(u, i, j + 1));
      vt_ = A2 * (F3(v, i - 1, j) + F3(v, i + 2, j)) + A1 * (F3(v, i, j) + F3(v, i + 1, j));
    }
    bool avg = (j < js + off) || (j >= je - off + 1) || (i < s + off) || (i >= e - off + 1);
    if (avg) {
      ut_ = RC(0.5) * (F3(u, i, j) + F3(u, i, j + 1));
      vt_ = RC(0.5) * (F3(v, i, j) + F3(v, i + 1, j));
    }
    W3(utmp, i, j) = ut_;
    W3(vtmp, i, j) = vt_;
    // initialize_delpc_ptc (c_sw.py:372-376)
    W3(delpc, i, j) = RC(0.0);
    W3(ptc, i, j) = RC(0.0);
    if (i >= s - 2 && i < e + 3 && j >= js - 2 && j < je + 3) {
      real cs = F2(g.cosa_s, i, j), r2 = F2(g.rsin2, i, j);
      W3(ua, i, j) = (ut_ - vt_ * cs) * r2;
      W3(va, i, j) = (vt_ - ut_ * cs) * r2;
    }
  }));
  // fill_corners_x on utmp (3 cells, from vtmp) and ua (2 cells, from va)
  FV3B_CHECK(launch_box(Box{0, 6, 0, 2, 0, nz}, st, [=] __device__(int t, int x, int y, int k) {
    PT_SETUP(d, t, k);
    const int i = corner_i6(d, x), j = y == 0 ? js - 1 : je + 1;
    CornerRule r;
    if (corner_x(d, i, j, true, -RC(1.0), RC(1.0), RC(1.0), -RC(1.0), r)) W3(utmp, i, j) = r.mult * F3(vtmp, i + r.di, j + r.dj);
    if (corner_x(d, i, j, false, -RC(1.0), RC(1.0), RC(1.0), -RC(1.0), r)) W3(ua, i, j) = r.mult * F3(va, i + r.di, j + r.dj);
  }));
  // ut_main + east_west_edges (d2a2c_vect.py:45-93, 263-273); the ut_main
  // columns in warps of their own
  FV3B_CHECK(launch_box_split(Box{s - 3, e + 4, js - 1, je + 2, 0, nz}, s + 2, e, st,
                              [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    real cu = F2(g.cosa_u, i, j), ru = F2(g.rsin_u, i, j);
    if (i >= s + 2 && i <= e - 1) {
      real ucv = A2 * (F3(utmp, i - 2, j) + F3(utmp, i + 1, j)) + A1 * (F3(utmp, i - 1, j) + F3(utmp, i, j));
      W3(uc, i, j) = ucv;
      W3(ut, i, j) = (ucv - F3(v, i, j) * cu) * ru;
    } else if (i == s - 1 || i == e) {
      real ucv = C1 * F3(utmp, i - 2, j) + C2 * F3(utmp, i - 1, j) + C3 * F3(utmp, i, j);
      W3(uc, i, j) = ucv;
      W3(ut, i, j) = (ucv - F3(v, i, j) * cu) * ru;
    } else if (i == s || i == e + 1) {
      real t1 = F2(g.dxa, i - 2, j) + F2(g.dxa, i - 1, j);
      real t2 = F2(g.dxa, i, j) + F2(g.dxa, i + 1, j);
      real n1 = (t1 + F2(g.dxa, i - 1, j)) * F3(ua, i - 1, j) - F2(g.dxa, i - 1, j) * F3(ua, i - 2, j);
      real n2 = (t1 + F2(g.dxa, i, j)) * F3(ua, i, j) - F2(g.dxa, i, j) * F3(ua, i + 1, j);
      real utc = RC(0.5) * (n1 / t1 + n2 / t2);
      W3(ut, i, j) = utc;
      W3(uc, i, j) = utc > 0 ? utc * F2(g.sin_sg3, i - 1, j) : utc * F2(g.sin_sg1, i, j);
    } else if (i == s + 1 || i == e + 2) {
      real ucv = C1 * F3(utmp, i + 1, j) + C2 * F3(utmp, i, j) + C3 * F3(utmp, i - 1, j);
      W3(uc, i, j) = ucv;
      W3(ut, i, j) = (ucv - F3(v, i, j) * cu) * ru;
    }
  }));
  // fill_corners_y on vtmp (3 cells, from utmp) and va (2 cells, from ua)
  FV3B_CHECK(launch_box(Box{0, 6, 0, 2, 0, nz}, st, [=] __device__(int t, int x, int y, int k) {
    PT_SETUP(d, t, k);
    const int i = y == 0 ? s - 1 : e + 1, j = corner_j6(d, x);
    CornerRule r;
    if (corner_y(d, i, j, true, -RC(1.0), RC(1.0), RC(1.0), -RC(1.0), r)) W3(vtmp, i, j) = r.mult * F3(utmp, i + r.di, j + r.dj);
    if (corner_y(d, i, j, false, -RC(1.0), RC(1.0), RC(1.0), -RC(1.0), r)) W3(va, i, j) = r.mult * F3(ua, i + r.di, j + r.dj);
  }));
  // north_south_edges + vt_main (d2a2c_vect.py:96-138, 276-286)
  FV3B_CHECK(launch_box(Box{s - 1, e + 2, js - 1, je + 3, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    real cv = F2(g.cosa_v, i, j), rv = F2(g.rsin_v, i, j);
    real vcv;
    if (j == js - 1 || j == je) {
      vcv = C1 * F3(vtmp, i, j - 2) + C2 * F3(vtmp, i, j - 1) + C3 * F3(vtmp, i, j);
    } else if (j == js || j == je + 1) {
      real t1 = F2(g.dya, i, j - 2) + F2(g.dya, i, j - 1);
      real t2 = F2(g.dya, i, j) + F2(g.dya, i, j + 1);
      real n1 = (t1 + F2(g.dya, i, j - 1)) * F3(va, i, j - 1) - F2(g.dya, i, j - 1) * F3(va, i, j - 2);
      real n2 = (t1 + F2(g.dya, i, j)) * F3(va, i, j) - F2(g.dya, i, j) * F3(va, i, j + 1);
      real vtc = RC(0.5) * (n1 / t1 + n2 / t2);
      W3(vt, i, j) = vtc;
      W3(vc, i, j) = vtc > 0 ? vtc * F2(g.sin_sg4, i, j - 1) : vtc * F2(g.sin_sg2, i, j);
      return;
    } else if (j == js + 1 || j == je + 2) {
      vcv = C1 * F3(vtmp, i, j + 1) + C2 * F3(vtmp, i, j) + C3 * F3(vtmp, i, j - 1);
    } else {
      vcv = A2 * (F3(vtmp, i, j - 2) + F3(vtmp, i, j + 1)) + A1 * (F3(vtmp, i, j - 1) + F3(vtmp, i, j));
    }
    W3(vc, i, j) = vcv;
    W3(vt, i, j) = (vcv - F3(u, i, j) * cv) * rv;
  }));

  // ---- divergence_corner (c_sw.py:172-287), cell corners of the compute domain
  if (nord > 0) {
    FV3B_CHECK(launch_box(Box{s, e + 2, js, je + 2, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
      PT_SETUP(d, t, k);
      auto ufv = [&](int ii, int jj) {
        return (F3(u, ii, jj) - RC(0.25) * (F3(va, ii, jj - 1) + F3(va, ii, jj)) *
                                    (F2(g.cos_sg4, ii, jj - 1) + F2(g.cos_sg2, ii, jj))) *
               F2(g.dyc, ii, jj) * RC(0.5) * (F2(g.sin_sg4, ii, jj - 1) + F2(g.sin_sg2, ii, jj));
      };
      auto vfv = [&](int ii, int jj) {
        return (F3(v, ii, jj) - RC(0.25) * (F3(ua, ii - 1, jj) + F3(ua, ii, jj)) *
                                    (F2(g.cos_sg3, ii - 1, jj) + F2(g.cos_sg1, ii, jj))) *
               F2(g.dxc, ii, jj) * RC(0.5) * (F2(g.sin_sg3, ii - 1, jj) + F2(g.sin_sg1, ii, jj));
      };
      real rac = F2(g.rarea_c, i, j);
      real uf = ufv(i, j), vf = vfv(i, j);
      real dd;
      bool ew = (i == s || i == e + 1), ns = (j == js || j == je + 1);
      real vf0 = F3(v, i, j) * F2(g.dxc, i, j) * RC(0.5) * (F2(g.sin_sg3, i - 1, j) + F2(g.sin_sg1, i, j));
      real vf1 = F3(v, i, j - 1) * F2(g.dxc, i, j - 1) * RC(0.5) * (F2(g.sin_sg3, i - 1, j - 1) + F2(g.sin_sg1, i, j - 1));
      real uf0 = F3(u, i, j) * F2(g.dyc, i, j) * RC(0.5) * (F2(g.sin_sg4, i, j - 1) + F2(g.sin_sg2, i, j));
      real uf1b = F3(u, i - 1, j) * F2(g.dyc, i - 1, j) * RC(0.5) * (F2(g.sin_sg4, i - 1, j - 1) + F2(g.sin_sg2, i - 1, j));
      if (ns && ew) {
        if (j == js)
          dd = (-vf0 + uf1b - uf0) * rac;
        else
          dd = (vf1 + uf1b - uf0) * rac;
      } else if (ns) {
        real vf1b = (F3(v, i, j - 1) - RC(0.25) * (F3(ua, i - 1, j - 1) + F3(ua, i, j - 1)) *
                                             (F2(g.cos_sg3, i - 1, j - 1) + F2(g.cos_sg1, i, j - 1))) *
                      F2(g.dxc, i, j - 1) * RC(0.5) * (F2(g.sin_sg3, i - 1, j - 1) + F2(g.sin_sg1, i, j - 1));
        dd = (vf1b - vf + uf1b - uf0) * rac;
      } else if (ew) {
        real uf1 = (F3(u, i - 1, j) - RC(0.25) * (F3(va, i - 1, j - 1) + F3(va, i - 1, j)) *
                                            (F2(g.cos_sg4, i - 1, j - 1) + F2(g.cos_sg2, i - 1, j))) *
                     F2(g.dyc, i - 1, j) * RC(0.5) * (F2(g.sin_sg4, i - 1, j - 1) + F2(g.sin_sg2, i - 1, j));
        dd = (vf1 - vf0 + uf1 - uf) * rac;
      } else {
        dd = (vfv(i, j - 1) - vf + ufv(i - 1, j) - uf) * rac;
      }
      W3(divgd, i, j) = dd;
    }));
  }
  // ---- geoadjust_ut / vt (c_sw.py:20-43) and fill_corners_x on delp, pt, w
  FV3B_CHECK(launch_box(Box{s - 1, e + 3, js - 1, je + 3, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    if (j < je + 2) {
      real x = F3(ut, i, j);
      W3(ut, i, j) = x > 0 ? dt2 * x * F2(g.dy, i, j) * F2(g.sin_sg3, i - 1, j) : dt2 * x * F2(g.dy, i, j) * F2(g.sin_sg1, i, j);
    }
    if (i < e + 2) {
      real y = F3(vt, i, j);
      W3(vt, i, j) = y > 0 ? dt2 * y * F2(g.dx, i, j) * F2(g.sin_sg4, i, j - 1) : dt2 * y * F2(g.dx, i, j) * F2(g.sin_sg2, i, j);
    }
  }));
  FV3B_CHECK(launch_box(Box{0, 6, 0, 2, 0, nz}, st, [=] __device__(int t, int x, int y, int k) {
    PT_SETUP(d, t, k);
    const int i = corner_i6(d, x), j = y == 0 ? js - 1 : je + 1;
    CornerRule r;
    if (corner_x(d, i, j, false, RC(1.0), RC(1.0), RC(1.0), RC(1.0), r)) {
      real a = F3(delp, i + r.di, j + r.dj), b = F3(pt, i + r.di, j + r.dj), c = F3(w, i + r.di, j + r.dj);
      W3(delp, i, j) = a;
      W3(pt, i, j) = b;
      W3(w, i, j) = c;
    }
  }));
  // compute_nonhydro_fluxes_x (c_sw.py:67-82)
  FV3B_CHECK(launch_box(Box{s - 1, e + 3, js - 1, je + 2, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    real utc = F3(ut, i, j);
    bool p = utc > RC(0.0);
    int ii = p ? i - 1 : i;
    real fx1 = utc * F3(delp, ii, j);
    W3(tfx1, i, j) = fx1;
    W3(tfx, i, j) = fx1 * F3(pt, ii, j);
    W3(tfx2, i, j) = fx1 * F3(w, ii, j);
  }));
  // fill_corners_y on delp, pt, w
  FV3B_CHECK(launch_box(Box{0, 6, 0, 2, 0, nz}, st, [=] __device__(int t, int x, int y, int k) {
    PT_SETUP(d, t, k);
    const int i = y == 0 ? s - 1 : e + 1, j = corner_j6(d, x);
    CornerRule r;
    if (corner_y(d, i, j, false, RC(1.0), RC(1.0), RC(1.0), RC(1.0), r)) {
      real a = F3(delp, i + r.di, j + r.dj), b = F3(pt, i + r.di, j + r.dj), c = F3(w, i + r.di, j + r.dj);
      W3(delp, i, j) = a;
      W3(pt, i, j) = b;
      W3(w, i, j) = c;
    }
  }));
  // transportdelp_update_vorticity_and_kineticenergy (c_sw.py:85-169)
  FV3B_CHECK(launch_box(Box{s - 1, e + 2, js - 1, je + 2, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    auto fy = [&](int jj, real& f1, real& f, real& f2) {
      real vtc = F3(vt, i, jj);
      int j2 = vtc > RC(0.0) ? jj - 1 : jj;
      f1 = vtc * F3(delp, i, j2);
      f = f1 * F3(pt, i, j2);
      f2 = f1 * F3(w, i, j2);
    };
    real fy1a, fya, fy2a, fy1b, fyb, fy2b;
    fy(j, fy1a, fya, fy2a);
    fy(j + 1, fy1b, fyb, fy2b);
    real ra = F2(g.rarea, i, j);
    real dp = F3(delp, i, j);
    real dpc = dp + (F3(tfx1, i, j) - F3(tfx1, i + 1, j) + fy1a - fy1b) * ra;
    W3(delpc, i, j) = dpc;
    W3(ptc, i, j) = (F3(pt, i, j) * dp + (F3(tfx, i, j) - F3(tfx, i + 1, j) + fya - fyb) * ra) / dpc;
    W3(omga, i, j) = (F3(w, i, j) * dp + (F3(tfx2, i, j) - F3(tfx2, i + 1, j) + fy2a - fy2b) * ra) / dpc;
    real uav = F3(ua, i, j), vav = F3(va, i, j);
    real ke = uav > RC(0.0) ? F3(uc, i, j) : F3(uc, i + 1, j);
    real vort = vav > RC(0.0) ? F3(vc, i, j) : F3(vc, i, j + 1);
    if ((j == js - 1 || j == je) && vav <= RC(0.0)) vort = vort * F2(g.sin_sg4, i, j) + F3(u, i, j + 1) * F2(g.cos_sg4, i, j);
    if ((j == js || j == je + 1) && vav > RC(0.0)) vort = vort * F2(g.sin_sg2, i, j) + F3(u, i, j) * F2(g.cos_sg2, i, j);
    if ((i == e || i == s - 1) && uav <= RC(0.0)) ke = ke * F2(g.sin_sg3, i, j) + F3(v, i + 1, j) * F2(g.cos_sg3, i, j);
    if ((i == e + 1 || i == s) && uav > RC(0.0)) ke = ke * F2(g.sin_sg1, i, j) + F3(v, i, j) * F2(g.cos_sg1, i, j);
    W3(tke, i, j) = RC(0.5) * dt2 * (uav * ke + vav * vort);
    W3(tvort, i, j) = vort;
  }));
  // circulation_cgrid + absolute_vorticity (c_sw.py:46-48, 292-322)
  FV3B_CHECK(launch_box(Box{s, e + 2, js, je + 2, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    real fx = F2(g.dxc, i, j) * F3(uc, i, j);
    real fy = F2(g.dyc, i, j) * F3(vc, i, j);
    real fx1 = F2(g.dxc, i, j - 1) * F3(uc, i, j - 1);
    real fy1 = F2(g.dyc, i - 1, j) * F3(vc, i - 1, j);
    real vcv;
    bool cj = (j == js || j == je + 1);
    if (i == s && cj)
      vcv = fx1 - fx + fy;
    else if (i == e + 1 && cj)
      vcv = fx1 - fx - fy1;
    else
      vcv = fx1 - fx - fy1 + fy;
    W3(tvort, i, j) = F2(g.fC, i, j) + F2(g.rarea_c, i, j) * vcv;
  }));
  // update_y_velocity (vc) and update_x_velocity (uc) (c_sw.py:325-369)
  FV3B_CHECK(launch_box(Box{s, e + 2, js, je + 2, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    if (i <= e) {
      real vcv = F3(vc, i, j);
      real tf = (j == js || j == je + 1) ? dt2 * F3(u, i, j)
                                           : dt2 * (F3(u, i, j) - vcv * F2(g.cosa_v, i, j)) / F2(g.sina_v, i, j);
      real flux = tf > RC(0.0) ? F3(tvort, i, j) : F3(tvort, i + 1, j);
      W3(vc, i, j) = vcv - tf * flux + F2(g.rdyc, i, j) * (F3(tke, i, j - 1) - F3(tke, i, j));
    }
    if (j <= je) {
      real ucv = F3(uc, i, j);
      real tf = (i == s || i == e + 1) ? dt2 * F3(v, i, j)
                                         : dt2 * (F3(v, i, j) - ucv * F2(g.cosa_u, i, j)) / F2(g.sina_u, i, j);
      real flux = tf > RC(0.0) ? F3(tvort, i, j) : F3(tvort, i, j + 1);
      W3(uc, i, j) = ucv + tf * flux + F2(g.rdxc, i, j) * (F3(tke, i - 1, j) - F3(tke, i, j));
    }
  }));
  return FV3B_OK;
}

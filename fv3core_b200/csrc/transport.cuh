// Piecewise-parabolic fluxes, the 2-D finite-volume transport and del-n
// flux damping, shared by the D-grid stages.
//
// References: fv3core/stencils/xppm.py, yppm.py, ppm.py (PPM flux),
// xtp_u.py / ytp_v.py (wind self-advection), fvtp2d.py (Lin-Rood 2-D
// transport), delnflux.py (del-n damping).  The y-direction code is the
// x-direction code with the roles of i and j exchanged (an AXIS template
// parameter); the statement order of the reference is kept so that FP64
// results agree to rounding.
#pragma once
#include <algorithm>
#include <map>
#include <mutex>

#include "corners.cuh"
#include "ctx.cuh"
#include "stencil.cuh"

namespace fv3b {

// ppm.py:8-20
constexpr real PPM_C1 = -RC(2.0) / RC(14.0), PPM_C2 = RC(11.0) / RC(14.0), PPM_C3 = RC(5.0) / RC(14.0);
constexpr real PPM_P1 = RC(7.0) / RC(12.0), PPM_P2 = -RC(1.0) / RC(12.0);

// Accessor of a 3-D field along one axis through point (i, j) of level k:
// at(o) = f[i + o, j] (AXIS 0) or f[i, j + o] (AXIS 1).
template <int AXIS>
struct Line3 {
  const real* p;
  idx_t base;  // index of (i, j, k)
  idx_t step;  // 1 or sj
  __device__ __forceinline__ real operator()(int o) const { return p[base + o * step]; }
};

template <int AXIS>
struct Line2 {
  const real* p;
  idx_t base;
  idx_t step;
  __device__ __forceinline__ real operator()(int o) const { return p[base + o * step]; }
};

template <int AXIS>
__device__ __forceinline__ Line3<AXIS> line3(const Dims& d, const real* p, int t, int i, int j, int k) {
  return Line3<AXIS>{p, idx3(d, t, i, j, k), AXIS == 0 ? idx_t(1) : d.sj};
}
template <int AXIS>
__device__ __forceinline__ Line2<AXIS> line2(const Dims& d, const real* p, int t, int i, int j) {
  return Line2<AXIS>{p, idx2(d, t, i, j), AXIS == 0 ? idx_t(1) : (idx_t)d.ni};
}

// The reference's y-corner-copied copy of q (CopyCornersXY, corners.py:64-117)
// read on the fly from q: a point of a cube-corner block takes its copy
// source.  Sources never lie in a corner block, so this equals the copy
// whether or not q's own corners already hold their x copies.
__device__ __forceinline__ real qy_at(const Dims& d, const real* q, int t, int i, int j, int k) {
  int si, sj;
  if (copy_corner_y(d, i, j, si, sj)) return q[idx3(d, t, si, sj, k)];
  return q[idx3(d, t, i, j, k)];
}
struct LineQY {
  Dims d;
  const real* q;
  int t, i, j, k;
  __device__ __forceinline__ real operator()(int o) const { return qy_at(d, q, t, i, j + o, k); }
};

// compute_al (xppm.py:148-181) for the cell at offset o of the line; pos is
// the absolute index (along AXIS) of offset 0, s/e the compute bounds.
template <typename Q, typename A>
__device__ __forceinline__ real ppm_al(const Q& q, const A& dxa, int o, int pos, int s, int e) {
  int ii = pos + o;
  if (ii == s + 1 || ii == e + 2) return PPM_C3 * q(o - 1) + PPM_C2 * q(o) + PPM_C1 * q(o + 1);
  if (ii == s || ii == e + 1)
    return RC(0.5) * (((RC(2.0) * dxa(o - 1) + dxa(o - 2)) * q(o - 1) - dxa(o - 1) * q(o - 2)) / (dxa(o - 2) + dxa(o - 1)) +
                  ((RC(2.0) * dxa(o) + dxa(o + 1)) * q(o) - dxa(o) * q(o + 1)) / (dxa(o) + dxa(o + 1)));
  if (ii == s - 1 || ii == e) return PPM_C1 * q(o - 2) + PPM_C2 * q(o - 1) + PPM_C3 * q(o);
  return PPM_P1 * (q(o - 1) + q(o)) + PPM_P2 * (q(o - 2) + q(o + 1));
}

// The three interface values around cell offset 0 (offsets -1, 0, 1) of a
// line.  Away from the tile edges (no offset on an edge row) the six cells
// are loaded once and the interior formula is used; otherwise each value
// takes ppm_al's edge rules.  Same operations in the same order either way.
// The edge-row case (the rows next to tile edges).  Kept inline: an
// out-of-line version measured slower.
template <typename Q, typename A>
__device__ __forceinline__ void ppm_al3_edges(const Q q, const A dxa, int pos, int s, int e, real* al) {
  al[0] = ppm_al(q, dxa, -1, pos, s, e);
  al[1] = ppm_al(q, dxa, 0, pos, s, e);
  al[2] = ppm_al(q, dxa, 1, pos, s, e);
}

template <typename Q, typename A>
__device__ __forceinline__ void ppm_al3(const Q& q, const A& dxa, int pos, int s, int e, real& alm, real& al0,
                                        real& alp) {
  if (pos - 1 >= s + 2 && pos + 1 <= e - 1) {
    const real q_3 = q(-3), q_2 = q(-2), q_1 = q(-1), q0 = q(0), q1 = q(1), q2 = q(2);
    alm = PPM_P1 * (q_2 + q_1) + PPM_P2 * (q_3 + q0);
    al0 = PPM_P1 * (q_1 + q0) + PPM_P2 * (q_2 + q1);
    alp = PPM_P1 * (q0 + q1) + PPM_P2 * (q_1 + q2);
    return;
  }
  real al[3];
  ppm_al3_edges(q, dxa, pos, s, e, al);
  alm = al[0];
  al0 = al[1];
  alp = al[2];
}

__device__ __forceinline__ bool ppm_smooth(real bl, real b0, real br, int mord) {
  if (mord == 5) return bl * br < 0;
  return (RC(3.0) * fabs(b0)) < fabs(bl - br);
}

// Mean of q advected through the interface at offset 0 (between cells -1
// and 0) for Courant number c: get_flux (xppm.py:65-72) with fx1_fn,
// get_advection_mask and apply_flux (xppm.py:19-61).
template <typename Q, typename A>
__device__ __forceinline__ real ppm_flux(const Q& q, const A& dxa, real c, int pos, int s, int e, int mord) {
  real alm, al0, alp;
  ppm_al3(q, dxa, pos, s, e, alm, al0, alp);
  real qm = q(-1), q0 = q(0);
  real blm = alm - qm, brm = al0 - qm, b0m = blm + brm;
  real bl0 = al0 - q0, br0 = alp - q0, b00 = bl0 + br0;
  real mask = (ppm_smooth(blm, b0m, brm, mord) || ppm_smooth(bl0, b00, br0, mord)) ? RC(1.0) : RC(0.0);
  real fx1 = c > RC(0.0) ? (RC(1.0) - c) * (brm - c * b0m) : (RC(1.0) + c) * (bl0 + c * b00);
  return c > RC(0.0) ? qm + fx1 * mask : q0 + fx1 * mask;
}

// ------------------------------------------------------------------ ord 8
// The ord-8 limiter of tracer transport (hord = 8): xppm.py:85-266 and
// ppm.py:22-36.  ppm.py:16-18
constexpr real PPM_S11 = RC(11.0) / RC(14.0), PPM_S14 = RC(4.0) / RC(7.0), PPM_S15 = RC(3.0) / RC(14.0);

// basic_operations.sign (basic_operations.py:34-40): |a|, negative unless b > 0
__device__ __forceinline__ real sign_of(real a, real b) { return b > RC(0.0) ? fabs(a) : -fabs(a); }

// dm_iord8plus (xppm.py:85-90) of the cell at offset o; the dm_left /
// dm_right temporaries of bl_br_edges are this function of the neighbour
template <typename Q>
__device__ __forceinline__ real dm_ord8(const Q& q, int o) {
  const real qm = q(o - 1), q0 = q(o), qp = q(o + 1);
  const real xt = RC(0.25) * (qp - qm);
  const real dqr = fmax(fmax(q0, qm), qp) - q0;
  const real dql = q0 - fmin(fmin(q0, qm), qp);
  return sign_of(fmin(fmin(fabs(xt), dqr), dql), xt);
}

// al_iord8plus (xppm.py:93-95): interface value left of cell o
template <typename Q>
__device__ __forceinline__ real al_ord8(const Q& q, int o) {
  return RC(0.5) * (q(o - 1) + q(o)) + (RC(1.0) / RC(3.0)) * (dm_ord8(q, o - 1) - dm_ord8(q, o));
}

// xt_dxa_edge_0 / xt_dxa_edge_1 with xt_minmax (xppm.py:105-145), cell o
template <typename Q, typename A>
__device__ __forceinline__ real xt_dxa_edge0(const Q& q, const A& dxa, int o) {
  const real qm = q(o - 1), q0 = q(o), q1 = q(o + 1), q2 = q(o + 2);
  const real d0 = dxa(o), dm = dxa(o - 1), d1 = dxa(o + 1), d2 = dxa(o + 2);
  const real xt = RC(0.5) * (((RC(2.0) * d0 + dm) * q0 - d0 * qm) / (dm + d0) +
                             ((RC(2.0) * d1 + d2) * q1 - d1 * q2) / (d1 + d2));
  const real minq = fmin(fmin(fmin(qm, q0), q1), q2);
  const real maxq = fmax(fmax(fmax(qm, q0), q1), q2);
  return fmin(fmax(xt, minq), maxq);
}
template <typename Q, typename A>
__device__ __forceinline__ real xt_dxa_edge1(const Q& q, const A& dxa, int o) {
  const real qm2 = q(o - 2), qm = q(o - 1), q0 = q(o), q1 = q(o + 1);
  const real d0 = dxa(o), dm = dxa(o - 1), dm2 = dxa(o - 2), d1 = dxa(o + 1);
  const real xt = RC(0.5) * (((RC(2.0) * dm + dm2) * qm - dm * qm2) / (dm2 + dm) +
                             ((RC(2.0) * d0 + d1) * q0 - d0 * q1) / (d0 + d1));
  const real minq = fmin(fmin(fmin(qm2, qm), q0), q1);
  const real maxq = fmax(fmax(fmax(qm2, qm), q0), q1);
  return fmin(fmax(xt, minq), maxq);
}

// Edge perturbations (bl, br) of the cell at offset o, absolute index p:
// compute_blbr_ord8plus (xppm.py:250-266) = blbr_iord8 (98-102) away from
// the tile edges; bl_br_edges (185-246) and the standard constraint
// (pert_ppm_standard_constraint_fcn, ppm.py:22-36) on the three cells at
// each edge.  The edge regions are tested last first, so that where two of
// them meet the later one wins, as the reference's sequential regions do.
template <typename Q, typename A>
__device__ __forceinline__ void blbr_ord8(const Q& q, const A& dxa, int o, int p, int s, int e, real& bl,
                                          real& br) {
  const real q0 = q(o);
  const real dm0 = dm_ord8(q, o);
  const bool near_s = p >= s - 1 && p <= s + 1, near_e = p >= e - 1 && p <= e + 1;
  if (!near_s && !near_e) {
    const real xt = RC(2.0) * dm0;
    bl = -RC(1.0) * sign_of(fmin(fabs(xt), fabs(al_ord8(q, o) - q0)), xt);
    br = sign_of(fmin(fabs(xt), fabs(al_ord8(q, o + 1) - q0)), xt);
    return;
  }
  real xbl, xbr;
  if (p == e + 1) {
    xbl = xt_dxa_edge1(q, dxa, o);
    xbr = PPM_S11 * (q(o + 1) - q0) - PPM_S14 * dm_ord8(q, o + 1) + q0;
  } else if (p == e) {
    xbl = PPM_S15 * q0 + PPM_S11 * q(o - 1) + PPM_S14 * dm_ord8(q, o - 1);
    xbr = xt_dxa_edge0(q, dxa, o);
  } else if (p == e - 1) {
    xbl = al_ord8(q, o);
    xbr = PPM_S15 * q(o + 1) + PPM_S11 * q0 + PPM_S14 * dm0;
  } else if (p == s + 1) {
    xbl = PPM_S15 * q(o - 1) + PPM_S11 * q0 - PPM_S14 * dm0;
    xbr = al_ord8(q, o + 1);
  } else if (p == s) {
    xbl = xt_dxa_edge1(q, dxa, o);
    xbr = PPM_S15 * q0 + PPM_S11 * q(o + 1) - PPM_S14 * dm_ord8(q, o + 1);
  } else {  // p == s - 1
    xbl = PPM_S14 * dm_ord8(q, o - 1) + PPM_S11 * (q(o - 1) - q0) + q0;
    xbr = xt_dxa_edge0(q, dxa, o);
  }
  real l = xbl - q0, r = xbr - q0;
  if (l * r < RC(0.0)) {
    const real da1 = l - r;
    const real da2 = da1 * da1;
    const real a6da = RC(3.0) * (l + r) * da1;
    if (a6da < -da2)
      r = -RC(2.0) * l;
    else if (a6da > da2)
      l = -RC(2.0) * r;
  } else {
    l = RC(0.0);
    r = RC(0.0);
  }
  bl = l;
  br = r;
}

// get_flux_ord8plus (xppm.py:75-82): mean of q advected through the
// interface at offset 0 with the ord-8 perturbations of the upwind cell
template <typename Q, typename A>
__device__ __forceinline__ real ppm_flux8(const Q& q, const A& dxa, real c, int pos, int s, int e) {
  real bl, br;
  if (c > RC(0.0)) {
    blbr_ord8(q, dxa, -1, pos - 1, s, e, bl, br);
    const real b0 = bl + br;
    return q(-1) + (RC(1.0) - c) * (br - c * b0);
  }
  blbr_ord8(q, dxa, 0, pos, s, e, bl, br);
  const real b0 = bl + br;
  return q(0) + (RC(1.0) + c) * (bl + c * b0);
}

// The PPM flux of order ORD8 ? 8 : mord.
template <bool ORD8, typename Q, typename A>
__device__ __forceinline__ real ppm_flux_ord(const Q& q, const A& dxa, real c, int pos, int s, int e, int mord) {
  if constexpr (ORD8) {
    return ppm_flux8(q, dxa, c, pos, s, e);
  } else {
    return ppm_flux(q, dxa, c, pos, s, e, mord);
  }
}

// Scratch and options of one FiniteVolumeTransport call.
struct FvTp2dArgs {
  const real* q_base;   // field, its cube-corner blocks holding their x copies
  const real* crx;
  const real* cry;
  const real* xfx;
  const real* yfx;
  const real* x_unit;   // x_mass_flux or xfx
  const real* y_unit;
  real* fx;
  real* fy;
  int hord;             // 5, 6, 7 (monotonic PPM) or 8 (ord-8 limiter)
  real* fx_mean;
  real* fy_mean;
  real* q_adv_x;
  real* q_adv_y;
};

// FiniteVolumeTransport.__call__ (fvtp2d.py:249-362) without the damping
// step; three passes: inner PPM, q_i/q_j, outer PPM + final fluxes.  Inner
// and outer PPM have the same order here (the reference's hord = 10, inner
// 8 and outer 10, fails its own compile_assert and is rejected).
template <bool ORD8>
inline cudaError_t fvtp2d_impl(const Dims d, const fv3b_metrics g, const FvTp2dArgs a, cudaStream_t st) {
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec, nk = d.nk;
  const int full = d.ni - 1;
  const int mord = a.hord < 0 ? -a.hord : a.hord;
  cudaError_t err;
  // inner PPM: fy_mean on [is-3, ie+4] x [js, je+1], fx_mean on [is, ie+1] x [js-3, je+4];
  // columns [is+3, ie-2] (both fluxes on the interior path) in warps of their own
  err = launch_box_split(Box{s - 3, e + 5, js - 3, je + 5, 0, nk}, s + 3, e - 1, st,
                         [=] __device__(int t, int i, int j, int k) {
    const idx_t o = idx3(d, t, i, j, k);
    if (j >= js && j < je + 2) {
      auto dya = line2<1>(d, g.dya, t, i, j);
      // the line reads rows j-3 .. j+2; a read can fall in a cube-corner
      // block only from a halo column within three rows of a tile edge
      if ((i >= s && i <= e) || (j >= js + 3 && j <= je - 2)) {  // plain reads
        a.fy_mean[o] = ppm_flux_ord<ORD8>(line3<1>(d, a.q_base, t, i, j, k), dya, a.cry[o], j, js, je, mord);
      } else {
        a.fy_mean[o] = ppm_flux_ord<ORD8>(LineQY{d, a.q_base, t, i, j, k}, dya, a.cry[o], j, js, je, mord);
      }
    }
    if (i >= s && i < e + 2) {
      a.fx_mean[o] = ppm_flux_ord<ORD8>(line3<0>(d, a.q_base, t, i, j, k), line2<0>(d, g.dxa, t, i, j), a.crx[o],
                                        i, s, e, mord);
    }
  });
  if (err != cudaSuccess) return err;
  // q_i (fvtp2d.py:33-47) on [0, n+6) x [js, je+4), q_j (50-60) on [is, ie+4) x [0, n+6)
  err = launch_box(Box{0, full, 0, full, 0, nk}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    real area = F2(g.area, i, j);
    if (j >= js && j < je + 4) {
      real fyy0 = F3(a.yfx, i, j) * F3(a.fy_mean, i, j);
      real fyy1 = F3(a.yfx, i, j + 1) * F3(a.fy_mean, i, j + 1);
      W3(a.q_adv_y, i, j) =
          ((i >= s && i <= e ? F3(a.q_base, i, j) : qy_at(d, a.q_base, t, i, j, k)) * area + fyy0 - fyy1) /
          (area + F3(a.yfx, i, j) - F3(a.yfx, i, j + 1));
    }
    if (i >= s && i < e + 4) {
      real fx10 = F3(a.xfx, i, j) * F3(a.fx_mean, i, j);
      real fx11 = F3(a.xfx, i + 1, j) * F3(a.fx_mean, i + 1, j);
      real awx = area + F3(a.xfx, i, j) - F3(a.xfx, i + 1, j);
      W3(a.q_adv_x, i, j) = (F3(a.q_base, i, j) * area + fx10 - fx11) / awx;
    }
  });
  if (err != cudaSuccess) return err;
  // outer PPM and final_fluxes (fvtp2d.py:63-93) on [is, ie+1] x [js, je+1],
  // the interior-path columns [is+3, ie-2] in warps of their own
  return launch_box_split(Box{s, e + 2, js, je + 2, 0, nk}, s + 3, e - 1, st,
                          [=] __device__(int t, int i, int j, int k) {
    const idx_t o = idx3(d, t, i, j, k);
    if (j <= je) {
      real xo = ppm_flux_ord<ORD8>(line3<0>(d, a.q_adv_y, t, i, j, k), line2<0>(d, g.dxa, t, i, j), a.crx[o], i, s,
                                   e, mord);
      a.fx[o] = RC(0.5) * (xo + a.fx_mean[o]) * a.x_unit[o];
    }
    if (i <= e) {
      real yo = ppm_flux_ord<ORD8>(line3<1>(d, a.q_adv_x, t, i, j, k), line2<1>(d, g.dya, t, i, j), a.cry[o], j, js,
                                   je, mord);
      a.fy[o] = RC(0.5) * (yo + a.fy_mean[o]) * a.y_unit[o];
    }
  });
}

// hord 5, 6, 7 or 8 (the caller rejects the rest)
inline cudaError_t fvtp2d(const Dims d, const fv3b_metrics g, const FvTp2dArgs a, cudaStream_t st) {
  return a.hord == 8 ? fvtp2d_impl<true>(d, g, a, st) : fvtp2d_impl<false>(d, g, a, st);
}

// The x half of CopyCornersXY in place (corners.py:64-117): only the 3 x 3
// cube-corner blocks of q change; levels [0, nlev) (all npz+1 by default).
inline cudaError_t copy_corners_x_inplace(const Dims d, real* q, cudaStream_t st, int nlev = -1) {
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  // 4 corner blocks of 3 x 3 points
  return launch_box(Box{0, 12, 0, 3, 0, nlev < 0 ? d.nk : nlev}, st, [=] __device__(int t, int x, int y, int k) {
    PT_SETUP(d, t, k);
    const int c = x / 3, a = x % 3;
    const int i = (c == 0 || c == 2) ? s - 3 + a : e + 1 + a;
    const int j = (c < 2) ? js - 3 + y : je + 1 + y;
    int si, sj;
    if (copy_corner_x(d, i, j, si, sj)) W3(q, i, j) = F3(q, si, sj);
  });
}

// Per-level damping column on the device: nord band value and damp.
struct DelnCol {
  const real* nord;  // [nk] per-level nord (band value, see nord_at)
  const real* damp;  // [nk], divided by rscale^nmax on levels that iterate
  real rscale;       // factor of every del-n pass (power of two; 1 in double builds)
};

// nord of level k: the reference folds the column into bands k = 0, 1, 2, 3+
// (delnflux.py intervals with externals nord0..nord3).
__device__ __forceinline__ int nord_at(const real* nord, int k) { return (int)nord[k < 3 ? k : 3]; }

// One point of a del-n flux pass: fx = del6_v * (d2(i-1, j) - d2(i, j)) and
// fy = del6_u * (d2(i, j-1) - d2(i, j)) on the pass's region (lo halo rows;
// levels with nord = 0 the compute-domain faces), corner points mapped to
// their copy sources first (fx_calc_stencil_nord / fy_calc_stencil_nord,
// delnflux.py:183-233).  D2(i, j) gives d2 at a point.
// DelnFlux's final step (add_diffusive_component / diffusive_damp,
// delnflux.py:276-294) done by the pass that produces the final fluxes:
// fx += fx2 (or 0.5 damp (mass(i-1) + mass(i)) fx2) on [is, ie+1] x
// [js, je+1].  Points of that box the final pass does not compute take the
// value the flux buffer already holds, as the separate stencil would.
struct DelnCombine {
  real* fx = nullptr;  // nullptr: no combine (DelnFluxNoSG)
  real* fy = nullptr;
  const real* mass = nullptr;
};

template <typename D2F>
__device__ __forceinline__ void deln_flux_point(const Dims& d, const fv3b_metrics& g, int t, int i, int j, int k,
                                                int lo, int nk_, bool first, real* wx, real* wy, const D2F& D2,
                                                const DelnCombine& cb = DelnCombine{}, const real* damp = nullptr) {
  PT_SETUP(d, t, k);
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  // reads at (i-1, j), (i, j), (i, j-1) can only hit a corner block when
  // i and j are both within one point of the tile's edge rows
  const bool corners = nk_ > 0 && (i <= s || i >= e + 1) && (j <= js || j >= je + 1);
  auto d2x = [&](int ii, int jj) {
    int si, sj;
    if (corners && copy_corner_x(d, ii, jj, si, sj)) return D2(si, sj);
    return D2(ii, jj);
  };
  auto d2y = [&](int ii, int jj) {
    int si, sj;
    if (corners && copy_corner_y(d, ii, jj, si, sj)) return D2(si, sj);
    return D2(ii, jj);
  };
  bool fx_in, fy_in;
  if (nk_ > 0) {
    fx_in = i >= s - lo && i < e + 2 + lo && j >= js - lo && j < je + 1 + lo;
    fy_in = i >= s - lo && i < e + 1 + lo && j >= js - lo && j < je + 2 + lo;
  } else {
    fx_in = i >= s && i < e + 2 && j >= js && j < je + 1;
    fy_in = i >= s && i < e + 1 && j >= js && j < je + 2;
  }
  // both fluxes before either store, so that the shared d2 reads are loaded once
  real vx = RC(0.0), vy = RC(0.0);
  if (fx_in) vx = F2(g.del6_v, i, j) * (d2x(i - 1, j) - d2x(i, j));
  if (fy_in) vy = F2(g.del6_u, i, j) * (d2y(i, j - 1) - d2y(i, j));
  if (cb.fx == nullptr) {
    if (fx_in) W3(wx, i, j) = first ? vx : -vx;
    if (fy_in) W3(wy, i, j) = first ? vy : -vy;
    return;
  }
  if (!(i >= s && i < e + 2 && j >= js && j < je + 2)) return;
  const real fx2 = fx_in ? (first ? vx : -vx) : F3(wx, i, j);
  const real fy2 = fy_in ? (first ? vy : -vy) : F3(wy, i, j);
  if (cb.mass == nullptr) {
    W3(cb.fx, i, j) = F3(cb.fx, i, j) + fx2;
    W3(cb.fy, i, j) = F3(cb.fy, i, j) + fy2;
  } else {
    const real dk = damp[k];
    W3(cb.fx, i, j) = F3(cb.fx, i, j) + RC(0.5) * dk * (F3(cb.mass, i - 1, j) + F3(cb.mass, i, j)) * fx2;
    W3(cb.fy, i, j) = F3(cb.fy, i, j) + RC(0.5) * dk * (F3(cb.mass, i, j - 1) + F3(cb.mass, i, j)) * fy2;
  }
}

// A later del-n pass (p >= 1) as a tiled kernel: a 32 x 4 block of one
// level computes the d2 values its fluxes read (its own points plus the row
// below and the column to the left) once into shared memory, instead of
// each thread recomputing three of them.  Blocks that touch a cube-corner
// zone take the per-point path (corner sources may lie outside the tile).
// Same operations in the same order either way.
struct DelnIterArgs {
  Dims d;
  fv3b_metrics g;
  DelnCol col;
  const real* px;
  const real* py;
  real* wx;
  real* wy;
  DelnCombine cb;
  int lo, i0, i1, j0, j1, nlev;
  bool final_pass;
};

constexpr int DELN_TX = 32, DELN_TY = 4;

static __global__ void __launch_bounds__(DELN_TX* DELN_TY) deln_iter_kernel(const DelnIterArgs a) {
  __shared__ real sd2[DELN_TY + 1][DELN_TX + 1];  // rows jb-1.., columns ib-1..
  const Dims& d = a.d;
  const int t = blockIdx.z / a.nlev, k = blockIdx.z % a.nlev;
  const int nk_ = nord_at(a.col.nord, k);
  if (nk_ == 0) return;  // whole block: one level
  const int ib = a.i0 + blockIdx.x * DELN_TX, jb = a.j0 + blockIdx.y * DELN_TY;
  const int i = ib + threadIdx.x, j = jb + threadIdx.y;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  const idx_t b3 = t * d.st + k * d.sk, b2 = t * d.st2;
  auto D2 = [&](int ii, int jj) {
    const idx_t o = b3 + jj * d.sj + ii;
    return (a.px[o] - a.px[o + 1] + a.py[o] - a.py[o + d.sj]) * a.g.rarea[b2 + jj * d.sj + ii] * a.col.rscale;
  };
  const bool near_corner = (ib <= s || ib + DELN_TX - 1 >= e + 1) && (jb <= js || jb + DELN_TY - 1 >= je + 1);
  if (near_corner) {
    if (i < a.i1 && j < a.j1) {
      if (a.final_pass)
        deln_flux_point(d, a.g, t, i, j, k, a.lo, nk_, false, a.wx, a.wy, D2, a.cb, a.col.damp);
      else
        deln_flux_point(d, a.g, t, i, j, k, a.lo, nk_, false, a.wx, a.wy, D2);
    }
    return;
  }
  // d2 at points whose four flux reads stay inside the arrays; others unused
  auto D2_safe = [&](int ii, int jj) {
    return (ii >= 0 && jj >= 0 && ii + 1 < d.ni && jj + 1 < d.nj) ? D2(ii, jj) : RC(0.0);
  };
  sd2[threadIdx.y + 1][threadIdx.x + 1] = D2_safe(i, j);
  if (threadIdx.y == 0) sd2[0][threadIdx.x + 1] = D2_safe(i, jb - 1);
  if (threadIdx.x == 0) sd2[threadIdx.y + 1][0] = D2_safe(ib - 1, j);
  __syncthreads();
  if (!(i < a.i1 && j < a.j1)) return;
  PT_SETUP(d, t, k);
  const int lo = a.lo;
  const bool fx_in = i >= s - lo && i < e + 2 + lo && j >= js - lo && j < je + 1 + lo;
  const bool fy_in = i >= s - lo && i < e + 1 + lo && j >= js - lo && j < je + 2 + lo;
  const real d2c = sd2[threadIdx.y + 1][threadIdx.x + 1];
  real vx = RC(0.0), vy = RC(0.0);
  if (fx_in) vx = F2(a.g.del6_v, i, j) * (sd2[threadIdx.y + 1][threadIdx.x] - d2c);
  if (fy_in) vy = F2(a.g.del6_u, i, j) * (sd2[threadIdx.y][threadIdx.x + 1] - d2c);
  const DelnCombine& cb = a.cb;
  if (!a.final_pass || cb.fx == nullptr) {
    if (fx_in) W3(a.wx, i, j) = -vx;
    if (fy_in) W3(a.wy, i, j) = -vy;
    return;
  }
  if (!(i >= s && i < e + 2 && j >= js && j < je + 2)) return;
  const real fx2 = fx_in ? -vx : F3(a.wx, i, j);
  const real fy2 = fy_in ? -vy : F3(a.wy, i, j);
  if (cb.mass == nullptr) {
    W3(cb.fx, i, j) = F3(cb.fx, i, j) + fx2;
    W3(cb.fy, i, j) = F3(cb.fy, i, j) + fy2;
  } else {
    const real dk = a.col.damp[k];
    W3(cb.fx, i, j) = F3(cb.fx, i, j) + RC(0.5) * dk * (F3(cb.mass, i - 1, j) + F3(cb.mass, i, j)) * fx2;
    W3(cb.fy, i, j) = F3(cb.fy, i, j) + RC(0.5) * dk * (F3(cb.mass, i, j - 1) + F3(cb.mass, i, j)) * fy2;
  }
}

// ------------------------------------------------------------ fused chain
// The whole del-n chain of one level (passes 0 .. NMAX, NMAX = 1 or 2) for
// one tile of the final fluxes, every pass in shared memory: q is read once
// and only the final fluxes (or their combine into fx, fy) are written,
// where the pass-by-pass form reads and writes two flux fields per pass.
//
// The window is the tile widened by NMAX + 1 points (low sides) and NMAX
// (high sides) and is one warp wide, so a thread keeps one window column
// and the same rows through every pass, with the metric terms of its
// points in registers.  Pass p is computed on the tile widened by NMAX - p
// points (what the next pass reads), its d2 on the points those fluxes
// read.  A pass writes only inside its own region, as the reference's does,
// into one of two flux sets that alternate as the global buffers do, so the
// points the final combine reads outside the final region hold the value
// of pass NMAX - 2 there, as the buffer does in the pass-by-pass form (for
// NMAX = 1 no pass of the chain writes them: the buffer is read).
//
// Most tiles lie inside every pass's region and away from the cube
// corners: they take the path without region tests.  The others test the
// region per point and map the d2 reads of corner points to their copy
// sources inside the window; a pass-0 source outside the window is damp q
// read from q.  deln_window_ok checks on the host, for the grid at hand,
// that every later-pass source lies inside the window; where it does not,
// the chain runs pass by pass.  Levels with nord = 0 take their single pass
// here.  Same operations in the same order as the pass-by-pass form, so the
// results are the same numbers.
constexpr int CHAIN_TY = 16, CHAIN_BY = 8;

template <int NMAX>
struct DelnTile {
  static constexpr int TX = 32 - 2 * NMAX - 1;            // output columns
  static constexpr int WY = CHAIN_TY + 2 * NMAX + 1;       // window rows
  static constexpr int R = (WY + CHAIN_BY - 1) / CHAIN_BY;  // window rows per thread
};

struct DelnChainArgs {
  Dims d;
  fv3b_metrics g;
  DelnCol col;
  const real* q;
  real* fx2;  // final fluxes; with a combine, the final-pass buffer
  real* fy2;
  DelnCombine cb;
  int mass_weighted;
  int nlev;
};

template <int NMAX>
static __global__ void __launch_bounds__(32 * CHAIN_BY) deln_chain_kernel(const DelnChainArgs a) {
  using G = DelnTile<NMAX>;
  constexpr int TX = G::TX, WY = G::WY, R = G::R, WN = 32 * WY;
  __shared__ real sd2[WN];
  __shared__ real sfx[2][WN];
  __shared__ real sfy[2][WN];
  const Dims& d = a.d;
  const int t = blockIdx.z / a.nlev, k = blockIdx.z % a.nlev;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  const int i0 = s + blockIdx.x * TX, j0 = js + blockIdx.y * CHAIN_TY;
  const int wi0 = i0 - NMAX - 1, wj0 = j0 - NMAX - 1;
  const int x = threadIdx.x, ty = threadIdx.y;
  const int i = wi0 + x;
  const idx_t b3 = t * d.st + k * d.sk, b2 = t * d.st2;
  const int nk_ = nord_at(a.col.nord, k);
  const real damp = a.col.damp[k];
  const real* q = a.q;
  const bool mw = a.mass_weighted != 0;
  const bool out_col = x >= NMAX + 1 && x < NMAX + 1 + TX && i < e + 2;
  if (nk_ == 0) {
    // one pass on the compute-domain faces, combined now if asked
    if (!out_col) return;
    auto D2 = [&](int ii, int jj) {
      const real qv = q[b3 + jj * d.sj + ii];
      return mw ? qv : damp * qv;
    };
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int y = ty + r * CHAIN_BY, j = wj0 + y;
      if (y >= NMAX + 1 && y < NMAX + 1 + CHAIN_TY && j < je + 2)
        deln_flux_point(d, a.g, t, i, j, k, NMAX, 0, true, a.fx2, a.fy2, D2, a.cb, a.col.damp);
    }
    return;
  }
  const int i1 = min(i0 + TX, e + 2), j1 = min(j0 + CHAIN_TY, je + 2);
  // inside every region, no corner point, the window inside the arrays
  const bool slow = i1 == e + 2 || j1 == je + 2 ||
                    ((i0 - NMAX <= s || i1 - 1 + NMAX >= e + 1) && (j0 - NMAX <= js || j1 - 1 + NMAX >= je + 1));
  real m_ra[R], m_dv[R], m_du[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int y = ty + r * CHAIN_BY, jj = wj0 + y;
    const bool ok = y < WY && i < d.ni && jj < d.nj;
    const idx_t o2 = b2 + jj * d.sj + i;
    m_ra[r] = ok ? a.g.rarea[o2] : RC(0.0);
    m_dv[r] = ok ? a.g.del6_v[o2] : RC(0.0);
    m_du[r] = ok ? a.g.del6_u[o2] : RC(0.0);
    if (y < WY) {
      real v = RC(0.0);
      if (ok) {
        const real qv = q[b3 + jj * d.sj + i];
        v = mw ? qv : damp * qv;
      }
      sd2[y * 32 + x] = v;
    }
  }
  __syncthreads();
#pragma unroll
  for (int p = 0; p <= NMAX; ++p) {
    if (p > 0) {
      // d2 of pass p from the fluxes of pass p - 1, window shrunk by p
      const int ps = (NMAX - p + 1) & 1;
      if (x >= p && x < 32 - p) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int y = ty + r * CHAIN_BY;
          if (y >= p && y < WY - p) {
            const int c = y * 32 + x;
            real v = RC(0.0);
            if (!slow || (i + 1 < d.ni && wj0 + y + 1 < d.nj))
              v = (sfx[ps][c] - sfx[ps][c + 1] + sfy[ps][c] - sfy[ps][c + 32]) * m_ra[r] * a.col.rscale;
            sd2[c] = v;
          }
        }
      }
      __syncthreads();
    }
    // fluxes of pass p, window shrunk by p + 1 on the low sides and p on the high sides
    const int set = (NMAX - p) & 1, lo = NMAX - p;
    if (x >= p + 1 && x < 32 - p) {
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int y = ty + r * CHAIN_BY;
        if (!(y >= p + 1 && y < WY - p)) continue;
        const int c = y * 32 + x;
        const real d2c = sd2[c];
        if (!slow) {
          const real vx = m_dv[r] * (sd2[c - 1] - d2c);
          const real vy = m_du[r] * (sd2[c - 32] - d2c);
          sfx[set][c] = p == 0 ? vx : -vx;
          sfy[set][c] = p == 0 ? vy : -vy;
          continue;
        }
        const int j = wj0 + y;
        const bool fx_in = i >= s - lo && i < e + 2 + lo && j >= js - lo && j < je + 1 + lo;
        const bool fy_in = i >= s - lo && i < e + 1 + lo && j >= js - lo && j < je + 2 + lo;
        const bool corners = (i <= s || i >= e + 1) && (j <= js || j >= je + 1);
        // d2 of this pass at storage point (ii, jj)
        auto d2w = [&](int ii, int jj) -> real {
          const int xx = ii - wi0, yy = jj - wj0;
          if (p == 0 && (xx < 0 || xx >= 32 || yy < 0 || yy >= WY)) {
            const real qv = q[b3 + jj * d.sj + ii];
            return mw ? qv : damp * qv;
          }
          return sd2[yy * 32 + xx];
        };
        if (fx_in) {
          int ai = i - 1, aj = j, bi = i, bj = j;
          if (corners) {
            int si, sj;
            if (copy_corner_x(d, i - 1, j, si, sj)) ai = si, aj = sj;
            if (copy_corner_x(d, i, j, si, sj)) bi = si, bj = sj;
          }
          const real vx = m_dv[r] * (d2w(ai, aj) - d2w(bi, bj));
          sfx[set][c] = p == 0 ? vx : -vx;
        }
        if (fy_in) {
          int ai = i, aj = j - 1, bi = i, bj = j;
          if (corners) {
            int si, sj;
            if (copy_corner_y(d, i, j - 1, si, sj)) ai = si, aj = sj;
            if (copy_corner_y(d, i, j, si, sj)) bi = si, bj = sj;
          }
          const real vy = m_du[r] * (d2w(ai, aj) - d2w(bi, bj));
          sfy[set][c] = p == 0 ? vy : -vy;
        }
      }
    }
    __syncthreads();
  }
  if (!out_col) return;
  PT_SETUP(d, t, k);
  const DelnCombine& cb = a.cb;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int y = ty + r * CHAIN_BY, j = wj0 + y;
    if (!(y >= NMAX + 1 && y < NMAX + 1 + CHAIN_TY && j < je + 2)) continue;
    const int c = y * 32 + x;
    const bool fx_in = j < je + 1, fy_in = i < e + 1;  // the final region (i >= is, j >= js hold)
    if (cb.fx == nullptr) {
      if (fx_in) W3(a.fx2, i, j) = sfx[0][c];
      if (fy_in) W3(a.fy2, i, j) = sfy[0][c];
      continue;
    }
    const real fx2 = (fx_in || NMAX >= 2) ? sfx[0][c] : F3(a.fx2, i, j);
    const real fy2 = (fy_in || NMAX >= 2) ? sfy[0][c] : F3(a.fy2, i, j);
    if (cb.mass == nullptr) {
      W3(cb.fx, i, j) = F3(cb.fx, i, j) + fx2;
      W3(cb.fy, i, j) = F3(cb.fy, i, j) + fy2;
    } else {
      W3(cb.fx, i, j) = F3(cb.fx, i, j) + RC(0.5) * damp * (F3(cb.mass, i - 1, j) + F3(cb.mass, i, j)) * fx2;
      W3(cb.fy, i, j) = F3(cb.fy, i, j) + RC(0.5) * damp * (F3(cb.mass, i, j - 1) + F3(cb.mass, i, j)) * fy2;
    }
  }
}

// Whether every d2 read of the fused chain's later passes (p >= 1) at a
// corner point, mapped to its copy source, lies inside the tile's window
// and reads fluxes of the pass before inside that pass's region: an
// enumeration over the tiles that hold corner points (the other reads lie
// inside by construction).  Results cached per (n, halo, nmax).
template <int NMAX>
inline bool deln_window_ok_impl(const Dims& d) {
  using G = DelnTile<NMAX>;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  auto fxr = [&](int lo, int i, int j) { return i >= s - lo && i < e + 2 + lo && j >= js - lo && j < je + 1 + lo; };
  auto fyr = [&](int lo, int i, int j) { return i >= s - lo && i < e + 1 + lo && j >= js - lo && j < je + 2 + lo; };
  for (int i0 = s; i0 < e + 2; i0 += G::TX)
    for (int j0 = js; j0 < je + 2; j0 += CHAIN_TY) {
      const int i1 = std::min(i0 + G::TX, e + 2), j1 = std::min(j0 + CHAIN_TY, je + 2);
      const int wi0 = i0 - NMAX - 1, wj0 = j0 - NMAX - 1;
      for (int p = 1; p <= NMAX; ++p) {
        const int lo = NMAX - p;
        for (int i = i0 - lo; i < i1 + lo; ++i)
          for (int j = j0 - lo; j < j1 + lo; ++j) {
            if (!((i <= s || i >= e + 1) && (j <= js || j >= je + 1))) continue;
            for (int kind = 0; kind < 2; ++kind) {
              if (!(kind == 0 ? fxr(lo, i, j) : fyr(lo, i, j))) continue;
              const int pts[2][2] = {{kind == 0 ? i - 1 : i, kind == 0 ? j : j - 1}, {i, j}};
              for (const auto& pt : pts) {
                int ii = pt[0], jj = pt[1], si, sj;
                if (kind == 0 ? copy_corner_x(d, ii, jj, si, sj) : copy_corner_y(d, ii, jj, si, sj)) ii = si, jj = sj;
                const int xx = ii - wi0, yy = jj - wj0;
                if (xx < p || xx >= 32 - p || yy < p || yy >= G::WY - p) return false;
                if (!(fxr(lo + 1, ii, jj) && fxr(lo + 1, ii + 1, jj) && fyr(lo + 1, ii, jj) &&
                      fyr(lo + 1, ii, jj + 1)))
                  return false;
              }
            }
          }
      }
    }
  return true;
}

inline bool deln_window_ok(const Dims& d, int nmax) {
  static std::mutex mu;
  static std::map<long long, bool> cache;
  const long long key = ((long long)d.n * 64 + d.h) * 4 + nmax;
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  const bool ok = d.h >= 3 && (nmax == 1 ? deln_window_ok_impl<1>(d) : deln_window_ok_impl<2>(d));
  cache[key] = ok;
  return ok;
}

// DelnFluxNoSG.__call__ (delnflux.py:1156-1207): del-n diffusive fluxes of q
// into fx2/fy2.  Corner copies of d2 are applied on read (a point of a
// corner block reads its copy source), which gives the values the reference
// reads after copying the corners in place.
//
// The reference alternates a d2 stencil (d2 = damp * q, then the divergence
// of the last fluxes times rarea) with a flux stencil that differences d2.
// Here each flux pass computes the d2 values it needs on the fly from q or
// from the previous pass's fluxes, with the reference's operation order, so
// d2 is never stored: nmax + 1 passes instead of 2 * (nmax + 1).  Every d2
// point a pass reads (corner sources included) lies inside the region where
// the reference computes d2, so the values are the same.  Consecutive
// passes ping-pong between (fx2, fy2) and the scratch pair (ax, ay), ending
// in (fx2, fy2); levels with nord = 0 take the first pass only, written to
// (fx2, fy2).
// nlev is the number of levels (npz by default; UpdateHeightOnDGrid runs it
// on npz + 1 interface levels).
inline cudaError_t delnflux_nosg(const Dims d, const fv3b_metrics g, const real* q, real* fx2, real* fy2,
                                 DelnCol col, real* ax, real* ay, bool mass_weighted, int nmax, cudaStream_t st,
                                 int nlev = -1, DelnCombine cb = DelnCombine{}) {
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec, nz = nlev < 0 ? d.nz : nlev;
  // pass p writes (fx2, fy2) when nmax - p is even, so the last pass does
  auto out_x = [&](int p) { return ((nmax - p) % 2 == 0) ? fx2 : ax; };
  auto out_y = [&](int p) { return ((nmax - p) % 2 == 0) ? fy2 : ay; };
  if ((nmax == 1 || nmax == 2) && deln_window_ok(d, nmax)) {
    DelnChainArgs a{d, g, col, q, fx2, fy2, cb, mass_weighted ? 1 : 0, nz};
    const int len = e + 2 - s;
    const int tx = nmax == 1 ? DelnTile<1>::TX : DelnTile<2>::TX;
    const dim3 grid((len + tx - 1) / tx, (len + CHAIN_TY - 1) / CHAIN_TY, tile_slots() * nz);
    if (nmax == 1)
      deln_chain_kernel<1><<<grid, dim3(32, CHAIN_BY, 1), 0, st>>>(a);
    else
      deln_chain_kernel<2><<<grid, dim3(32, CHAIN_BY, 1), 0, st>>>(a);
    note_launch();
    return cudaGetLastError();
  }
  // first pass: d2 = damp * q (d2_damp_interval) or q (copy_stencil_interval)
  {
    const int lo = nmax;
    real *wx = out_x(0), *wy = out_y(0);
    cudaError_t err = launch_box(Box{s - lo, e + 2 + lo, js - lo, je + 2 + lo, 0, nz}, st,
                                 [=] __device__(int t, int i, int j, int k) {
                                   const int nk_ = nord_at(col.nord, k);
                                   const idx_t b3 = t * d.st + k * d.sk;
                                   const real damp = col.damp[k];
                                   auto D2 = [&](int ii, int jj) {
                                     const real qv = q[b3 + jj * d.sj + ii];
                                     return mass_weighted ? qv : damp * qv;
                                   };
                                   // levels with nord = 0 (all levels when nmax = 0)
                                   // end here: combine now if asked
                                   if (nk_ > 0)
                                     deln_flux_point(d, g, t, i, j, k, lo, nk_, true, wx, wy, D2);
                                   else
                                     deln_flux_point(d, g, t, i, j, k, lo, nk_, true, fx2, fy2, D2, cb, col.damp);
                                 });
    if (err != cudaSuccess) return err;
  }
  // later passes on levels with nord > 0: d2 from the previous fluxes
  // (d2_highorder_stencil, delnflux.py:159-181), then the fluxes
  // (fx/fy_calc_stencil_column)
  for (int p = 1; p <= nmax; ++p) {
    const int lo = nmax - p;
    DelnIterArgs a{d, g, col, out_x(p - 1), out_y(p - 1), out_x(p), out_y(p), cb,
                   lo, s - lo, e + 2 + lo, js - lo, je + 2 + lo, nz, p == nmax};
    const dim3 grid((a.i1 - a.i0 + DELN_TX - 1) / DELN_TX, (a.j1 - a.j0 + CHAIN_TY - 1) / CHAIN_TY, tile_slots() * nz);
    deln_iter_kernel<<<grid, dim3(DELN_TX, CHAIN_TY, 1), 0, st>>>(a);
    note_launch();
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
  }
  return cudaSuccess;
}

// DelnFlux.__call__ (delnflux.py:963-998): damped fluxes added to fx, fy on
// the cell corners of the compute domain.
inline cudaError_t delnflux(const Dims d, const fv3b_metrics g, const real* q, real* fx, real* fy, DelnCol col,
                           const real* mass, real* fx2, real* fy2, real* ax, real* ay, int nmax, cudaStream_t st) {
  DelnCombine cb;
  cb.fx = fx;
  cb.fy = fy;
  cb.mass = mass;
  return delnflux_nosg(d, g, q, fx2, fy2, col, ax, ay, mass != nullptr, nmax, st, -1, cb);
}


}  // namespace fv3b

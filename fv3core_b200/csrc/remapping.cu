// LagrangianToEulerian: the vertical remapping of DynamicalCore.step_dynamics
// (fv3core/stencils/remapping.py:205-628, map_single.py, remap_profile.py,
// mapn_tracer.py, fillz.py, moist_cv.py), without the saturation adjustment.
//
// Every field a remap touches is a set of independent columns, so each
// stage is a column kernel: one thread per (tile, i, j) column, neighbouring
// threads on neighbouring i (each level access is one coalesced row).  The
// PPM profile (cs_profile) and the Lagrangian contributions run in FP64 in
// per-thread work arrays sized by a level bucket (NK >= npz + 1), in both
// builds: the remap differences pressures of ~1e5 Pa across layers of
// ~1e2..1e3 Pa, which FP32 cannot resolve to 1e-4.  The Eulerian pressures
// ak + bk ps, their logarithms and thicknesses are recomputed per column
// from ps instead of being stored, and the Lagrangian pressures are the
// state's pe (the reference's pe1 copy) until the last stage overwrites pe.
//
// Launches, in the reference's order where one reads what another writes:
//   1. moist pt, delz adjustment, ps, delp = dp2, pk (pointwise per level);
//   2. pt remapped in log pressure (kord_tm, iv 1, qmin 184 K); peln = log pe2;
//   3. each tracer remapped (kord_tr, the sixth kord 9, iv 0), then fillz;
//   4. w (kord_wz, iv -2, bottom value wsd);
//   5. delz (kord_wz, iv 1), then delz = -delz dp2;
//   6. moist pkz, then (do_sat_adj) the fast saturation adjustment on levels
//      [kmp, npz), then the last-step pt conversion (or pt / pkz);
//   7. u on pressures averaged to the D-grid y faces (kord_mt, iv -1);
//   8. v on pressures averaged to the x faces;
//   9. update_ua and copy_from_below (ua, the interior pe).
// Statement order and branch structure follow the reference, and exp / log
// are the library's own (fmath.h), so FP64 results agree with the oracle
// bit for bit.
#include <math.h>

#include <type_traits>

#include "ctx.cuh"
#include "fmath.h"
#include "sat_adjust.cuh"
#include "stencil.cuh"

using namespace fv3b;

namespace {

// fv3core/utils/global_constants.py
constexpr double RDGAS_D = 287.05, RVGAS_D = 461.50, GRAV_D = 9.80665, CP_AIR_D = 1004.6;
constexpr double CV_AIR_D = CP_AIR_D - RDGAS_D, RDG_D = -RDGAS_D / GRAV_D;
constexpr double CV_VAP_D = 3.0 * RVGAS_D, C_ICE_D = 1972.0, C_LIQ_D = 4.1855e3;

constexpr int NTRACER = 8;
constexpr unsigned char EXTM = 1, EXT5 = 2, EXT6 = 4;

// per-thread work arrays of one column remap
template <int NK>
struct MapWork {
  double a1[NK], a2[NK], a3[NK], a4[NK];
  double q[NK], gam[NK];  // interface values (npz + 1) and the profile's gam
  double p1[NK], p2[NK];  // source and target interface pressures (npz + 1)
  unsigned char ext[NK];  // extm / ext5 / ext6 bits
};

__device__ __forceinline__ double min3(double a, double p, double lac) {
  // a if (a < p) and (a < lac) else p if p < lac else lac
  return (a < p && a < lac) ? a : (p < lac ? p : lac);
}
__device__ __forceinline__ double max3(double a, double p, double lac) {
  return (a > p && a > lac) ? a : (p > lac ? p : lac);
}

// posdef_constraint_iv1 (remap_profile.py:73-92)
__device__ __forceinline__ void posdef_iv1(double a1, double& a2, double& a3, double& a4) {
  const double da1 = a3 - a2;
  const double da2 = da1 * da1;
  const double a6da = a4 * da1;
  if (((a1 - a2) * (a1 - a3)) >= 0.0) {
    a2 = a1;
    a3 = a1;
    a4 = 0.0;
  } else if (a6da < -1.0 * da2) {
    a4 = 3.0 * (a2 - a1);
    a3 = a2 - a4;
  } else if (a6da > da2) {
    a4 = 3.0 * (a3 - a1);
    a2 = a3 - a4;
  }
}

// remap_constraint (remap_profile.py:95-115)
__device__ __forceinline__ void remap_constraint(double a1, double& a2, double& a3, double& a4, bool extm) {
  const double da1 = a3 - a2;
  const double da2 = da1 * da1;
  const double a6da = a4 * da1;
  if (extm) {
    a2 = a1;
    a3 = a1;
    a4 = 0.0;
  } else if (a6da < -da2) {
    a4 = 3.0 * (a2 - a1);
    a3 = a2 - a4;
  } else if (a6da > da2) {
    a4 = 3.0 * (a3 - a1);
    a2 = a3 - a4;
  }
}

// posdef_constraint_iv0 (remap_profile.py:44-70)
__device__ __forceinline__ void posdef_iv0(double a1, double& a2, double& a3, double& a4) {
  if (a1 <= 0.0) {
    a2 = a1;
    a3 = a1;
    a4 = 0.0;
  } else {
    const double d = a3 - a2;
    if (fabs(a3 - a2) < -a4 && (a1 + 0.25 * (d * d) / a4 + a4 * (1.0 / 12.0)) < 0.0) {
      if ((a1 < a3) && (a1 < a2)) {
        a3 = a1;
        a2 = a1;
        a4 = 0.0;
      } else if (a3 > a2) {
        a4 = 3.0 * (a2 - a1);
        a3 = a2 - a4;
      } else {
        a4 = 3.0 * (a3 - a1);
        a2 = a3 - a4;
      }
    }
  }
}

// RemapProfile (remap_profile.py:495-638): the PPM coefficients a2..a4 of
// the km layer means a1 over layers of thickness dp(k) = p1[k+1] - p1[k].
template <int NK>
__device__ void remap_profile(MapWork<NK>& w, int km, int iv, int kord, double qs, double qmin) {
  const double* a1 = w.a1;
  double* q = w.q;
  double* gam = w.gam;
  auto dp = [&](int k) { return w.p1[k + 1] - w.p1[k]; };
  // set_initial_vals (118-214)
  if (iv == -2) {
    q[0] = 1.5 * a1[0];
    gam[1] = 0.5;
    {
      const double gr = dp(0) / dp(1);
      const double bet = 2.0 + gr + gr - gam[1];
      q[1] = (3.0 * (a1[0] + a1[1]) - q[0]) / bet;
    }
    for (int k = 2; k < km; ++k) {
      const double ogr = dp(k - 2) / dp(k - 1);
      const double obet = 2.0 + ogr + ogr - gam[k - 1];
      gam[k] = ogr / obet;
    }
    for (int k = 2; k < km - 1; ++k) {
      const double gr = dp(k - 1) / dp(k);
      const double bet = 2.0 + gr + gr - gam[k];
      q[k] = (3.0 * (a1[k - 1] + a1[k]) - q[k - 1]) / bet;
    }
    {
      const int k = km - 1;
      const double gr = dp(k - 1) / dp(k);
      q[k] = (3.0 * (a1[k - 1] + a1[k]) - gr * qs - q[k - 1]) / (2.0 + gr + gr - gam[k]);
    }
    q[km] = qs;
    for (int k = km - 2; k >= 0; --k) q[k] = q[k] - gam[k + 1] * q[k + 1];
  } else {
    {
      const double gr = dp(1) / dp(0);
      const double bet = gr * (gr + 0.5);
      q[0] = ((gr + gr) * (gr + 1.0) * a1[0] + a1[1]) / bet;
      gam[0] = (1.0 + gr * (gr + 1.5)) / bet;
    }
    for (int k = 1; k < km; ++k) {
      const double d4 = dp(k - 1) / dp(k);
      const double bet = 2.0 + d4 + d4 - gam[k - 1];
      q[k] = (3.0 * (a1[k - 1] + d4 * a1[k]) - q[k - 1]) / bet;
      gam[k] = d4 / bet;
    }
    {
      const double d4 = dp(km - 2) / dp(km - 1);
      const double a_bot = 1.0 + d4 * (d4 + 1.5);
      q[km] = (2.0 * d4 * (d4 + 1.0) * a1[km - 1] + a1[km - 2] - a_bot * q[km - 1]) /
              (d4 * (d4 + 0.5) - a_bot * gam[km - 1]);
    }
    for (int k = km - 1; k >= 0; --k) q[k] = q[k] - gam[k] * q[k + 1];
  }

  // apply_constraints (217-295): gam = a1 - a1(k-1), q within its
  // neighbouring means (one side only at a local extremum)
  for (int k = 1; k < km; ++k) gam[k] = a1[k] - a1[k - 1];
  auto tmp_of = [&](int k) { return a1[k - 1] > a1[k] ? a1[k - 1] : a1[k]; };
  auto tmp2_of = [&](int k) { return a1[k - 1] < a1[k] ? a1[k - 1] : a1[k]; };
  {
    const int k = 1;
    if (q[k] >= tmp_of(k)) q[k] = tmp_of(k);
    if (q[k] <= tmp2_of(k)) q[k] = tmp2_of(k);
  }
  for (int k = 2; k < km - 1; ++k) {
    const double tmp = tmp_of(k), tmp2 = tmp2_of(k);
    if ((gam[k - 1] * gam[k + 1]) > 0) {
      if (q[k] >= tmp) q[k] = tmp;
      if (q[k] <= tmp2) q[k] = tmp2;
    } else if (gam[k - 1] > 0) {
      if (q[k] <= tmp2) q[k] = tmp2;
    } else {
      if (q[k] >= tmp) q[k] = tmp;
      if (iv == 0 && q[k] < 0.0) q[k] = 0.0;
    }
  }
  {
    const int k = km - 1;
    if (q[k] >= tmp_of(k)) q[k] = tmp_of(k);
    if (q[k] <= tmp2_of(k)) q[k] = tmp2_of(k);
  }
  double* a2 = w.a2;
  double* a3 = w.a3;
  double* a4 = w.a4;
  unsigned char* ext = w.ext;
  for (int k = 0; k < km; ++k) {
    a2[k] = q[k];
    a3[k] = q[k + 1];
  }
  for (int k = 0; k < km; ++k) {
    bool extm;
    if (k == 0 || k == km - 1)
      extm = (a2[k] - a1[k]) * (a3[k] - a1[k]) > 0.0;
    else
      extm = gam[k] * gam[k + 1] < 0.0;
    unsigned char b = extm ? EXTM : 0;
    if (kord > 9) {
      const double x0 = 2.0 * a1[k] - (a2[k] + a3[k]);
      const double x1 = fabs(a2[k] - a3[k]);
      a4[k] = 3.0 * x0;
      if (fabs(x0) > x1) b |= EXT5;
      if (fabs(a4[k]) > x1) b |= EXT6;
    }
    ext[k] = b;
  }

  // set_interpolation_coefficients (298-492)
  if (iv == 0) {
    if (a2[0] < 0.0) a2[0] = 0.0;
  } else if (iv == -1) {
    if (a2[0] * a1[0] <= 0.0) a2[0] = 0.0;
  }
  if (iv == 2) {
    a2[0] = a1[0];
    a3[0] = a1[0];
    a4[0] = 0.0;
    a4[1] = 3.0 * (2.0 * a1[1] - (a2[1] + a3[1]));
  } else {
    for (int k = 0; k < 2; ++k) a4[k] = 3.0 * (2.0 * a1[k] - (a2[k] + a3[k]));
    posdef_iv1(a1[0], a2[0], a3[0], a4[0]);
  }
  remap_constraint(a1[1], a2[1], a3[1], a4[1], ext[1] & EXTM);
  for (int k = 2; k < km - 2; ++k) {
    const double b1 = a1[k];
    double b2 = a2[k], b3 = a3[k], b4 = a4[k];
    if (kord < 9) {
      const double pmp_1 = b1 - gam[k + 1];
      const double lac_1 = pmp_1 + 1.5 * gam[k + 2];
      double tmin = min3(b1, pmp_1, lac_1);
      double tmax0 = b2 > tmin ? b2 : tmin;
      double tmax = max3(b1, pmp_1, lac_1);
      b2 = tmax0 < tmax ? tmax0 : tmax;
      const double pmp_2 = b1 + 2.0 * gam[k + 1];
      const double lac_2 = pmp_2 - 1.5 * gam[k - 1];
      tmin = min3(b1, pmp_2, lac_2);
      tmax0 = b3 > tmin ? b3 : tmin;
      tmax = max3(b1, pmp_2, lac_2);
      b3 = tmax0 < tmax ? tmax0 : tmax;
      b4 = 3.0 * (2.0 * b1 - (b2 + b3));
    } else if (kord == 9) {
      const double pmp_1 = b1 - 2.0 * gam[k + 1];
      const double lac_1 = pmp_1 + 1.5 * gam[k + 2];
      const double pmp_2 = b1 + 2.0 * gam[k];
      const double lac_2 = pmp_2 - 1.5 * gam[k - 1];
      const bool e0 = ext[k] & EXTM;
      if ((e0 && (ext[k - 1] & EXTM)) || (e0 && (ext[k + 1] & EXTM)) || (e0 && (qmin > 0.0 && b1 < qmin))) {
        b2 = b1;
        b3 = b1;
        b4 = 0.0;
      } else {
        b4 = 6.0 * b1 - 3.0 * (b2 + b3);
        if (fabs(b4) > fabs(b2 - b3)) {
          double tmin = min3(b1, pmp_1, lac_1);
          double tmax0 = b2 > tmin ? b2 : tmin;
          double tmax = max3(b1, pmp_1, lac_1);
          b2 = tmax0 < tmax ? tmax0 : tmax;
          tmin = min3(b1, pmp_2, lac_2);
          tmax0 = b3 > tmin ? b3 : tmin;
          tmax = max3(b1, pmp_2, lac_2);
          b3 = tmax0 < tmax ? tmax0 : tmax;
          b4 = 6.0 * b1 - 3.0 * (b2 + b3);
        }
      }
    } else {  // kord 10
      const double pmp_1 = b1 - 2.0 * gam[k + 1];
      const double lac_1 = pmp_1 + 1.5 * gam[k + 2];
      const double pmp_2 = b1 + 2.0 * gam[k];
      const double lac_2 = pmp_2 - 1.5 * gam[k - 1];
      const double tmin2 = min3(b1, pmp_1, lac_1);
      const double tmax2 = max3(b1, pmp_1, lac_1);
      const double t2 = b2 > tmin2 ? b2 : tmin2;
      double tmin3 = b1 < pmp_2 ? b1 : pmp_2;
      tmin3 = lac_2 < tmin3 ? lac_2 : tmin3;
      double tmax3 = b1 > pmp_2 ? b1 : pmp_2;
      tmax3 = lac_2 > tmax3 ? lac_2 : tmax3;
      const double t3 = b3 > tmin3 ? b3 : tmin3;
      const bool e5 = ext[k] & EXT5, e6 = ext[k] & EXT6;
      const bool e5n = (ext[k - 1] & EXT5) || (ext[k + 1] & EXT5);
      const bool e6n = (ext[k - 1] & EXT6) || (ext[k + 1] & EXT6);
      if (e5) {
        if (e5n) {
          b2 = b1;
          b3 = b1;
        } else if (e6n) {
          b2 = t2 < tmax2 ? t2 : tmax2;
          b3 = t3 < tmax3 ? t3 : tmax3;
        }
      } else if (e6) {
        if (e5n) {
          b2 = t2 < tmax2 ? t2 : tmax2;
          b3 = t3 < tmax3 ? t3 : tmax3;
        }
      }
      b4 = 3.0 * (2.0 * b1 - (b2 + b3));
    }
    if (iv == 0) posdef_iv0(b1, b2, b3, b4);
    a2[k] = b2;
    a3[k] = b3;
    a4[k] = b4;
  }
  {
    const int k = km - 1;
    if (iv == 0) {
      if (a3[k] < 0.0) a3[k] = 0.0;
    }
    if (iv == -1) {
      if (a3[k] * a1[k] <= 0.0) a3[k] = 0.0;
    }
  }
  for (int k = km - 2; k < km; ++k) a4[k] = 3.0 * (2.0 * a1[k] - (a2[k] + a3[k]));
  remap_constraint(a1[km - 2], a2[km - 2], a3[km - 2], a4[km - 2], ext[km - 2] & EXTM);
  posdef_iv1(a1[km - 1], a2[km - 1], a3[km - 1], a4[km - 1]);
}

// lagrangian_contributions (map_single.py:19-66): the mean of the profile
// over each target layer [p2[k], p2[k+1]], into out[k].  L is the absolute
// source level (the reference's relative offset lev plus k); it stays below
// km so that no read leaves the column even for inputs whose surfaces
// disagree at the bottom.
template <int NK>
__device__ void lagrangian_contributions(MapWork<NK>& w, int km, double* out) {
  const double* p1 = w.p1;
  const double* p2 = w.p2;
  auto dp1 = [&](int k) { return p1[k + 1] - p1[k]; };
  int L = 0;
  for (int k = 0; k < km; ++k) {
    const double pl = (p2[k] - p1[L]) / dp1(L);
    if (p2[k + 1] <= p1[L + 1]) {
      const double pr = (p2[k + 1] - p1[L]) / dp1(L);
      out[k] = w.a2[L] + 0.5 * (w.a4[L] + w.a3[L] - w.a2[L]) * (pr + pl) -
               w.a4[L] * 1.0 / 3.0 * (pr * (pr + pl) + pl * pl);
    } else {
      double qsum = (p1[L + 1] - p2[k]) * (w.a2[L] + 0.5 * (w.a4[L] + w.a3[L] - w.a2[L]) * (1.0 + pl) -
                                           w.a4[L] * 1.0 / 3.0 * (1.0 + pl * (1.0 + pl)));
      L = L + 1 < km ? L + 1 : km - 1;
      while (L + 1 < km && p1[L + 1] < p2[k + 1]) {
        qsum += dp1(L) * w.a1[L];
        L = L + 1;
      }
      const double dp = p2[k + 1] - p1[L];
      const double esl = dp / dp1(L);
      qsum += dp * (w.a2[L] + 0.5 * esl * (w.a3[L] - w.a2[L] + w.a4[L] * (1.0 - (2.0 / 3.0) * esl)));
      out[k] = qsum / (p2[k + 1] - p2[k]);
    }
  }
}

// MapSingle (map_single.py:130-173) of one column: w.a1 holds the layer
// means, w.p1 / w.p2 the source / target interfaces; the remapped means go
// to w.q[0..km).
template <int NK>
__device__ __forceinline__ void map_column(MapWork<NK>& w, int km, int iv, int kord, double qs, double qmin) {
  remap_profile<NK>(w, km, iv, kord, qs, qmin);
  lagrangian_contributions<NK>(w, km, w.q);
}

// fix_tracer (fillz.py:10-98) on one column q[0..km) with layer thickness
// dp(k); the column's zfix, sums and borrow records are the thread's own.
template <int NK, typename DPF>
__device__ void fix_tracer(double* q, const DPF& dp, int km) {
  double dm[NK], dm_pos[NK], lower_fix[NK], upper_fix[NK];
  for (int k = 0; k < km; ++k) {
    lower_fix[k] = 0.0;
    upper_fix[k] = 0.0;
  }
  int zfix = 0;
  // fix_top
  if (q[0] < 0) q[0] = 0;
  dm[0] = q[0] * dp(0);
  if (q[0] < 0.0) q[1] = q[1] + q[0] * dp(0) / dp(1);
  // fix_interior
  for (int k = 1; k < km - 1; ++k) {
    if (lower_fix[k - 1] != 0.0) q[k] = q[k] - (lower_fix[k - 1] / dp(k));
    if (q[k] < 0.0) {
      zfix += 1;
      if (q[k - 1] > 0.0) {
        const double a = q[k - 1] * dp(k - 1), b = -(q[k] * dp(k));
        const double dq = a < b ? a : b;
        q[k] = q[k] + dq / dp(k);
        upper_fix[k] = dq;
      }
      if ((q[k] < 0.0) && (q[k + 1] > 0.0)) {
        const double a = q[k + 1] * dp(k + 1), b = -(q[k] * dp(k));
        const double dq = a < b ? a : b;
        q[k] = q[k] + dq / dp(k);
        lower_fix[k] = dq;
      }
    }
  }
  for (int k = 0; k < km - 1; ++k) {
    if (upper_fix[k + 1] != 0.0) q[k] = q[k] - upper_fix[k + 1] / dp(k);
    dm[k] = q[k] * dp(k);
    dm_pos[k] = dm[k] > 0.0 ? dm[k] : 0.0;
  }
  // fix_bottom
  {
    const int k = km - 1;
    if (lower_fix[k - 1] != 0.0) q[k] = q[k] - (lower_fix[k - 1] / dp(k));
    const double qup = q[k - 1] * dp(k - 1);
    const double qly = -q[k] * dp(k);
    const double dup = qup < qly ? qup : qly;
    if ((q[k] < 0.0) && (q[k - 1] > 0.0)) {
      zfix += 1;
      q[k] = q[k] + (dup / dp(k));
      upper_fix[k] = dup;
    }
    dm[k] = q[k] * dp(k);
    dm_pos[k] = dm[k] > 0.0 ? dm[k] : 0.0;
  }
  {
    const int k = km - 2;
    if (upper_fix[k + 1] != 0.0) {
      q[k] = q[k] - (upper_fix[k + 1] / dp(k));
      dm[k] = q[k] * dp(k);
      dm_pos[k] = dm[k] > 0.0 ? dm[k] : 0.0;
    }
  }
  double sum0 = 0.0, sum1 = 0.0;
  for (int k = 1; k < km; ++k) {
    sum0 += dm[k];
    sum1 += dm_pos[k];
  }
  // final_check
  const double fac = sum0 > 0.0 ? sum0 / sum1 : 0.0;
  if (zfix > 0 && fac > 0.0) {
    for (int k = 1; k < km; ++k) {
      const double v = fac * dm[k] / dp(k);
      q[k] = v > 0.0 ? v : 0.0;
    }
  }
}

struct RemapArgs {
  Dims d;
  fv3b_remap_fields f;
  fv3b_remap_config c;
  const double* ak;
  const double* bk;
  double ptop, akap, zvir;
  int last_step;
};

// Eulerian interface pressure pe2 of level k (0..npz) for surface pressure
// ps: ptop, ak + bk ps, ps (init_pe and pressure_updates, remapping.py
// 33-40, 101-112).
__device__ __forceinline__ double pe2_at(const RemapArgs& a, int k, double ps) {
  if (k == 0) return a.ptop;
  if (k == a.d.nz) return ps;
  return a.ak[k] + a.bk[k] * ps;
}

// the column launches; each kernel body is Body<NK>::run(args, t, i, j)
template <int NK, template <int> class Body>
cudaError_t launch_remap_nk(const RemapArgs& a, int i0, int i1, int j0, int j1, cudaStream_t s) {
  return launch_columns(i0, i1, j0, j1, s, [=] __device__(int t, int i, int j) { Body<NK>::run(a, t, i, j); });
}

template <template <int> class Body>
cudaError_t launch_remap(const RemapArgs& a, int i0, int i1, int j0, int j1, cudaStream_t s) {
  const int K = a.d.nz + 1;
  if (K <= 16) return launch_remap_nk<16, Body>(a, i0, i1, j0, j1, s);
  if (K <= 32) return launch_remap_nk<32, Body>(a, i0, i1, j0, j1, s);
  if (K <= 64) return launch_remap_nk<64, Body>(a, i0, i1, j0, j1, s);
  if (K <= 80) return launch_remap_nk<80, Body>(a, i0, i1, j0, j1, s);
  if (K <= 96) return launch_remap_nk<96, Body>(a, i0, i1, j0, j1, s);
  if (K <= MAXLEV) return launch_remap_nk<MAXLEV, Body>(a, i0, i1, j0, j1, s);
  return cudaErrorInvalidValue;
}

// 2. pt in log pressure: source peln, target log(pe2) (pn2, with pn2(npz)
// = peln(npz), remapping.py:105-134); afterwards peln = pn2 (48-54).
template <int NK>
struct MapPt {
  static __device__ void run(const RemapArgs& a, int t, int i, int j) {
    const Dims& d = a.d;
    const int nz = d.nz;
    const idx_t o = idx3(d, t, i, j, 0), sk = d.sk;
    MapWork<NK> w;
    const double ps = a.f.pe[o + nz * sk];
    for (int k = 0; k <= nz; ++k) {
      w.p1[k] = a.f.peln[o + k * sk];
      w.p2[k] = k < nz ? fm::fm_log(pe2_at(a, k, ps)) : w.p1[nz];
    }
    for (int k = 0; k < nz; ++k) w.a1[k] = a.f.pt[o + k * sk];
    map_column<NK>(w, nz, 1, abs(a.c.kord_tm), 0.0, 184.0);
    for (int k = 0; k < nz; ++k) a.f.pt[o + k * sk] = static_cast<real>(w.q[k]);
    for (int k = 0; k <= nz; ++k) a.f.peln[o + k * sk] = static_cast<real>(w.p2[k]);
  }
};

// 3. the tracers (mapn_tracer.py:67-83): blockIdx.z selects the tracer
template <int NK>
struct MapTracer {
  static __device__ void run(const RemapArgs& a, int t, int i, int j) {
    const Dims& d = a.d;
    const int nz = d.nz;
    const idx_t o = idx3(d, t, i, j, 0), sk = d.sk;
    const int n = blockIdx.z;
    real* qf = a.f.tracers[n];
    MapWork<NK> w;
    const double ps = a.f.pe[o + nz * sk];
    for (int k = 0; k <= nz; ++k) {
      w.p1[k] = a.f.pe[o + k * sk];
      w.p2[k] = pe2_at(a, k, ps);
    }
    for (int k = 0; k < nz; ++k) w.a1[k] = qf[o + k * sk];
    map_column<NK>(w, nz, 0, n == 5 ? 9 : abs(a.c.kord_tr), 0.0, 0.0);
    if (a.c.fill) fix_tracer<NK>(w.q, [&](int k) { return w.p2[k + 1] - w.p2[k]; }, nz);
    for (int k = 0; k < nz; ++k) qf[o + k * sk] = static_cast<real>(w.q[k]);
  }
};

// the tracers: one launch, blockIdx.z selects the tracer
template <int NK>
__global__ void tracer_kernel(RemapArgs a, int i0, int i1, int j0, int j1) {
  const int ncol_i = i1 - i0;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncol_i * (j1 - j0)) return;
  MapTracer<NK>::run(a, blockIdx.y, i0 + c % ncol_i, j0 + c / ncol_i);
}

template <int NK>
cudaError_t launch_tracers_nk(const RemapArgs& a, int i0, int i1, int j0, int j1, cudaStream_t s) {
  const int block = launch_shape().col;
  const int ncol = (i1 - i0) * (j1 - j0);
  dim3 grid((ncol + block - 1) / block, tile_slots(), NTRACER);
  tracer_kernel<NK><<<grid, block, 0, s>>>(a, i0, i1, j0, j1);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_remap_tracers(const RemapArgs& a, int i0, int i1, int j0, int j1, cudaStream_t s) {
  const int K = a.d.nz + 1;
  if (K <= 16) return launch_tracers_nk<16>(a, i0, i1, j0, j1, s);
  if (K <= 32) return launch_tracers_nk<32>(a, i0, i1, j0, j1, s);
  if (K <= 64) return launch_tracers_nk<64>(a, i0, i1, j0, j1, s);
  if (K <= 80) return launch_tracers_nk<80>(a, i0, i1, j0, j1, s);
  if (K <= 96) return launch_tracers_nk<96>(a, i0, i1, j0, j1, s);
  if (K <= MAXLEV) return launch_tracers_nk<MAXLEV>(a, i0, i1, j0, j1, s);
  return cudaErrorInvalidValue;
}

// 4. w with the bottom value wsd (iv -2)
template <int NK>
struct MapW {
  static __device__ void run(const RemapArgs& a, int t, int i, int j) {
    const Dims& d = a.d;
    const int nz = d.nz;
    const idx_t o = idx3(d, t, i, j, 0), sk = d.sk;
    MapWork<NK> w;
    const double ps = a.f.pe[o + nz * sk];
    for (int k = 0; k <= nz; ++k) {
      w.p1[k] = a.f.pe[o + k * sk];
      w.p2[k] = pe2_at(a, k, ps);
    }
    for (int k = 0; k < nz; ++k) w.a1[k] = a.f.w[o + k * sk];
    map_column<NK>(w, nz, -2, abs(a.c.kord_wz), a.f.wsd[idx2(d, t, i, j)], 0.0);
    for (int k = 0; k < nz; ++k) a.f.w[o + k * sk] = static_cast<real>(w.q[k]);
  }
};

// 5. delz (iv 1), then undo_delz_adjust (remapping.py:43-54) with the new
// delp (= dp2)
template <int NK>
struct MapDelz {
  static __device__ void run(const RemapArgs& a, int t, int i, int j) {
    const Dims& d = a.d;
    const int nz = d.nz;
    const idx_t o = idx3(d, t, i, j, 0), sk = d.sk;
    MapWork<NK> w;
    const double ps = a.f.pe[o + nz * sk];
    for (int k = 0; k <= nz; ++k) {
      w.p1[k] = a.f.pe[o + k * sk];
      w.p2[k] = pe2_at(a, k, ps);
    }
    for (int k = 0; k < nz; ++k) w.a1[k] = a.f.delz[o + k * sk];
    map_column<NK>(w, nz, 1, abs(a.c.kord_wz), 0.0, 0.0);
    for (int k = 0; k < nz; ++k) {
      const real dz = static_cast<real>(w.q[k]);
      a.f.delz[o + k * sk] = -dz * a.f.delp[o + k * sk];
    }
  }
};

// 7. u on [is, ie] x [js, je+1]: pressures_mapu (remapping.py:137-159),
// source pe0 = pe (k 0), 0.5 (pe(j-1) + pe) below; target
// ak + 0.5 bk (ps(j-1) + ps) with ps the bottom pe
template <int NK>
struct MapU {
  static __device__ void run(const RemapArgs& a, int t, int i, int j) {
    const Dims& d = a.d;
    const int nz = d.nz;
    const idx_t o = idx3(d, t, i, j, 0), om = idx3(d, t, i, j - 1, 0), sk = d.sk;
    MapWork<NK> w;
    const double pb = a.f.pe[o + nz * sk], pbm = a.f.pe[om + nz * sk];
    w.p1[0] = a.f.pe[o];
    for (int k = 1; k <= nz; ++k) w.p1[k] = 0.5 * ((double)a.f.pe[om + k * sk] + (double)a.f.pe[o + k * sk]);
    for (int k = 0; k <= nz; ++k) {
      const double bkh = 0.5 * a.bk[k];
      w.p2[k] = a.ak[k] + bkh * (pbm + pb);
    }
    for (int k = 0; k < nz; ++k) w.a1[k] = a.f.u[o + k * sk];
    map_column<NK>(w, nz, -1, abs(a.c.kord_mt), 0.0, 0.0);
    for (int k = 0; k < nz; ++k) a.f.u[o + k * sk] = static_cast<real>(w.q[k]);
  }
};

// 8. v on [is, ie+1] x [js, je]: pressures_mapv (162-177), pe3 = ak at k 0
template <int NK>
struct MapV {
  static __device__ void run(const RemapArgs& a, int t, int i, int j) {
    const Dims& d = a.d;
    const int nz = d.nz;
    const idx_t o = idx3(d, t, i, j, 0), om = idx3(d, t, i - 1, j, 0), sk = d.sk;
    MapWork<NK> w;
    const double pb = a.f.pe[o + nz * sk], pbm = a.f.pe[om + nz * sk];
    w.p1[0] = a.f.pe[o];
    w.p2[0] = a.ak[0];
    for (int k = 1; k <= nz; ++k) {
      const double bkh = 0.5 * a.bk[k];
      w.p1[k] = 0.5 * ((double)a.f.pe[om + k * sk] + (double)a.f.pe[o + k * sk]);
      w.p2[k] = a.ak[k] + bkh * (pbm + pb);
    }
    for (int k = 0; k < nz; ++k) w.a1[k] = a.f.v[o + k * sk];
    map_column<NK>(w, nz, -1, abs(a.c.kord_mt), 0.0, 0.0);
    for (int k = 0; k < nz; ++k) a.f.v[o + k * sk] = static_cast<real>(w.q[k]);
  }
};

bool kord_ok(int kord) { return kord >= -10 && kord <= 10 && kord != 0; }

}  // namespace

extern "C" int fv3b_remap_setup(fv3b_ctx* ctx, const double* ak, const double* bk) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && ak && bk, "fv3b_remap_setup: null argument");
  const int nlev = ctx->d.nz + 1;
  FV3B_REQUIRE(nlev <= MAXLEV, "fv3b_remap_setup: npz out of range");
  if (ctx->remap_akbk == nullptr) {
    cudaError_t e = cudaMalloc((void**)&ctx->remap_akbk, sizeof(double) * 2 * MAXLEV);
    FV3B_CHECK(e);
  }
  double host[2 * MAXLEV] = {0};
  for (int k = 0; k < nlev; ++k) {
    host[k] = ak[k];
    host[MAXLEV + k] = bk[k];
  }
  cudaError_t e = cudaMemcpy(ctx->remap_akbk, host, sizeof(host), cudaMemcpyHostToDevice);
  FV3B_CHECK(e);
  if (ctx->sat_tables == nullptr) {
    e = cudaMalloc((void**)&ctx->sat_tables, sizeof(double) * 4 * satadj::TAB_N);
    FV3B_CHECK(e);
    satadj::sat_tables_kernel<<<(satadj::TAB_N + 127) / 128, 128>>>(ctx->sat_tables);
    note_launch();
    e = cudaGetLastError();
    FV3B_CHECK(e);
    e = cudaDeviceSynchronize();
    FV3B_CHECK(e);
  }
  ctx->remap_nlev = nlev;
  return FV3B_OK;
}

extern "C" int fv3b_lagrangian_to_eulerian(fv3b_ctx* ctx, const fv3b_remap_fields* fields,
                                           const fv3b_remap_config* config, const fv3b_sat_adjust_config* sat,
                                           double ptop, double akap, double zvir, double mdt, int kmp,
                                           int last_step, void* stream) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && fields && config, "fv3b_lagrangian_to_eulerian: null argument");
  const fv3b_remap_fields& f = *fields;
  for (int n = 0; n < NTRACER; ++n) FV3B_REQUIRE(f.tracers[n], "fv3b_lagrangian_to_eulerian: null tracer");
  FV3B_REQUIRE(f.pt && f.delp && f.delz && f.peln && f.u && f.v && f.w && f.ua && f.va && f.cappa && f.q_con &&
                   f.pkz && f.pk && f.pe && f.ps && f.wsd,
               "fv3b_lagrangian_to_eulerian: null field");
  FV3B_REQUIRE(ctx->remap_akbk && ctx->remap_nlev == ctx->d.nz + 1,
               "fv3b_lagrangian_to_eulerian: call fv3b_remap_setup first");
  FV3B_REQUIRE(config->kord_tm < 0, "fv3b_lagrangian_to_eulerian: kord_tm >= 0 (map ppm) is not implemented");
  FV3B_REQUIRE(kord_ok(config->kord_tm) && kord_ok(config->kord_tr) && kord_ok(config->kord_wz) &&
                   kord_ok(config->kord_mt),
               "fv3b_lagrangian_to_eulerian: |kord| must be in 1..10");
  FV3B_REQUIRE(ctx->d.nz >= 5, "fv3b_lagrangian_to_eulerian: need npz >= 5");
  if (sat) {
    FV3B_REQUIRE(f.qcld && f.hs, "fv3b_lagrangian_to_eulerian: the saturation adjustment needs qcld and hs");
    FV3B_REQUIRE(!sat->hydrostatic, "fv3b_lagrangian_to_eulerian: hydrostatic is not implemented");
    FV3B_REQUIRE(kmp >= 0 && kmp < ctx->d.nz, "fv3b_lagrangian_to_eulerian: kmp out of range");
    FV3B_REQUIRE(mdt > 0.0, "fv3b_lagrangian_to_eulerian: mdt must be positive");
  }
  const Dims d = ctx->d;
  cudaStream_t st = (cudaStream_t)stream;
  RemapArgs a;
  a.d = d;
  a.f = f;
  a.c = *config;
  a.ak = ctx->remap_akbk;
  a.bk = ctx->remap_akbk + MAXLEV;
  a.ptop = ptop;
  a.akap = akap;
  a.zvir = zvir;
  a.last_step = last_step;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec, nz = d.nz;
  const real zv = static_cast<real>(zvir);
  const real cv_air = RC(CV_AIR_D), cv_vap = RC(CV_VAP_D), c_liq = RC(C_LIQ_D), c_ice = RC(C_ICE_D);
  const real rdgas = RC(RDGAS_D), rdg = RC(RDG_D);
  real* const* tr = f.tracers;  // qvapor, qliquid, qrain, qice, qsnow, qgraupel, ...
  real *qv = tr[0], *qlq = tr[1], *qr = tr[2], *qi = tr[3], *qsn = tr[4], *qg = tr[5];
  const double* akp = a.ak;
  const double* bkp = a.bk;
  // 1. moist_cv_pt_pressure and pn2_pk_delp (remapping.py:57-134), pointwise
  FV3B_CHECK(launch_box(Box{s, e + 1, js, je + 1, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    const real qvk = F3(qv, i, j);
    const real ql = F3(qlq, i, j) + F3(qr, i, j);
    const real qs = F3(qi, i, j) + F3(qsn, i, j) + F3(qg, i, j);
    const real gz = ql + qs;
    const real cvm = (RC(1.0) - (qvk + gz)) * cv_air + qvk * cv_vap + ql * c_liq + qs * c_ice;
    W3(f.q_con, i, j) = gz;
    const real cappa = rdgas / (rdgas + cvm / (RC(1.0) + zv * qvk));
    W3(f.cappa, i, j) = cappa;
    const real dp = F3(f.delp, i, j), dz = F3(f.delz, i, j), pt = F3(f.pt, i, j);
    W3(f.pt, i, j) = pt * static_cast<real>(fm::fm_exp(cappa / (RC(1.0) - cappa) * fm::fm_log(rdg * dp / dz * pt)));
    W3(f.delz, i, j) = -dz / dp;
    // ps, dp2, pk of the Eulerian levels
    const double ps = f.pe[idx3(d, t, i, j, nz)];
    if (k == 0) f.ps[idx2(d, t, i, j)] = static_cast<real>(ps);
    auto pe2 = [&](int kk) -> double {
      if (kk == 0) return ptop;
      if (kk == nz) return ps;
      return akp[kk] + bkp[kk] * ps;
    };
    const double p0 = pe2(k);
    W3(f.delp, i, j) = static_cast<real>(pe2(k + 1) - p0);
    W3(f.pk, i, j) = static_cast<real>(fm::fm_exp(akap * fm::fm_log(p0)));
  }));
  // 2-5. the column remaps
  FV3B_CHECK(launch_remap<MapPt>(a, s, e + 1, js, je + 1, st));
  FV3B_CHECK(launch_remap_tracers(a, s, e + 1, js, je + 1, st));
  FV3B_CHECK(launch_remap<MapW>(a, s, e + 1, js, je + 1, st));
  FV3B_CHECK(launch_remap<MapDelz>(a, s, e + 1, js, je + 1, st));
  // 6. moist_cv_pkz (moist_cv.py:171-194), then moist_pt_last_step (139-162,
  // levels 0..npz, dtmp 0) or adjust_divide_stencil; with the saturation
  // adjustment between them, three launches instead of one
  const bool do_sat = sat != nullptr;
  if (do_sat) {
    FV3B_CHECK(launch_box(Box{s, e + 1, js, je + 1, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
      PT_SETUP(d, t, k);
      const real qvk = F3(qv, i, j);
      const real ql = F3(qlq, i, j) + F3(qr, i, j);
      const real qs = F3(qi, i, j) + F3(qsn, i, j) + F3(qg, i, j);
      const real gz = ql + qs;
      const real cvm = (RC(1.0) - (qvk + gz)) * cv_air + qvk * cv_vap + ql * c_liq + qs * c_ice;
      W3(f.q_con, i, j) = gz;
      const real cappa = rdgas / (rdgas + cvm / (RC(1.0) + zv * qvk));
      W3(f.cappa, i, j) = cappa;
      W3(f.pkz, i, j) = static_cast<real>(
          fm::fm_exp(cappa * fm::fm_log(rdg * F3(f.delp, i, j) / F3(f.delz, i, j) * F3(f.pt, i, j))));
    }));
    // SatAdjust3d.__call__ (saturation_adjustment.py:970-1024): the per-call
    // factors on the host, with the C library's exp (as Python's math.exp)
    satadj::Params prm;
    prm.cfg = *sat;
    prm.mdt = mdt;
    prm.sdt = 0.5 * mdt;
    prm.zvir = zvir;
    prm.fac_i2s = 1.0 - exp(-mdt / sat->tau_i2s);
    prm.fac_v2l = 1.0 - exp(-prm.sdt / sat->tau_v2l);
    prm.fac_r2g = 1.0 - exp(-mdt / sat->tau_r2g);
    prm.fac_l2r = 1.0 - exp(-mdt / sat->tau_l2r);
    const double fac_l2v = 1.0 - exp(-prm.sdt / sat->tau_l2v);
    prm.fac_l2v = fac_l2v < sat->sat_adj0 ? fac_l2v : sat->sat_adj0;
    prm.fac_imlt = 1.0 - exp(-prm.sdt / sat->tau_imlt);
    prm.fac_smlt = 1.0 - exp(-mdt / sat->tau_smlt);
    prm.c_air = CV_AIR_D;
    prm.c_vap = CV_VAP_D;
    prm.d0_vap = prm.c_vap - C_LIQ_D;
    prm.lv00 = satadj::HLV - prm.d0_vap * satadj::TICE;
    prm.last_step = last_step;
    const real* area = ctx->m.area;
    const double* tb = ctx->sat_tables;
    FV3B_CHECK(launch_box(Box{s, e + 1, js, je + 1, kmp, nz}, st, [=] __device__(int t, int i, int j, int k) {
      const idx_t o = idx3(d, t, i, j, k), o2 = idx2(d, t, i, j);
      satadj::Point P;
      P.qv = qv[o];
      P.ql = qlq[o];
      P.qi = qi[o];
      P.qr = qr[o];
      P.qs = qsn[o];
      P.qg = qg[o];
      P.cappa = f.cappa[o];
      P.pt = f.pt[o];
      P.dp = f.delp[o];
      P.delz = f.delz[o];
      P.qa = f.qcld[o];
      P.area = area[o2];
      P.hs = f.hs[o2];
      P.pkz = f.pkz[o];
      P.q_con = f.q_con[o];
      satadj::sat_adjust_point(P, prm, tb);
      qv[o] = static_cast<real>(P.qv);
      qlq[o] = static_cast<real>(P.ql);
      qi[o] = static_cast<real>(P.qi);
      qr[o] = static_cast<real>(P.qr);
      qsn[o] = static_cast<real>(P.qs);
      qg[o] = static_cast<real>(P.qg);
      f.cappa[o] = static_cast<real>(P.cappa);
      f.pt[o] = static_cast<real>(P.pt);
      f.q_con[o] = static_cast<real>(P.q_con);
      f.qcld[o] = static_cast<real>(P.qa);
      f.pkz[o] = static_cast<real>(P.pkz);
    }));
  }
  FV3B_CHECK(launch_box(Box{s, e + 1, js, je + 1, 0, nz + 1}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    const real qvk = F3(qv, i, j);
    if (k < nz && !do_sat) {
      const real ql = F3(qlq, i, j) + F3(qr, i, j);
      const real qs = F3(qi, i, j) + F3(qsn, i, j) + F3(qg, i, j);
      const real gz = ql + qs;
      const real cvm = (RC(1.0) - (qvk + gz)) * cv_air + qvk * cv_vap + ql * c_liq + qs * c_ice;
      W3(f.q_con, i, j) = gz;
      const real cappa = rdgas / (rdgas + cvm / (RC(1.0) + zv * qvk));
      W3(f.cappa, i, j) = cappa;
      W3(f.pkz, i, j) = static_cast<real>(
          fm::fm_exp(cappa * fm::fm_log(rdg * F3(f.delp, i, j) / F3(f.delz, i, j) * F3(f.pt, i, j))));
    }
    if (last_step) {
      const real gz = F3(qlq, i, j) + F3(qr, i, j) + F3(qi, i, j) + F3(qsn, i, j) + F3(qg, i, j);
      const real dtmp = RC(0.0);
      W3(f.pt, i, j) = (F3(f.pt, i, j) + dtmp * F3(f.pkz, i, j)) / ((RC(1.0) + zv * qvk) * (RC(1.0) - gz));
    } else if (k < nz) {
      W3(f.pt, i, j) = F3(f.pt, i, j) / F3(f.pkz, i, j);
    }
  }));
  // 7-8. the D-grid winds
  FV3B_CHECK(launch_remap<MapU>(a, s, e + 1, js, je + 2, st));
  FV3B_CHECK(launch_remap<MapV>(a, s, e + 2, js, je + 1, st));
  // 9. update_ua (remapping.py:180-191) on [is, ie] x [js, je+1] and
  // copy_from_below (194-196) on the compute domain: ua(k) = pe2(k+1), the
  // extra row from row je below level npz-1; pe(k) = ua(k-1)
  FV3B_CHECK(launch_box(Box{s, e + 1, js, je + 2, 0, nz}, st, [=] __device__(int t, int i, int j, int k) {
    // pe2 of the row read: ptop, ak + bk ps, ps with ps its bottom pe (the
    // extra row has only its init_pe values, of which ps is read)
    const int jr = (j == je + 1 && k < nz - 1) ? je : j;
    const double ps = f.pe[idx3(d, t, i, jr, nz)];
    const int kk = k + 1;
    const double v = kk == nz ? ps : akp[kk] + bkp[kk] * ps;
    f.ua[idx3(d, t, i, j, k)] = static_cast<real>(v);
  }));
  FV3B_CHECK(launch_box(Box{s, e + 1, js, je + 1, 1, nz}, st, [=] __device__(int t, int i, int j, int k) {
    f.pe[idx3(d, t, i, j, k)] = f.ua[idx3(d, t, i, j, k - 1)];
  }));
  return FV3B_OK;
}

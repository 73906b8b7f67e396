// The fast saturation adjustment of the vertical remapping: SatAdjust3d
// (fv3core/stencils/saturation_adjustment.py:544-1024), run by
// LagrangianToEulerian when do_sat_adj is set (remapping.py:570-589).
//
// Every point is independent, so the adjustment is one FP64 function of a
// point's values (sat_adjust_point), called by one thread per point.  The
// saturation tables (es over ice / water and their differences,
// qs_table2_fn, qs_tablew_fn, des2_table, desw_table) are functions of an
// integer table index; the reference evaluates them on the fly, here they
// are evaluated once per context by the same device functions (the
// library's exp and log, fmath.h) into a table of every index a point can
// reach (-1 .. 2622), so each lookup returns the value the reference
// computes.  Statement order, branch structure and the
// association of every expression follow the reference, so FP64 results
// agree with the oracle bit for bit.  Nonhydrostatic only (the caller
// rejects hydrostatic); the total-energy fixer (consv_te) is off, as in
// every configuration the remapping accepts.
#pragma once
#include <math.h>

#include "fmath.h"

namespace fv3b {
namespace satadj {

// fv3core/utils/global_constants.py and saturation_adjustment.py:16-39
constexpr double RVGAS = 461.50, RDGAS = 287.05, GRAV = 9.80665, HLV = 2.5e6, HLF = 3.3358e5;
constexpr double C_ICE = 1972.0, C_LIQ = 4.1855e3, CP_VAP = 4.0 * RVGAS, TICE = 273.16;
constexpr double RDG = -RDGAS / GRAV;
constexpr double DC_VAP = CP_VAP - C_LIQ, DC_ICE = C_LIQ - C_ICE;
constexpr double LV0 = HLV - DC_VAP * TICE, LI00 = HLF - DC_ICE * TICE;
constexpr double LI2 = LV0 + LI00, D2ICE = DC_VAP + DC_ICE;
constexpr double E00 = 611.21, TMIN = TICE - 160.0, DELT = 0.1;
constexpr double T_WFR = TICE - 40.0, TICE0 = TICE - 0.01;
constexpr double LAT2 = (HLV + HLF) * (HLV + HLF);
constexpr double QS_LENGTH = 2621;

// the per-call scalars of SatAdjust3d.__call__ (970-1024), host-computed
struct Params {
  double sdt, zvir, fac_i2s, c_air, c_vap, mdt, fac_r2g, fac_smlt, fac_l2r, fac_imlt, d0_vap, lv00, fac_v2l,
      fac_l2v;
  int last_step;
  fv3b_sat_adjust_config cfg;
};

__device__ __forceinline__ double dmin(double a, double b) { return a < b ? a : b; }
__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }
// basic_operations.dim (basic_operations.py:44-46)
__device__ __forceinline__ double dim(double a, double b) { return a - b > 0 ? a - b : 0.0; }

__device__ __forceinline__ double tem_lower(double i) { return TMIN + DELT * i; }
__device__ __forceinline__ double tem_upper(double i) { return 253.16 + DELT * i; }

// q_table_oneline (52-60)
__device__ __forceinline__ double q_table(double dhc, double lhc, double tem) {
  return E00 * fm::fm_exp((dhc * fm::fm_log(tem / TICE) + (tem - TICE) / (tem * TICE) * lhc) / RVGAS);
}
__device__ __forceinline__ double vapor(double tem) { return q_table(DC_VAP, LV0, tem); }
__device__ __forceinline__ double ice(double tem) { return q_table(D2ICE, LI2, tem); }

// qs_table2_fn (94-128)
__device__ double qs_table2(double i) {
  const double tem0 = tem_lower(i);
  if (i == 1599.0) {
    double table = ice(tem0);
    const double tu = tem_upper(i - 1400.0);
    table = (0.05 * (TICE - tu)) * table + (0.05 * (tu - 253.16)) * vapor(tu);
    const double m1 = ice(tem_lower(1598.0));
    const double p1 = vapor(tem_lower(1600.0));
    return 0.25 * (m1 + 2.0 * table + p1);
  }
  if (i == 1600.0) {
    const double table = vapor(tem_upper(i - 1400.0));
    const double m1 = ice(tem_lower(1599.0));
    const double p1 = vapor(tem_lower(1601.0));
    return 0.25 * (m1 + 2.0 * table + p1);
  }
  return i < 1600.0 ? ice(tem0) : vapor(tem0);
}

// qs_tablew_fn (131-134)
__device__ __forceinline__ double qs_tablew(double i) { return vapor(tem_lower(i)); }

// des2_table / desw_table with des_end (137-167): the last index takes the
// difference to its predecessor in table2 (des_end reads qs_table2_fn for
// both tables)
__device__ double des2(double i) {
  const double t = qs_table2(i);
  double des = dmax(0.0, qs_table2(i + 1.0) - t);
  if (i == QS_LENGTH - 1) des = dmax(0.0, t - qs_table2(i - 1.0));
  return des;
}
__device__ double desw(double i) {
  const double t = qs_tablew(i);
  double des = dmax(0.0, qs_tablew(i + 1.0) - t);
  if (i == QS_LENGTH - 1) des = dmax(0.0, t - qs_table2(i - 1.0));
  return des;
}

// the precomputed tables: [4][TAB_N] doubles, index i at offset i + 1
constexpr int TAB_N = 2624;  // indices -1 .. 2622
enum { TAB_W = 0, TAB_2 = 1, DES_W = 2, DES_2 = 3 };

__device__ __forceinline__ double tab_at(const double* tab, int which, double i) {
  int ii = (int)i + 1;
  ii = ii < 0 ? 0 : (ii > TAB_N - 1 ? TAB_N - 1 : ii);
  return tab[which * TAB_N + ii];
}

// fills the tables: one thread per index
__global__ void sat_tables_kernel(double* tab) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= TAB_N) return;
  const double i = (double)(x - 1);
  tab[TAB_W * TAB_N + x] = qs_tablew(i);
  tab[TAB_2 * TAB_N + x] = qs_table2(i);
  tab[DES_W * TAB_N + x] = desw(i);
  tab[DES_2 * TAB_N + x] = des2(i);
}

// ap1_for_wqs2 (454-457)
__device__ __forceinline__ double ap1_of(double ta) {
  const double ap1 = 10.0 * dim(ta, TMIN) + 1.0;
  return dmin(ap1, QS_LENGTH) - 1;
}

// wqs2_fn_w / wqs2_fn_2 with wqsat_and_dqdt (487-519)
template <bool WATER>
__device__ void wqs2(const double* tb, double ta, double den, double& wqsat, double& dqdt) {
  const double ap1 = ap1_of(ta);
  const double it = floor(ap1);
  const double it2 = floor(ap1 - 0.5);
  const double it2_p1 = it2 + 1;
  const int T = WATER ? TAB_W : TAB_2, D = WATER ? DES_W : DES_2;
  const double tab = tab_at(tb, T, it);
  const double des = tab_at(tb, D, it);
  const double des_2 = tab_at(tb, D, it2);
  const double des_p1 = tab_at(tb, D, it2_p1);
  const double es = tab + (ap1 - it) * des;
  const double denom = RVGAS * ta * den;
  wqsat = es / denom;
  dqdt = 10.0 * (des_2 + (ap1 - it2) * (des_p1 - des_2));
  dqdt = dqdt / denom;
}

// compute_cvm (170-172)
__device__ __forceinline__ double cvm_of(double mc_air, double qv, double c_vap, double q_liq, double q_sol) {
  return mc_air + qv * c_vap + q_liq * C_LIQ + q_sol * C_ICE;
}

// update_latent_heat_coefficient_i / _l (398-416)
__device__ __forceinline__ void lat_i(double pt1, double cvm, double& lhi, double& icp2) {
  lhi = LI00 + DC_ICE * pt1;
  icp2 = lhi / cvm;
}
__device__ __forceinline__ void lat(double pt1, double cvm, double lv00, double d0_vap, double& lhl, double& lhi,
                                    double& lcp2, double& icp2) {
  lhl = lv00 + d0_vap * pt1;
  lcp2 = lhl / cvm;
  lat_i(pt1, cvm, lhi, icp2);
}

// minmax_tmp_h20 (202-205)
__device__ __forceinline__ double minmax_tmp(double qa, double qb) { return dmin(-qa, dmax(qb, 0.0)); }

// the point values the stencil reads and writes
struct Point {
  double qv, ql, qi, qr, qs, qg, cappa, pt, dp, delz, qa, area, hs, pkz, q_con;
};

// satadjust (544-932), nonhydrostatic, consv_te off
__device__ void sat_adjust_point(Point& P, const Params& p, const double* tb) {
  const fv3b_sat_adjust_config& c = p.cfg;
  double qv = P.qv, ql = P.ql, qi = P.qi, qr = P.qr, qs = P.qs, qg = P.qg;
  double q_liq = ql + qr;
  double q_sol = qi + qs + qg;
  double qpz = q_liq + q_sol;
  double pt1 = P.pt / ((1.0 + p.zvir * qv) * (1.0 - qpz));
  qpz = qpz + qv;
  const double den = -P.dp / (GRAV * P.delz);
  const double mc_air = (1.0 - qpz) * p.c_air;
  double cvm = cvm_of(mc_air, qv, p.c_vap, q_liq, q_sol);
  double lhi, icp2, lhl, lcp2;
  lat_i(pt1, cvm, lhi, icp2);
  // fix negative cloud ice with snow
  if (qi < 0.0) {
    qs = qs + qi;
    qi = 0.0;
  }
  // melt_cloud_ice (185-199)
  if ((qi > 1.0e-8) && (pt1 > TICE)) {
    const double factmp = p.fac_imlt * (pt1 - TICE) / icp2;
    double sink = qi < factmp ? qi : factmp;
    qi = qi - sink;
    ql = ql + sink;
    q_liq = q_liq + sink;
    q_sol = q_sol - sink;
    cvm = cvm_of(mc_air, qv, p.c_vap, q_liq, q_sol);
    sink = -sink;
    pt1 = pt1 + sink * lhi / cvm;
  }
  lat_i(pt1, cvm, lhi, icp2);
  // fix_negative_snow (208-218)
  if (qs < 0.0) {
    qg = qg + qs;
    qs = 0.0;
  } else if (qg < 0.0) {
    const double tmp = minmax_tmp(qg, qs);
    qg = qg + tmp;
    qs = qs - tmp;
  }
  // fix_negative_cloud_water (221-232)
  if (ql < 0.0) {
    const double tmp = minmax_tmp(ql, qr);
    ql = ql + tmp;
    qr = qr - tmp;
  } else if (qr < 0.0) {
    const double tmp = minmax_tmp(qr, ql);
    ql = ql - tmp;
    qr = qr + tmp;
  }
  // complete_freezing (235-246)
  {
    const double dtmp = TICE - 48.0 - pt1;
    if (ql > 0.0 && dtmp > 0.0) {
      const double sink = dmin(ql, dtmp / icp2);
      ql = ql - sink;
      qi = qi + sink;
      q_liq = q_liq - sink;
      q_sol = q_sol + sink;
      cvm = cvm_of(mc_air, qv, p.c_vap, q_liq, q_sol);
      pt1 = pt1 + sink * lhi / cvm;
    }
  }
  double wqsat, dq2dt;
  wqs2<true>(tb, pt1, den, wqsat, dq2dt);
  lat(pt1, cvm, p.lv00, p.d0_vap, lhl, lhi, lcp2, icp2);
  double diff_ice = dim(TICE, pt1) / 48.0;
  double dimmin = dmin(1.0, diff_ice);
  double tcp3 = lcp2 + icp2 * dimmin;
  double dq0 = (qv - wqsat) / (1.0 + tcp3 * dq2dt);
  double src;
  if (dq0 > 0) {
    src = dmin(c.sat_adj0 * dq0, dmax(c.ql_gen - ql, p.fac_v2l * dq0));
  } else {
    const double factor = -dmin(1, p.fac_l2v * 10.0 * (1.0 - qv / wqsat));
    src = -dmin(ql, factor * dq0);
  }
  // wqsat_correct (443-450)
  qv = qv - src;
  ql = ql + src;
  q_liq = q_liq + src;
  cvm = cvm_of(mc_air, qv, p.c_vap, q_liq, q_sol);
  pt1 = pt1 + src * lhl / cvm;
  lat(pt1, cvm, p.lv00, p.d0_vap, lhl, lhi, lcp2, icp2);
  diff_ice = dim(TICE, pt1) / 48.0;
  dimmin = dmin(1.0, diff_ice);
  tcp3 = lcp2 + icp2 * dimmin;
  if (p.last_step) {
    wqs2<true>(tb, pt1, den, wqsat, dq2dt);
    dq0 = (qv - wqsat) / (1.0 + tcp3 * dq2dt);
    if (dq0 > 0) {
      src = dq0;
    } else {
      const double factor = -dmin(1, p.fac_l2v * 10.0 * (1.0 - qv / wqsat));
      src = -dmin(ql, factor * dq0);
    }
    qv = qv - src;
    ql = ql + src;
    q_liq = q_liq + src;
    cvm = cvm_of(mc_air, qv, p.c_vap, q_liq, q_sol);
    pt1 = pt1 + src * lhl / cvm;
    lat(pt1, cvm, p.lv00, p.d0_vap, lhl, lhi, lcp2, icp2);
  }
  // homogenous_freezing (249-262)
  {
    const double dtmp = T_WFR - pt1;
    if (ql > 0.0 && dtmp > 0.0) {
      double sink = dmin(ql, dtmp / icp2);
      sink = dmin(sink, ql * dtmp * 0.125);
      ql = ql - sink;
      qi = qi + sink;
      q_liq = q_liq - sink;
      q_sol = q_sol + sink;
      cvm = cvm_of(mc_air, qv, p.c_vap, q_liq, q_sol);
      pt1 = pt1 + sink * lhi / cvm;
    }
  }
  lat_i(pt1, cvm, lhi, icp2);
  const double exptc = fm::fm_exp(0.66 * (TICE0 - pt1));
  // heterogeneous_freezing (265-280), dt_bigg = mdt
  {
    const double tc = TICE0 - pt1;
    if (ql > 0.0 && tc > 0.0) {
      double sink = 3.3333e-10 * p.mdt * (exptc - 1.0) * den * (ql * ql);
      sink = dmin(ql, sink);
      sink = dmin(sink, tc / icp2);
      ql = ql - sink;
      qi = qi + sink;
      q_liq = q_liq - sink;
      q_sol = q_sol + sink;
      cvm = cvm_of(mc_air, qv, p.c_vap, q_liq, q_sol);
      pt1 = pt1 + sink * lhi / cvm;
    }
  }
  lat_i(pt1, cvm, lhi, icp2);
  // make_graupel (283-297)
  {
    const double dtmp = (TICE - 0.1) - pt1;
    if (qr > 1e-7 && dtmp > 0.0) {
      const double rf = dtmp * 0.025;
      const double rainfac = rf * rf;
      const double tmp = 1.0 < rainfac ? qr : rainfac * qr;
      const double sink = dmin(tmp, p.fac_r2g * dtmp / icp2);
      qr = qr - sink;
      qg = qg + sink;
      q_liq = q_liq - sink;
      q_sol = q_sol + sink;
      cvm = cvm_of(mc_air, qv, p.c_vap, q_liq, q_sol);
      pt1 = pt1 + sink * lhi / cvm;
    }
  }
  lat_i(pt1, cvm, lhi, icp2);
  // melt_snow (300-320)
  {
    const double dtmp = pt1 - (TICE + 0.1);
    const double dimqs = dim(c.qs_mlt, ql);
    if (qs > 1e-7 && dtmp > 0.0) {
      const double sf = dtmp * 0.1;
      const double snowfac = sf * sf;
      double tmp = 1.0 < snowfac ? qs : snowfac * qs;
      const double sink = dmin(tmp, p.fac_smlt * dtmp / icp2);
      tmp = dmin(sink, dimqs);
      qs = qs - sink;
      ql = ql + tmp;
      qr = qr + sink - tmp;
      q_liq = q_liq + sink;
      q_sol = q_sol - sink;
      cvm = cvm_of(mc_air, qv, p.c_vap, q_liq, q_sol);
      pt1 = pt1 - sink * lhi / cvm;
    }
  }
  // autoconversion_cloud_to_rain (323-329)
  if (ql > c.ql0_max) {
    const double sink = p.fac_l2r * (ql - c.ql0_max);
    qr = qr + sink;
    ql = ql - sink;
  }
  double iqs2, dqsdt;
  wqs2<false>(tb, pt1, den, iqs2, dqsdt);
  const double expsubl = fm::fm_exp(0.875 * fm::fm_log(qi * den));
  lat(pt1, cvm, p.lv00, p.d0_vap, lhl, lhi, lcp2, icp2);
  const double tcp2 = lcp2 + icp2;
  const double adj_fac = p.last_step ? 1.0 : c.sat_adj0;
  // sublimation (332-395)
  src = 0.0;
  if (pt1 < c.t_sub) {
    src = dim(qv, 1e-6);
  } else if (pt1 < TICE0) {
    const double dq = qv - iqs2;
    const double sink = adj_fac * dq / (1.0 + tcp2 * dqsdt);
    double pidep;
    if (qi > 1.0e-8) {
      pidep = p.sdt * dq * 349138.78 * expsubl / (iqs2 * den * LAT2 / (0.0243 * RVGAS * (pt1 * pt1)) + 4.42478e4);
    } else {
      pidep = 0.0;
    }
    if (dq > 0.0) {
      const double tmp = TICE - pt1;
      const double qi_crt = c.qi_lim < 0.1 * tmp ? c.qi_gen * c.qi_lim / den : c.qi_gen * 0.1 * tmp / den;
      const double maxtmp = qi_crt - qi > pidep ? qi_crt - qi : pidep;
      src = sink < maxtmp ? sink : maxtmp;
      src = src < tmp / tcp2 ? src : tmp / tcp2;
    } else {
      const double dimtmp = dim(pt1, c.t_sub);
      pidep = 1.0 < (dimtmp * 0.2) ? pidep : pidep * dimtmp * 0.2;
      src = pidep > sink ? pidep : sink;
      src = src > -qi ? src : -qi;
    }
  }
  qv = qv - src;
  qi = qi + src;
  q_sol = q_sol + src;
  cvm = cvm_of(mc_air, qv, p.c_vap, q_liq, q_sol);
  const double lh = lhl + lhi;
  pt1 = pt1 + src * lh / cvm;
  // virtual temperature and cappa
  const double q_con = q_liq + q_sol;
  double tmp = 1.0 + p.zvir * qv;
  const double pt = pt1 * tmp * (1.0 - q_con);
  tmp = tmp * RDGAS;
  const double cappa = tmp / (tmp + cvm);
  // fix negative graupel with available cloud ice
  if (qg < 0) {
    const double mintmp = dmin(-qg, dmax(0.0, qi));
    qg = qg + mintmp;
    qi = qi - mintmp;
  }
  // autoconversion from cloud ice to snow
  {
    const double qim = c.qi0_max / den;
    if (qi > qim) {
      const double sink = p.fac_i2s * (qi - qim);
      qi = qi - sink;
      qs = qs + sink;
    }
  }
  cvm = mc_air + (qv + q_liq + q_sol) * p.c_vap;
  lat(pt1, cvm, p.lv00, p.d0_vap, lhl, lhi, lcp2, icp2);
  // cloud fraction (do_qa is on, as SatAdjust3d passes it)
  if (p.last_step) {
    if (c.rad_snow) {
      q_sol = c.rad_graupel ? qi + qs + qg : qi + qs;
    } else {
      q_sol = qi;
    }
    q_liq = c.rad_rain ? ql + qr : ql;
    const double q_cond = q_sol + q_liq;
    const double tin = c.tintqs ? pt1 : pt1 - (lcp2 * q_cond + icp2 * q_sol);
    const double ap1 = ap1_of(tin);
    const double it = floor(ap1);
    const double wqs1 = (tab_at(tb, TAB_W, it) + (ap1 - it) * tab_at(tb, DES_W, it)) / (RVGAS * tin * den);
    const double iqs1 = (tab_at(tb, TAB_2, it) + (ap1 - it) * tab_at(tb, DES_2, it)) / (RVGAS * tin * den);
    double qstar;
    if (tin < T_WFR) {
      qstar = iqs1;
    } else if (tin >= TICE) {
      qstar = wqs1;
    } else {
      const double rqi = q_cond > 1e-6 ? q_sol / q_cond : (TICE - tin) / (TICE - T_WFR);
      qstar = rqi * iqs1 + (1.0 - rqi) * wqs1;
    }
    const double mindw = dmin(1.0, fabs(P.hs) / (10.0 * GRAV));
    const double dw = c.dw_ocean + (c.dw_land - c.dw_ocean) * mindw;
    const double dbl_sqrt_area = dw * sqrt(sqrt(P.area) / 100.0e3);
    const double maxtmp = dmax(0.01, dbl_sqrt_area);
    const double hvar = dmin(0.2, maxtmp);
    const double rh = qpz / qstar;
    double qa;
    if (rh > 0.75 && qpz > 1.0e-8) {
      const double dq = hvar * qpz;
      const double q_plus = qpz + dq;
      const double q_minus = qpz - dq;
      if (c.icloud_f == 2) {
        if (qpz > qstar) {
          qa = 1.0;
        } else if ((qstar < q_plus) && (q_cond > 1.0e-8)) {
          const double r = (q_plus - qstar) / dq;
          qa = dmin(1.0, r * r);
        } else {
          qa = 0.0;
        }
      } else {
        if (qstar < q_minus) {
          qa = 1.0;
        } else {
          if (qstar < q_plus) {
            qa = c.icloud_f == 0 ? (q_plus - qstar) / (dq + dq) : (q_plus - qstar) / (2.0 * dq * (1.0 - q_cond));
          } else {
            qa = 0.0;
          }
          if (q_cond > 1.0e-8) qa = dmax(c.cld_min, qa);
          qa = dmin(1, qa);
        }
      }
    } else {
      qa = 0.0;
    }
    P.qa = qa;
  }
  P.pkz = fm::fm_exp(cappa * fm::fm_log(RDG * P.dp / P.delz * pt));
  P.qv = qv;
  P.ql = ql;
  P.qi = qi;
  P.qr = qr;
  P.qs = qs;
  P.qg = qg;
  P.cappa = cappa;
  P.pt = pt;
  P.q_con = q_con;
}

}  // namespace satadj
}  // namespace fv3b

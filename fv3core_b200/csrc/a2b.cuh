// Fourth-order A-grid to B-grid interpolation (fv3core/stencils/a2b_ord4.py,
// AGrid2BGridFourthOrder.__call__ 606-676) on levels [k0, k1), three passes:
// corner/edge values, PPM volume means, interior interpolation.
#pragma once
#include "ctx.cuh"
#include "stencil.cuh"

namespace fv3b {

namespace a2b {
constexpr real C1 = RC(2.0) / RC(3.0), C2 = -RC(1.0) / RC(6.0);
constexpr real B1 = RC(7.0) / RC(12.0), B2 = -RC(1.0) / RC(12.0);
constexpr real A1 = RC(9.0) / RC(16.0), A2 = -RC(1.0) / RC(16.0);

// extrap_corner (a2b_ord4.py:45-57) with the grid-only ratio x1 / (x2 - x1)
// of its great-circle distances precomputed (fv3b_metrics.a2b_extrap)
__device__ __forceinline__ real extrap(real ratio, real qa, real qb) { return qa + ratio * (qa - qb); }

// ppm_volume_mean edge formulas (a2b_ord4.py:340-451) along one axis; L(o)
// reads qin at offset o, G(o) the A-grid spacing.
template <typename L, typename Gs>
__device__ __forceinline__ real vm_edge1(const L& q, const Gs& g) {
  real g_in = g(1) / g(0), g_ou = g(-2) / g(-1);
  return RC(0.5) * (((RC(2.0) + g_in) * q(0) - q(1)) / (RC(1.0) + g_in) + ((RC(2.0) + g_ou) * q(-1) - q(-2)) / (RC(1.0) + g_ou));
}
template <typename L, typename Gs>
__device__ __forceinline__ real vm_edge2(const L& q, const Gs& g) {
  real g_in = g(0) / g(-1), g_ou = g(-3) / g(-2);
  real left = RC(0.5) * (((RC(2.0) + g_in) * q(-1) - q(0)) / (RC(1.0) + g_in) + ((RC(2.0) + g_ou) * q(-2) - q(-3)) / (RC(1.0) + g_ou));
  real right = B2 * (q(-1) + q(2)) + B1 * (q(0) + q(1));
  return (RC(3.0) * (g_in * q(-1) + q(0)) - (g_in * left + right)) / (RC(2.0) + RC(2.0) * g_in);
}
template <typename L, typename Gs>
__device__ __forceinline__ real vm_edge3(const L& q, const Gs& g) {
  real g_in = g(-2) / g(-1), g_ou = g(1) / g(0);
  return RC(0.5) * (((RC(2.0) + g_in) * q(-1) - q(-2)) / (RC(1.0) + g_in) + ((RC(2.0) + g_ou) * q(0) - q(1)) / (RC(1.0) + g_ou));
}
template <typename L, typename Gs>
__device__ __forceinline__ real vm_edge4(const L& q, const Gs& g) {
  real g_in = g(-1) / g(0), g_ou = g(2) / g(1);
  real right = RC(0.5) * (((RC(2.0) + g_in) * q(0) - q(-1)) / (RC(1.0) + g_in) + ((RC(2.0) + g_ou) * q(1) - q(2)) / (RC(1.0) + g_ou));
  real left = B2 * (q(-3) + q(0)) + B1 * (q(-2) + q(-1));
  return (RC(3.0) * (q(-1) + g_in * q(0)) - (g_in * right + left)) / (RC(2.0) + RC(2.0) * g_in);
}
template <typename L, typename Gs>
__device__ __forceinline__ real volume_mean(const L& q, const Gs& g, int pos, int s, int e) {
  // statement order of ppm_volume_mean_x: general, s, s+1, e+1, e
  if (pos == e) return vm_edge4(q, g);
  if (pos == e + 1) return vm_edge3(q, g);
  if (pos == s + 1) return vm_edge2(q, g);
  if (pos == s) return vm_edge1(q, g);
  return B2 * (q(-2) + q(1)) + B1 * (q(-1) + q(0));
}
}  // namespace a2b

template <int AXIS>
struct A2BLine {
  const real* p;
  idx_t base, step;
  __device__ __forceinline__ real operator()(int o) const { return p[base + o * step]; }
};

inline cudaError_t a2b_ord4(const Dims d, const fv3b_metrics g, real* qin, real* qout, real* qx, real* qy,
                            real* edges, int k0, int k1, cudaStream_t st, bool replace = false) {
  using namespace a2b;
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec, h = d.h, n = d.n;
  cudaError_t err;
  if (k1 <= k0) return cudaSuccess;
  // corners (a2b_ord4.py:60-235, 616-654) and edges (313-336, 678-695)
  // one thread per boundary point of [is, ie+1] x [js, je+1]: the south and
  // north rows (corners included), then the west and east columns
  err = launch_box(Box{0, 4 * (n + 1), 0, 1, k0, k1}, st, [=] __device__(int t, int p, int, int k) {
    PT_SETUP(d, t, k);
    const int side = p / (n + 1), a = p % (n + 1);
    if (side >= 2 && (a == 0 || a == n)) return;  // corners belong to the rows
    const int i = side < 2 ? s + a : (side == 2 ? s : e + 1);
    const int j = side == 0 ? js : (side == 1 ? je + 1 : js + a);
    bool wcol = i == s, ecol = i == e + 1, srow = j == js, nrow = j == je + 1;
    real v;
    if ((wcol || ecol) && (srow || nrow)) {
      // offsets (near, far) of the three extrapolations; the reference's
      // _nw/_se stencils run at the (ie+1, js) / (is, je+1) corners
      int o[3][4];
      if (wcol && srow) {
        int oo[3][4] = {{0, 0, 1, 1}, {-1, 0, -2, 1}, {0, -1, 1, -2}};
        memcpy(o, oo, sizeof(o));
      } else if (ecol && srow) {
        int oo[3][4] = {{-1, 0, -2, 1}, {-1, -1, -2, -2}, {0, 0, 1, 1}};
        memcpy(o, oo, sizeof(o));
      } else if (ecol && nrow) {
        int oo[3][4] = {{-1, -1, -2, -2}, {0, -1, 1, -2}, {-1, 0, -2, 1}};
        memcpy(o, oo, sizeof(o));
      } else {
        int oo[3][4] = {{0, -1, 1, -2}, {-1, -1, -2, -2}, {0, 0, 1, 1}};
        memcpy(o, oo, sizeof(o));
      }
      const int corner = (wcol && srow) ? 0 : (ecol && srow) ? 1 : (ecol && nrow) ? 2 : 3;
      const real* ratio = g.a2b_extrap + (t * 4 + corner) * 3;
      real ec[3];
      for (int m = 0; m < 3; ++m) {
        int i1 = i + o[m][0], j1 = j + o[m][1], i2 = i + o[m][2], j2 = j + o[m][3];
        ec[m] = extrap(ratio[m], F3(qin, i1, j1), F3(qin, i2, j2));
      }
      v = (ec[0] + ec[1] + ec[2]) * (RC(1.0) / RC(3.0));
    } else if (wcol || ecol) {
      const real* ef = wcol ? g.edge_w : g.edge_e;
      real wgt = ef[t * (n + 1) + (j - h)];
      auto q2 = [&](int jj) {
        return (F3(qin, i - 1, jj) * F2(g.dxa, i, jj) + F3(qin, i, jj) * F2(g.dxa, i - 1, jj)) /
               (F2(g.dxa, i - 1, jj) + F2(g.dxa, i, jj));
      };
      v = wgt * q2(j - 1) + (RC(1.0) - wgt) * q2(j);
    } else {
      const real* ef = srow ? g.edge_s : g.edge_n;
      real wgt = ef[t * (n + 1) + (i - h)];
      auto q1 = [&](int ii) {
        return (F3(qin, ii, j - 1) * F2(g.dya, ii, j) + F3(qin, ii, j) * F2(g.dya, ii, j - 1)) /
               (F2(g.dya, ii, j - 1) + F2(g.dya, ii, j));
      };
      v = wgt * q1(i - 1) + (RC(1.0) - wgt) * q1(i);
    }
    W3(qout, i, j) = v;
    W3(edges, i, j) = v;
  });
  if (err != cudaSuccess) return err;
  // ppm_volume_mean_x on [is, ie+1] x [js-2, je+2], _y on [is-2, ie+2] x [js, je+1];
  // the columns of the interior formula (is+2 .. ie-1) in warps of their own
  err = launch_box_split(Box{s - 2, e + 3, js - 2, je + 3, k0, k1}, s + 2, e, st,
                         [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    idx_t b = idx3(d, t, i, j, k);
    idx_t b2 = idx2(d, t, i, j);
    if (i >= s && i < e + 2) {
      A2BLine<0> q{qin, b, 1};
      A2BLine<0> gx{g.dxa, b2, 1};
      W3(qx, i, j) = volume_mean(q, gx, i, s, e);
    }
    if (j >= js && j < je + 2) {
      A2BLine<1> q{qin, b, d.sj};
      A2BLine<1> gy{g.dya, b2, (idx_t)d.ni};
      W3(qy, i, j) = volume_mean(q, gy, j, js, je);
    }
  });
  if (err != cudaSuccess) return err;
  // a2b_interpolation (a2b_ord4.py:286-310) on interior cell corners, the
  // columns without the edge corrections (is+2 .. ie-1) in warps of their own
  err = launch_box_split(Box{s + 1, e + 1, js + 1, je + 1, k0, k1}, s + 2, e, st,
                         [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    real qxx = A2 * (F3(qx, i, j - 2) + F3(qx, i, j + 1)) + A1 * (F3(qx, i, j - 1) + F3(qx, i, j));
    real qyy = A2 * (F3(qy, i - 2, j) + F3(qy, i + 1, j)) + A1 * (F3(qy, i - 1, j) + F3(qy, i, j));
    if (j == js + 1) {
      real up = A2 * (F3(qx, i, j - 1) + F3(qx, i, j + 2)) + A1 * (F3(qx, i, j) + F3(qx, i, j + 1));
      qxx = C1 * (F3(qx, i, j - 1) + F3(qx, i, j)) + C2 * (F3(edges, i, j - 1) + up);
    }
    if (j == je) {
      real lo = A2 * (F3(qx, i, j - 3) + F3(qx, i, j)) + A1 * (F3(qx, i, j - 2) + F3(qx, i, j - 1));
      qxx = C1 * (F3(qx, i, j - 1) + F3(qx, i, j)) + C2 * (F3(edges, i, j + 1) + lo);
    }
    if (i == s + 1) {
      real right = A2 * (F3(qy, i - 1, j) + F3(qy, i + 2, j)) + A1 * (F3(qy, i, j) + F3(qy, i + 1, j));
      qyy = C1 * (F3(qy, i - 1, j) + F3(qy, i, j)) + C2 * (F3(edges, i - 1, j) + right);
    }
    if (i == e) {
      real left = A2 * (F3(qy, i - 3, j) + F3(qy, i, j)) + A1 * (F3(qy, i - 2, j) + F3(qy, i - 1, j));
      qyy = C1 * (F3(qy, i - 1, j) + F3(qy, i, j)) + C2 * (F3(edges, i + 1, j) + left);
    }
    W3(qout, i, j) = RC(0.5) * (qxx + qyy);
  });
  if (err != cudaSuccess || !replace) return err;
  return launch_box(Box{s, e + 2, js, je + 2, k0, k1}, st, [=] __device__(int t, int i, int j, int k) {
    PT_SETUP(d, t, k);
    W3(qin, i, j) = F3(qout, i, j);
  });
}

}  // namespace fv3b

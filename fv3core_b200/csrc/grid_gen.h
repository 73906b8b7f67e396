// Cubed-sphere grid generation: the metric terms of all six tiles computed
// point by point, for the device (csrc/grid_gen.cu) and for the host (a CPU
// test compiles this header with g++ and compares it with the numpy
// generator fv3core_b200/grid.py, which it restates operation for
// operation).
//
// The reference generates these fields in MetricTerms
// (fv3core/grid/generation.py:66-2137, gnomonic.py, geometry.py), on the
// host, one MPI rank per sub-tile, with halo updates between the steps.
// Here every output point is a closed-form function of the cube geometry:
// the corner points of each face are the gnomonic projection of an
// equiangular lattice; an edge-halo corner point is the neighbouring
// tile's point (the same gather as the dynamics' halo update); the 3x3
// cube-corner blocks extend the local lattice.  Lengths are great-circle
// distances times the radius, areas spherical excess times radius squared,
// angles those between great-circle tangents.  So a kernel computes each
// point on its own, with no halo update and no intermediate array.
//
// Layout: a 2-D field is [6][m][m], m = n + 2h + 1, storage indices equal
// to the reference's (compute domain from h); the device writes it with i
// fastest ([t][j][i]), the layout of the stage kernels' metric fields.
#pragma once
#include <math.h>

#include "dims.h"
#include "halo.cuh"

namespace fv3b {
namespace gg {

#define GG_HD __host__ __device__ inline

struct V3 {
  double x, y, z;
};
GG_HD V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
GG_HD V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
GG_HD V3 scale(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
GG_HD double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
GG_HD V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
GG_HD double norm(V3 a) { return sqrt(dot(a, a)); }
GG_HD V3 normalize(V3 a) {
  const double r = norm(a);
  return {a.x / r, a.y / r, a.z / r};
}
// numpy's maximum / minimum: NaN in either argument gives NaN
GG_HD double np_max(double a, double b) { return (a != a || b != b) ? a + b : (a > b ? a : b); }
GG_HD double np_min(double a, double b) { return (a != a || b != b) ? a + b : (a < b ? a : b); }

constexpr double PI = 3.14159265358979323846;
constexpr double TINY = 1.0e-30;

// face frames (centre, local x axis, local y axis), right handed, in the
// tile order of the halo connectivity
GG_HD void face_frame(int t, V3& c, V3& ex, V3& ey) {
  switch (t % 6) {
    case 0: c = {1, 0, 0}; ex = {0, 1, 0}; ey = {0, 0, 1}; break;
    case 1: c = {0, 1, 0}; ex = {-1, 0, 0}; ey = {0, 0, 1}; break;
    case 2: c = {0, 0, 1}; ex = {-1, 0, 0}; ey = {0, -1, 0}; break;
    case 3: c = {-1, 0, 0}; ex = {0, 0, -1}; ey = {0, -1, 0}; break;
    case 4: c = {0, -1, 0}; ex = {0, 0, -1}; ey = {1, 0, 0}; break;
    default: c = {0, 0, -1}; ex = {0, 1, 0}; ey = {1, 0, 0}; break;
  }
}

// Grid parameters of one generation.
struct Grid {
  Dims d;         // n, h and the index helpers of the halo map
  int n, h, m;    // m = n + 2h + 1 corner points per axis
  int lattice;    // 0 equiangular, 1 equal spacing along the edges (gnomonic_ed)
  double radius;
  double omega;
};

// face coordinate (1 at the face's edges) of lattice line a (offset from
// the first compute line): tan of equally spaced angles from the face
// centre (equiangular), or sqrt(2) tan of latitudes equally spaced along
// the edge meridian over [-asin(1/sqrt(3)), asin(1/sqrt(3))] (the
// reference's gnomonic_ed, fv3core/grid/global_setup.py:42-85)
GG_HD double face_coordinate(const Grid& g, int a) {
  if (g.lattice == 1) {
    const double alpha = asin(pow(3.0, -0.5));
    const double dely = 2.0 * alpha / g.n;
    return sqrt(2.0) * tan(-alpha + a * dely);
  }
  const double dal = 0.5 * PI / g.n;
  return tan(-0.25 * PI + a * dal);
}

// unit vector of lattice point (a, b) (offsets from the first compute
// corner) of face t: c + u(a) ex + u(b) ey, normalised
GG_HD V3 face_point(const Grid& g, int t, int a, int b) {
  const double ta = face_coordinate(g, a), tb = face_coordinate(g, b);
  V3 c, ex, ey;
  face_frame(t, c, ex, ey);
  const V3 p = {(c.x + ta * ex.x) + tb * ey.x, (c.y + ta * ex.y) + tb * ey.y, (c.z + ta * ex.z) + tb * ey.z};
  return normalize(p);
}

// corner point at storage (i, j), i, j in [0, m): an edge-halo point is the
// neighbouring tile's point it coincides with
GG_HD V3 corner(const Grid& g, int t, int i, int j) {
  const int sx[2] = {0, 0}, sy[2] = {0, 0};
  HaloSource src;
  if (halo_source(g.d, t, i, j, 0, sx, sy, g.h, src)) return face_point(g, src.t, src.i - g.h, src.j - g.h);
  return face_point(g, t, i - g.h, j - g.h);
}

// cell centre (A grid) of cell (i, j), i, j in [0, m - 1)
GG_HD V3 center(const Grid& g, int t, int i, int j) {
  return normalize(add(add(add(corner(g, t, i, j), corner(g, t, i + 1, j)), corner(g, t, i, j + 1)),
                       corner(g, t, i + 1, j + 1)));
}

// great-circle angle between unit vectors
GG_HD double gc_dist(V3 p, V3 q) { return atan2(norm(cross(p, q)), dot(p, q)); }

// unit tangent at p of the great circle towards q (NaN where q == p)
GG_HD V3 tangent(V3 p, V3 q) {
  const double s = dot(q, p);
  const V3 t = {q.x - s * p.x, q.y - s * p.y, q.z - s * p.z};
  const double r = norm(t);
  if (!(r > 0.0)) {
    const double nan = NAN;
    return {nan, nan, nan};
  }
  return {t.x / r, t.y / r, t.z / r};
}

GG_HD double cos_angle(V3 p, V3 q1, V3 q2) { return dot(tangent(p, q1), tangent(p, q2)); }

// spherical excess of a triangle (vector form of L'Huilier's theorem)
GG_HD double tri_area(V3 a, V3 b, V3 c) {
  const double num = fabs(dot(a, cross(b, c)));
  const double den = ((1.0 + dot(a, b)) + dot(b, c)) + dot(c, a);
  return 2.0 * atan2(num, den);
}
GG_HD double quad_area(V3 p1, V3 p2, V3 p3, V3 p4) { return tri_area(p1, p2, p3) + tri_area(p1, p3, p4); }

GG_HD void lonlat(V3 p, double& lon, double& lat) {
  lon = atan2(p.y, p.x);
  if (lon < 0) lon = lon + 2.0 * PI;
  lat = asin(np_min(np_max(p.z, -1.0), 1.0));
}

// The four corners, centre and edge midpoints of cell (i, j).
struct Cell {
  V3 p00, p10, p01, p11, c, mw, me, ms, mn;
};
GG_HD Cell cell(const Grid& g, int t, int i, int j) {
  Cell k;
  k.p00 = corner(g, t, i, j);
  k.p10 = corner(g, t, i + 1, j);
  k.p01 = corner(g, t, i, j + 1);
  k.p11 = corner(g, t, i + 1, j + 1);
  k.c = normalize(add(add(add(k.p00, k.p10), k.p01), k.p11));
  k.mw = normalize(add(k.p00, k.p01));
  k.me = normalize(add(k.p10, k.p11));
  k.ms = normalize(add(k.p00, k.p10));
  k.mn = normalize(add(k.p01, k.p11));
  return k;
}

// cos of the angle between the local x and y directions at the west (1),
// south (2), east (3), north (4) edge midpoint and the centre (5) of a cell,
// before the cube-corner convention (cos_sg / sin_sg of FV3)
GG_HD double cos_sg_raw(const Grid& g, int k, int t, int i, int j) {
  const Cell c = cell(g, t, i, j);
  switch (k) {
    case 1: return cos_angle(c.mw, c.c, c.p01);
    case 2: return cos_angle(c.ms, c.p10, c.c);
    case 3: return cos_angle(c.me, sub(scale(2.0, c.me), c.c), c.p11);
    case 4: return cos_angle(c.mn, c.p11, sub(scale(2.0, c.mn), c.c));
    default: return cos_angle(c.c, c.me, c.mn);
  }
}
GG_HD double sin_of(double cs) { return np_min(1.0, sqrt(np_max(0.0, 1.0 - cs * cs))); }

// cos_sg (sine = false) or sin_sg (sine = true) of cell (i, j), i, j in
// [0, m - 1), with FV3's convention in the 3x3 cube-corner halo blocks
// (which have no cell of their own; fv3core/grid/geometry.py:430-512): the
// block holds sin 1e-8, cos 1e8, except the edge angles facing the
// adjacent edge halos, rotated in from those halo cells
GG_HD double sg_cell(const Grid& g, int k, bool sine, int t, int i, int j) {
  const int h = g.h, N = g.m - 1;
  const bool lo_i = i < h, hi_i = i >= N - h, lo_j = j < h, hi_j = j >= N - h;
  auto raw = [&](int kk, int ii, int jj) {
    const double cs = cos_sg_raw(g, kk, t, ii, jj);
    return sine ? sin_of(cs) : cs;
  };
  if (!((lo_i || hi_i) && (lo_j || hi_j))) return raw(k, i, j);
  // rotations into the block, a in [0, h)
  if (lo_i && lo_j) {  // south-west
    if (k == 3 && i == h - 1) return raw(2, j, h);
    if (k == 4 && j == h - 1) return raw(1, h, i);
  } else if (lo_i && hi_j) {  // north-west
    if (k == 2 && j == N - h) return raw(1, h, N - 1 - i);
    if (k == 3 && i == h - 1) return raw(4, N - 1 - j, N - 1 - h);
  } else if (hi_i && lo_j) {  // south-east
    if (k == 1 && i == N - h) return raw(2, N - 1 - j, h);
    if (k == 4 && j == h - 1) return raw(3, N - 1 - h, N - 1 - i);
  } else {  // north-east
    if (k == 1 && i == N - h) return raw(4, N - 1 - (N - 1 - j), N - 1 - h);
    if (k == 2 && j == N - h) return raw(3, N - 1 - h, N - 1 - (N - 1 - i));
  }
  return sine ? 1.0e-8 : 1.0e8;
}

// the same, padded to [m][m] with zeros
GG_HD double sg(const Grid& g, int k, bool sine, int t, int i, int j) {
  if (i >= g.m - 1 || j >= g.m - 1) return 0.0;
  return sg_cell(g, k, sine, t, i, j);
}

// The 2-D fields, in the order of include/fv3core_b200.h's
// FV3B_GRID_FIELD_NAMES.
enum GridField {
  GF_DX, GF_DY, GF_DXA, GF_DYA, GF_DXC, GF_DYC,
  GF_RDX, GF_RDY, GF_RDXA, GF_RDYA, GF_RDXC, GF_RDYC,
  GF_AREA, GF_RAREA, GF_AREA_C, GF_RAREA_C,
  GF_SIN_SG1, GF_SIN_SG2, GF_SIN_SG3, GF_SIN_SG4, GF_SIN_SG5,
  GF_COS_SG1, GF_COS_SG2, GF_COS_SG3, GF_COS_SG4, GF_COS_SG5,
  GF_COSA, GF_SINA, GF_RSINA,
  GF_COSA_U, GF_COSA_V, GF_COSA_S, GF_SINA_U, GF_SINA_V, GF_RSIN_U, GF_RSIN_V, GF_RSIN2,
  GF_DEL6_U, GF_DEL6_V, GF_DIVG_U, GF_DIVG_V,
  GF_FC, GF_F0, GF_AGRID1, GF_AGRID2, GF_BGRID1, GF_BGRID2,
  GF_A11, GF_A12, GF_A21, GF_A22,
  GF_COUNT
};

// lengths (times the radius); zero outside the points the numpy generator
// fills (its arrays are padded to [m][m])
GG_HD double dx_at(const Grid& g, int t, int i, int j) {
  if (i >= g.m - 1) return 0.0;
  return gc_dist(corner(g, t, i, j), corner(g, t, i + 1, j)) * g.radius;
}
GG_HD double dy_at(const Grid& g, int t, int i, int j) {
  if (j >= g.m - 1) return 0.0;
  return gc_dist(corner(g, t, i, j), corner(g, t, i, j + 1)) * g.radius;
}
GG_HD double dxc_at(const Grid& g, int t, int i, int j) {
  const int N = g.m - 1;
  const int ii = i == 0 ? 1 : i;  // column 0 repeats column 1
  if (!(ii < N && j < N)) return 0.0;
  return gc_dist(center(g, t, ii - 1, j), center(g, t, ii, j)) * g.radius;
}
GG_HD double dyc_at(const Grid& g, int t, int i, int j) {
  const int N = g.m - 1;
  const int jj = j == 0 ? 1 : j;
  if (!(i < N && jj < N)) return 0.0;
  return gc_dist(center(g, t, i, jj - 1), center(g, t, i, jj)) * g.radius;
}
GG_HD double area_at(const Grid& g, int t, int i, int j) {
  if (i >= g.m - 1 || j >= g.m - 1) return 0.0;
  return quad_area(corner(g, t, i, j), corner(g, t, i + 1, j), corner(g, t, i + 1, j + 1), corner(g, t, i, j + 1)) *
         g.radius * g.radius;
}
// area of the dual (B-grid) cell around corner (i, j): the quadrilateral of
// the four surrounding centres; row and column 0 repeat 1
GG_HD double area_c_at(const Grid& g, int t, int i, int j) {
  const int N = g.m - 1;
  const int jj = j == 0 ? 1 : j;
  const int ii = i == 0 ? 1 : i;
  if (!(ii < N && jj >= 1 && jj < N)) return 0.0;
  return quad_area(center(g, t, ii - 1, jj - 1), center(g, t, ii, jj - 1), center(g, t, ii, jj),
                   center(g, t, ii - 1, jj)) *
         g.radius * g.radius;
}
// the angle between the grid lines through corner (i, j)
GG_HD double cosa_at(const Grid& g, int t, int i, int j) {
  if (!(i >= 1 && i < g.m - 1 && j >= 1 && j < g.m - 1)) return 0.0;
  const V3 p = corner(g, t, i, j);
  const double cfwd = cos_angle(p, corner(g, t, i + 1, j), corner(g, t, i, j + 1));
  const double cbwd =
      cos_angle(p, sub(scale(2.0, p), corner(g, t, i - 1, j)), sub(scale(2.0, p), corner(g, t, i, j - 1)));
  return 0.5 * (cfwd + cbwd);
}
GG_HD double sina_u_at(const Grid& g, int t, int i, int j) {
  return i >= 1 ? 0.5 * (sg(g, 3, true, t, i - 1, j) + sg(g, 1, true, t, i, j)) : 1.0;
}
GG_HD double sina_v_at(const Grid& g, int t, int i, int j) {
  return j >= 1 ? 0.5 * (sg(g, 4, true, t, i, j - 1) + sg(g, 2, true, t, i, j)) : 1.0;
}
GG_HD double recip_pos(double x) { return x > 0.0 ? 1.0 / x : 0.0; }
// distance between the west and east (dir 0) or south and north (dir 1)
// edge midpoints of cell (i, j)
GG_HD double dxya_at(const Grid& g, int dir, int t, int i, int j) {
  if (i >= g.m - 1 || j >= g.m - 1) return 0.0;
  const Cell c = cell(g, t, i, j);
  return (dir == 0 ? gc_dist(c.mw, c.me) : gc_dist(c.ms, c.mn)) * g.radius;
}

// lon / lat of cell centre (i, j), zero outside the cells
GG_HD void lonlat_a(const Grid& g, int t, int i, int j, double& lon, double& lat) {
  lon = 0.0;
  lat = 0.0;
  if (i >= g.m - 1 || j >= g.m - 1) return;
  lonlat(center(g, t, i, j), lon, lat);
}

// cubed-to-latlon coefficient q (0: a11, 1: a12, 2: a21, 3: a22) of cell
// (i, j): the projections of the grid directions towards the east and the
// north edge midpoints on the local east and north unit vectors, over
// sin_sg5 (fv3core/grid/geometry.py:588-601)
GG_HD double c2l_at(const Grid& g, int q, int t, int i, int j) {
  if (i >= g.m - 1 || j >= g.m - 1) return 0.0;
  const Cell c = cell(g, t, i, j);
  double lon, lat;
  lonlat(c.c, lon, lat);
  const V3 east = {-sin(lon), cos(lon), 0.0};
  const V3 north = {-sin(lat) * cos(lon), -sin(lat) * sin(lon), cos(lat)};
  const V3 ec1 = tangent(c.c, c.me), ec2 = tangent(c.c, c.mn);
  const double s5 = sg_cell(g, 5, true, t, i, j);
  switch (q) {
    case 0: return 0.5 * dot(ec2, north) / s5;
    case 1: return -0.5 * dot(ec1, north) / s5;
    case 2: return -0.5 * dot(ec2, east) / s5;
    default: return 0.5 * dot(ec1, east) / s5;
  }
}

// Field f at storage point (i, j) of tile t, i, j in [0, m).
GG_HD double field_at(const Grid& g, int f, int t, int i, int j) {
  const int hs = g.h, he = g.h + g.n;
  switch (f) {
    case GF_DX: return dx_at(g, t, i, j);
    case GF_DY: return dy_at(g, t, i, j);
    case GF_DXA: return dxya_at(g, 0, t, i, j);
    case GF_DYA: return dxya_at(g, 1, t, i, j);
    case GF_DXC: return dxc_at(g, t, i, j);
    case GF_DYC: return dyc_at(g, t, i, j);
    case GF_RDX: return recip_pos(dx_at(g, t, i, j));
    case GF_RDY: return recip_pos(dy_at(g, t, i, j));
    case GF_RDXA: return recip_pos(dxya_at(g, 0, t, i, j));
    case GF_RDYA: return recip_pos(dxya_at(g, 1, t, i, j));
    case GF_RDXC: return recip_pos(dxc_at(g, t, i, j));
    case GF_RDYC: return recip_pos(dyc_at(g, t, i, j));
    case GF_AREA: return area_at(g, t, i, j);
    case GF_RAREA: return recip_pos(area_at(g, t, i, j));
    case GF_AREA_C: return area_c_at(g, t, i, j);
    case GF_RAREA_C: return recip_pos(area_c_at(g, t, i, j));
    case GF_SIN_SG1: case GF_SIN_SG2: case GF_SIN_SG3: case GF_SIN_SG4: case GF_SIN_SG5:
      return sg(g, f - GF_SIN_SG1 + 1, true, t, i, j);
    case GF_COS_SG1: case GF_COS_SG2: case GF_COS_SG3: case GF_COS_SG4: case GF_COS_SG5:
      return sg(g, f - GF_COS_SG1 + 1, false, t, i, j);
    case GF_COSA: return cosa_at(g, t, i, j);
    case GF_SINA:
    case GF_RSINA: {
      const double ca = cosa_at(g, t, i, j);
      const double sa = sqrt(np_max(1.0 - ca * ca, 0.0));
      return f == GF_SINA ? sa : 1.0 / np_max(TINY, sa * sa);
    }
    case GF_COSA_U: return i >= 1 ? 0.5 * (sg(g, 3, false, t, i - 1, j) + sg(g, 1, false, t, i, j)) : 0.0;
    case GF_COSA_V: return j >= 1 ? 0.5 * (sg(g, 4, false, t, i, j - 1) + sg(g, 2, false, t, i, j)) : 0.0;
    case GF_COSA_S: return sg(g, 5, false, t, i, j);
    case GF_SINA_U: return sina_u_at(g, t, i, j);
    case GF_SINA_V: return sina_v_at(g, t, i, j);
    case GF_RSIN_U: {
      const double s = sina_u_at(g, t, i, j);
      return 1.0 / np_max(TINY, s * s);
    }
    case GF_RSIN_V: {
      const double s = sina_v_at(g, t, i, j);
      return 1.0 / np_max(TINY, s * s);
    }
    case GF_RSIN2: {
      const double s = sg(g, 5, true, t, i, j);
      return 1.0 / np_max(TINY, s * s);
    }
    // damping coefficients (fv3core/grid/geometry.py:514-585); on the tile's
    // edge rows the sine is the mean of the two sides' (same file)
    case GF_DIVG_U:
    case GF_DEL6_U: {
      const double dx = dx_at(g, t, i, j), dyc = dyc_at(g, t, i, j);
      if (j == hs || j == he) {
        const double s = 0.5 * (sg(g, 2, true, t, i, j) + sg(g, 4, true, t, i, j - 1));
        return f == GF_DIVG_U ? s * dyc / (dx > 0.0 ? dx : 1.0) : s * dx / (dyc > 0.0 ? dyc : 1.0);
      }
      const double sv = sina_v_at(g, t, i, j);
      if (f == GF_DIVG_U) return dx > 0.0 ? sv * dyc / dx : 0.0;
      return dyc > 0.0 ? sv * dx / dyc : 0.0;
    }
    case GF_DIVG_V:
    case GF_DEL6_V: {
      const double dy = dy_at(g, t, i, j), dxc = dxc_at(g, t, i, j);
      if (i == hs || i == he) {
        const double s = 0.5 * (sg(g, 1, true, t, i, j) + sg(g, 3, true, t, i - 1, j));
        return f == GF_DIVG_V ? s * dxc / (dy > 0.0 ? dy : 1.0) : s * dy / (dxc > 0.0 ? dxc : 1.0);
      }
      const double su = sina_u_at(g, t, i, j);
      if (f == GF_DIVG_V) return dy > 0.0 ? su * dxc / dy : 0.0;
      return dxc > 0.0 ? su * dy / dxc : 0.0;
    }
    case GF_FC: {
      double lon, lat;
      lonlat(corner(g, t, i, j), lon, lat);
      return 2.0 * g.omega * sin(lat);
    }
    case GF_F0: {
      if (i >= g.m - 1 || j >= g.m - 1) return 0.0;
      double lon, lat;
      lonlat_a(g, t, i, j, lon, lat);
      return 2.0 * g.omega * sin(lat);
    }
    case GF_AGRID1:
    case GF_AGRID2: {
      double lon, lat;
      lonlat_a(g, t, i, j, lon, lat);
      return f == GF_AGRID1 ? lon : lat;
    }
    case GF_BGRID1:
    case GF_BGRID2: {
      double lon, lat;
      lonlat(corner(g, t, i, j), lon, lat);
      return f == GF_BGRID1 ? lon : lat;
    }
    case GF_A11: return c2l_at(g, 0, t, i, j);
    case GF_A12: return c2l_at(g, 1, t, i, j);
    case GF_A21: return c2l_at(g, 2, t, i, j);
    default: return c2l_at(g, 3, t, i, j);
  }
}

// A -> B interpolation weight of point j (0 .. n) along tile edge e (0 west,
// 1 east, 2 south, 3 north; fv3core/grid/geometry.py:604-714): the share of
// the far side in the great-circle distances from the edge's corner point
// to the midpoints of the centre pairs on either side; 1e8 (the
// reference's fill) at the cube corners j = 0 and n
GG_HD double edge_factor(const Grid& g, int e, int t, int j) {
  const int n = g.n, h = g.h;
  if (j <= 0 || j >= n) return 1.0e8;
  V3 a_lo, a_hi, c;
  if (e < 2) {
    const int ii = e == 0 ? h : h + n;
    a_lo = normalize(add(center(g, t, ii - 1, h + j - 1), center(g, t, ii, h + j - 1)));
    a_hi = normalize(add(center(g, t, ii - 1, h + j), center(g, t, ii, h + j)));
    c = corner(g, t, ii, h + j);
  } else {
    const int jj = e == 2 ? h : h + n;
    a_lo = normalize(add(center(g, t, h + j - 1, jj - 1), center(g, t, h + j - 1, jj)));
    a_hi = normalize(add(center(g, t, h + j, jj - 1), center(g, t, h + j, jj)));
    c = corner(g, t, h + j, jj);
  }
  const double d1 = gc_dist(a_lo, c), d2 = gc_dist(a_hi, c);
  return d2 / (d1 + d2);
}

// x1 / (x2 - x1) of extrapolation m (0..2) at tile corner q (0..3: the
// B-grid points (is, js), (ie+1, js), (ie+1, je+1), (is, je+1)) of
// a2b_ord4's cube-corner values (extrap_corner, a2b_ord4.py:45-57), x1 and
// x2 the great-circle distances (a2b_ord4.py:38-41) from the corner to the
// near and far A-grid points
GG_HD double a2b_extrap_at(const Grid& g, int t, int q, int m) {
  // (near, far) A-grid offsets, in the reference's corner stencils' order
  const int off[4][3][4] = {
      {{0, 0, 1, 1}, {-1, 0, -2, 1}, {0, -1, 1, -2}},
      {{-1, 0, -2, 1}, {-1, -1, -2, -2}, {0, 0, 1, 1}},
      {{-1, -1, -2, -2}, {0, -1, 1, -2}, {-1, 0, -2, 1}},
      {{0, -1, 1, -2}, {-1, -1, -2, -2}, {0, 0, 1, 1}},
  };
  const int s = g.h, e = g.h + g.n - 1;
  const int ci = (q == 0 || q == 3) ? s : e + 1, cj = (q < 2) ? s : e + 1;
  double blon, blat;
  lonlat(corner(g, t, ci, cj), blon, blat);
  auto gcd = [&](int di, int dj) {
    double alon, alat;
    lonlat_a(g, t, ci + di, cj + dj, alon, alat);
    const double sb = sin((alat - blat) / 2.0), sa = sin((alon - blon) / 2.0);
    return asin(sqrt(sb * sb + cos(alat) * cos(blat) * (sa * sa))) * 2.0;
  };
  const double x1 = gcd(off[q][m][0], off[q][m][1]), x2 = gcd(off[q][m][2], off[q][m][3]);
  return x1 / (x2 - x1);
}

#undef GG_HD
}  // namespace gg
}  // namespace fv3b

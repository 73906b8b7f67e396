// Cubed-sphere halo exchange inside one device allocation.
//
// All six tiles live in one array, so the exchange that fv3gfs-util performs
// with MPI messages (the reference's halo updaters, fv3core/stencils/
// dyn_core.py:216-286) is a gather: each edge-halo point of tile t takes one
// value of a neighbouring tile, rotated for vector components.  The source
// of a halo point is computed in closed form here (no tables), from the cube
// connectivity of fv3gfs-util's TilePartitioner (0-based tiles):
//   even t: E -> (t+1, W), N -> (t+2, W, reversed), W -> (t-2, N, reversed),
//           S -> (t-1, N)
//   odd t:  E -> (t+2, S, reversed), N -> (t+1, S), W -> (t-1, E),
//           S -> (t-2, E, reversed)
// Positions use doubled indices along each axis: a cell centre at
// compute-relative offset a sits at 2a+1, an interface at 2a.  A point at
// depth d outside edge E maps to depth d inside the matching edge E' of the
// neighbour, at the same (or mirrored) position along the edge.  The 3x3
// corner blocks have no neighbour and are not written.
//
// The functions are host+device so that a host test can compare them with
// the Python gather tables.
#pragma once
#include "dims.h"

namespace fv3b {

enum HaloEdge { EDGE_W = 0, EDGE_E = 1, EDGE_S = 2, EDGE_N = 3 };

// Tile slot t belongs to cube t / 6 (one cube, or one member of a batched
// ensemble); its neighbours are tiles of the same cube.
__host__ __device__ __forceinline__ void edge_neighbor(int t, int edge, int& t2, int& e2, bool& rev) {
  const int tl = t % 6, base = t - tl;
  if (tl % 2 == 0) {
    switch (edge) {
      case EDGE_E: t2 = (tl + 1) % 6; e2 = EDGE_W; rev = false; break;
      case EDGE_N: t2 = (tl + 2) % 6; e2 = EDGE_W; rev = true; break;
      case EDGE_W: t2 = (tl + 4) % 6; e2 = EDGE_N; rev = true; break;
      default: t2 = (tl + 5) % 6; e2 = EDGE_N; rev = false; break;
    }
  } else {
    switch (edge) {
      case EDGE_E: t2 = (tl + 2) % 6; e2 = EDGE_S; rev = true; break;
      case EDGE_N: t2 = (tl + 1) % 6; e2 = EDGE_S; rev = false; break;
      case EDGE_W: t2 = (tl + 5) % 6; e2 = EDGE_E; rev = false; break;
      default: t2 = (tl + 4) % 6; e2 = EDGE_E; rev = true; break;
    }
  }
  t2 += base;
}

// axis (0 = x, 1 = y) normal to an edge, and the sign of the inward normal
__host__ __device__ __forceinline__ int edge_axis(int edge) { return edge <= EDGE_E ? 0 : 1; }
__host__ __device__ __forceinline__ int inward_sign(int edge) { return (edge == EDGE_W || edge == EDGE_S) ? 1 : -1; }

struct HaloSource {
  int t, i, j;  // storage indices of the source point
  int comp;     // source component (0 = x field, 1 = y field); scalars: 0
  int sign;     // +1 or -1 (vector components)
};

// Source of storage point (i, j) of tile t for a field whose component
// `comp` (0 or 1; scalars pass 0 and sx_of[0] == sx_of[1]) has staggering
// (sx_of[comp], sy_of[comp]) (1 = cell centre, 0 = interface).  Returns
// false unless (i, j) is an edge-halo point within n_halo of the edge.
__host__ __device__ __forceinline__ bool halo_source(const Dims& d, int t, int i, int j, int comp,
                                                    const int sx_of[2], const int sy_of[2], int n_halo,
                                                    HaloSource& out) {
  const int n = d.n, h = d.h, nn = 2 * n;
  const int sx = sx_of[comp], sy = sy_of[comp];
  const int a = i - h, b = j - h;
  const int X = 2 * a + sx, Y = 2 * b + sy;
  const bool xin = X >= 0 && X <= nn, yin = Y >= 0 && Y <= nn;
  int edge, dd, s;
  if (!xin && yin) {
    if (X > nn) {
      edge = EDGE_E;
      dd = X - nn;
      if (a >= n + (1 - sx) + n_halo) return false;
    } else {
      edge = EDGE_W;
      dd = -X;
      if (a < -n_halo) return false;
    }
    s = Y;
  } else if (xin && !yin) {
    if (Y > nn) {
      edge = EDGE_N;
      dd = Y - nn;
      if (b >= n + (1 - sy) + n_halo) return false;
    } else {
      edge = EDGE_S;
      dd = -Y;
      if (b < -n_halo) return false;
    }
    s = X;
  } else {
    return false;
  }
  int t2, e2;
  bool rev;
  edge_neighbor(t, edge, t2, e2, rev);
  const int s2 = rev ? nn - s : s;
  int X2, Y2;
  switch (e2) {
    case EDGE_W: X2 = dd; Y2 = s2; break;
    case EDGE_E: X2 = nn - dd; Y2 = s2; break;
    case EDGE_S: X2 = s2; Y2 = dd; break;
    default: X2 = s2; Y2 = nn - dd; break;
  }
  // our unit vector along `comp` as a multiple of one of the neighbour's
  const int out_axis = edge_axis(edge);
  const int out_sign = -inward_sign(edge);
  int comp2, sign;
  if (comp == out_axis) {
    comp2 = edge_axis(e2);
    sign = out_sign * inward_sign(e2);
  } else {
    comp2 = 1 - edge_axis(e2);  // along-edge axis of the neighbour edge
    sign = rev ? -1 : 1;
  }
  const int sx2 = sx_of[comp2], sy2 = sy_of[comp2];
  out.t = t2;
  out.i = (X2 - sx2) / 2 + h;
  out.j = (Y2 - sy2) / 2 + h;
  out.comp = comp2;
  out.sign = sign;
  return true;
}

// Number of candidate halo points per tile enumerated by halo_point(): four
// edges, n_halo rows, n + 1 positions along each edge.
__host__ __device__ __forceinline__ int halo_candidates(const Dims& d, int n_halo) {
  return 4 * n_halo * (d.n + 1);
}

// Candidate p (0 <= p < halo_candidates) as a storage point (i, j) of a
// field with staggering (sx, sy); false if the candidate is past the end of
// a cell-centred edge.
__host__ __device__ __forceinline__ bool halo_point(const Dims& d, int p, int sx, int sy, int n_halo, int& i,
                                                   int& j) {
  const int n = d.n, h = d.h, L = n + 1;
  const int edge = p / (n_halo * L);
  const int r = p % (n_halo * L);
  const int depth = r / L, along = r % L;
  if (edge <= EDGE_E) {
    if (along >= n + (1 - sy)) return false;
    j = h + along;
    i = edge == EDGE_W ? h - 1 - depth : h + n + (1 - sx) + depth;
  } else {
    if (along >= n + (1 - sx)) return false;
    i = h + along;
    j = edge == EDGE_S ? h - 1 - depth : h + n + (1 - sy) + depth;
  }
  return true;
}

// synchronize_vector_interfaces for D-grid winds: the u values on the south
// edge line (j = h) and the v values on the west edge line (i = h) of tile t
// overwrite the shared edge line of the neighbour across that edge, rotated
// as needed.  For source position `along` (0 <= along < n) on edge
// `edge` (EDGE_S for u, EDGE_W for v) returns the destination point and its
// component (0 = u, 1 = v) and sign.  Destinations are always u on a north
// edge line or v on an east edge line, never a source, so all copies of
// one synchronisation can run at once.
__host__ __device__ __forceinline__ void interface_sync_target(const Dims& d, int t, int edge, int along,
                                                              HaloSource& out) {
  const int n = d.n, h = d.h, nn = 2 * n;
  int t2, e2;
  bool rev;
  edge_neighbor(t, edge, t2, e2, rev);
  const int s = 2 * along + 1;
  const int s2 = rev ? nn - s : s;
  int X2, Y2;
  switch (e2) {
    case EDGE_W: X2 = 0; Y2 = s2; break;
    case EDGE_E: X2 = nn; Y2 = s2; break;
    case EDGE_S: X2 = s2; Y2 = 0; break;
    default: X2 = s2; Y2 = nn; break;
  }
  const int comp2 = 1 - edge_axis(e2);  // the neighbour's along-edge component
  const int sx2 = comp2 == 0 ? 1 : 0, sy2 = comp2 == 0 ? 0 : 1;
  out.t = t2;
  out.i = (X2 - sx2) / 2 + h;
  out.j = (Y2 - sy2) / 2 + h;
  out.comp = comp2;
  out.sign = rev ? -1 : 1;
}

}  // namespace fv3b

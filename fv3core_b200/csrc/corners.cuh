// Cube-corner halo rules in closed form.
//
// Each function returns true if storage point (i, j) lies in one of the
// four 3x3 corner halo blocks of a tile and sets (si, sj) to the point the
// reference copies from (fv3core/utils/corners.py):
//   copy_corner_x / _y : copy_corners_{x,y}_stencil_defn (corners.py:306-422),
//                        also delnflux.py copy_corners_{x,y}_nord
//   bgrid_corner_x / _y: fill_corners_bgrid_{x,y}_defn (corners.py:598-722),
//                        blocks of a cell-corner (B-grid) field
// Sources always lie in an edge halo or the compute domain, never in a
// corner block, so a corner fill can run in parallel with reads of its
// sources.
#pragma once
#include "dims.h"

namespace fv3b {

__host__ __device__ __forceinline__ bool copy_corner_x(const Dims& d, int i, int j, int& si, int& sj) {
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  if (i >= s - 3 && i <= s - 1) {
    int a = i - s;
    if (j >= js - 3 && j <= js - 1) { int b = j - js; si = s + b; sj = js - 1 - a; return true; }
    if (j >= je + 1 && j <= je + 3) { int b = j - je; si = s - b; sj = je + 1 + a; return true; }
  } else if (i >= e + 1 && i <= e + 3) {
    int a = i - e;
    if (j >= js - 3 && j <= js - 1) { int b = j - js; si = e - b; sj = js - 1 + a; return true; }
    if (j >= je + 1 && j <= je + 3) { int b = j - je; si = e + b; sj = je + 1 - a; return true; }
  }
  return false;
}

__host__ __device__ __forceinline__ bool copy_corner_y(const Dims& d, int i, int j, int& si, int& sj) {
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  if (i >= s - 3 && i <= s - 1) {
    int a = i - s;
    if (j >= js - 3 && j <= js - 1) { int b = j - js; si = s - 1 - b; sj = js + a; return true; }
    if (j >= je + 1 && j <= je + 3) { int b = j - je; si = s - 1 + b; sj = je - a; return true; }
  } else if (i >= e + 1 && i <= e + 3) {
    int a = i - e;
    if (j >= js - 3 && j <= js - 1) { int b = j - js; si = e + 1 + b; sj = js - a; return true; }
    if (j >= je + 1 && j <= je + 3) { int b = j - je; si = e + 1 - b; sj = je + a; return true; }
  }
  return false;
}

__device__ __forceinline__ bool bgrid_corner_x(const Dims& d, int i, int j, int& si, int& sj) {
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  if (i >= s - 3 && i <= s - 1) {
    int a = i - s;
    if (j >= js - 3 && j <= js - 1) { int b = j - js; si = s + b; sj = js - a; return true; }
    if (j >= je + 2 && j <= je + 4) { int b = j - (je + 1); si = s - b; sj = je + 1 + a; return true; }
  } else if (i >= e + 2 && i <= e + 4) {
    int a = i - (e + 1);
    if (j >= js - 3 && j <= js - 1) { int b = j - js; si = e + 1 - b; sj = js + a; return true; }
    if (j >= je + 2 && j <= je + 4) { int b = j - (je + 1); si = e + 1 + b; sj = je + 1 - a; return true; }
  }
  return false;
}

__device__ __forceinline__ bool bgrid_corner_y(const Dims& d, int i, int j, int& si, int& sj) {
  const int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  if (i >= s - 3 && i <= s - 1) {
    int a = i - s;
    if (j >= js - 3 && j <= js - 1) { int b = j - js; si = s - b; sj = js + a; return true; }
    if (j >= je + 2 && j <= je + 4) { int b = j - (je + 1); si = s + b; sj = je + 1 - a; return true; }
  } else if (i >= e + 2 && i <= e + 4) {
    int a = i - (e + 1);
    if (j >= js - 3 && j <= js - 1) { int b = j - js; si = e + 1 + b; sj = js - a; return true; }
    if (j >= je + 2 && j <= je + 4) { int b = j - (je + 1); si = e + 1 - b; sj = je + 1 + a; return true; }
  }
  return false;
}

// fill_corners_{2,3}cells_mult_{x,y} (fv3core/utils/corners.py:128-303):
// returns true and the source offset/multiplier if (i, j) is a filled corner
// point of the given kind.
struct CornerRule {
  int di, dj;
  real mult;
};

__device__ __forceinline__ bool corner_x(const Dims& d, int i, int j, bool three, real sw, real se, real nw,
                                         real ne, CornerRule& r) {
  int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  if (j == js - 1) {
    if (i == s - 1) { r = {0, 1, sw}; return true; }
    if (i == s - 2) { r = {1, 2, sw}; return true; }
    if (i == e + 1) { r = {0, 1, se}; return true; }
    if (i == e + 2) { r = {-1, 2, se}; return true; }
    if (three && i == s - 3) { r = {2, 3, sw}; return true; }
    if (three && i == e + 3) { r = {-2, 3, se}; return true; }
  } else if (j == je + 1) {
    if (i == s - 1) { r = {0, -1, nw}; return true; }
    if (i == s - 2) { r = {1, -2, nw}; return true; }
    if (i == e + 1) { r = {0, -1, ne}; return true; }
    if (i == e + 2) { r = {-1, -2, ne}; return true; }
    if (three && i == s - 3) { r = {2, -3, nw}; return true; }
    if (three && i == e + 3) { r = {-2, -3, ne}; return true; }
  }
  return false;
}

__device__ __forceinline__ bool corner_y(const Dims& d, int i, int j, bool three, real sw, real se, real nw,
                                         real ne, CornerRule& r) {
  int s = d.isc, e = d.iec, js = d.jsc, je = d.jec;
  if (i == s - 1) {
    if (j == js - 1) { r = {1, 0, sw}; return true; }
    if (j == js - 2) { r = {2, 1, sw}; return true; }
    if (j == je + 1) { r = {1, 0, nw}; return true; }
    if (j == je + 2) { r = {2, -1, nw}; return true; }
    if (three && j == js - 3) { r = {3, 2, sw}; return true; }
    if (three && j == je + 3) { r = {3, -2, nw}; return true; }
  } else if (i == e + 1) {
    if (j == js - 1) { r = {-1, 0, se}; return true; }
    if (j == js - 2) { r = {-2, 1, se}; return true; }
    if (j == je + 1) { r = {-1, 0, ne}; return true; }
    if (j == je + 2) { r = {-2, -1, ne}; return true; }
    if (three && j == js - 3) { r = {-3, 2, se}; return true; }
    if (three && j == je + 3) { r = {-3, -2, ne}; return true; }
  }
  return false;
}

}  // namespace fv3b

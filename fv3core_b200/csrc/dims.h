// Grid sizes and index arithmetic, usable from host and device code
// (kept free of kernel syntax so host-only tests can include it).
//
// Device layout of every field (all six cube tiles in one allocation):
//   3-D  double f[6][nk][nj][ni]   ni = nj = n + 2*halo + 1, nk = npz + 1
//   2-D  double g[6][nj][ni]       (metric terms, surface fields)
//   1-D  double c[nk]              (per-level constants)
// i is the fastest index so that a warp reads 32 consecutive i points.
// Index (t, i, j, k) uses the reference's storage indices (compute domain
// starts at i = j = halo).
#pragma once

#include <stdint.h>

#include "../../include/fv3core_b200.h"

#ifndef __CUDACC__
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif
#ifndef __forceinline__
#define __forceinline__ inline
#endif
#endif

namespace fv3b {

// Element type of the fields: double in the FP64 build, float in the
// mixed-precision build (FV3B_REAL_T=float, see include/fv3core_b200.h).
// RC(x) gives a floating constant that type, so constant-times-field
// arithmetic stays in the build's precision.
using real = fv3b_real;
#define RC(x) (static_cast<::fv3b::real>(x))

// Offsets into a field are 32-bit integers, which keeps the index
// arithmetic of the stencils to single 32-bit multiply-adds: a 3-D field of
// all six tiles must hold fewer than 2^31 elements (C1536 L79 holds 1.1e9).
// dims_fit checks it; every entry point that takes grid sizes calls it.
using idx_t = int;

struct Dims {
  int n, h, nz;
  int ni, nj, nk;
  // tile slots of the arrays: 6 for one cube, 6 x members for an ensemble
  // of same-resolution members kept in one allocation (member m owns tiles
  // 6m .. 6m+5)
  int nt;
  idx_t sj, sk, st;  // 3-D strides (i stride is 1)
  idx_t st2;         // 2-D tile stride (j stride is ni)
  int isc, iec, jsc, jec;  // compute domain (inclusive), storage indices
};

inline bool dims_fit(const fv3b_grid_dims* g) {
  if (g->npx < 1 || g->npz < 1 || g->n_halo < 0) return false;
  const long long ni = (long long)g->npx + 2LL * g->n_halo + 1;
  return 6LL * ni * ni * (g->npz + 1LL) < (1LL << 31);
}

inline Dims make_dims(const fv3b_grid_dims* g) {
  Dims d;
  d.n = g->npx;
  d.h = g->n_halo;
  d.nz = g->npz;
  d.ni = d.n + 2 * d.h + 1;
  d.nj = d.ni;
  d.nk = d.nz + 1;
  d.nt = 6;
  d.sj = d.ni;
  d.sk = d.ni * d.nj;
  d.st = d.sk * d.nk;
  d.st2 = d.ni * d.nj;
  d.isc = d.h;
  d.iec = d.h + d.n - 1;
  d.jsc = d.h;
  d.jec = d.h + d.n - 1;
  return d;
}

__host__ __device__ __forceinline__ idx_t idx3(const Dims& d, int t, int i, int j, int k) {
  return t * d.st + k * d.sk + j * d.sj + i;
}
__host__ __device__ __forceinline__ idx_t idx2(const Dims& d, int t, int i, int j) {
  return t * d.st2 + j * d.ni + i;
}

}  // namespace fv3b

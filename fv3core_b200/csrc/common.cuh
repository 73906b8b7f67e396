// Shared device/host helpers for the acoustic-substep kernels.
//
// Device layout of every field (all six cube tiles in one allocation):
//   3-D  double f[6][nk][nj][ni]   ni = nj = n + 2*halo + 1, nk = npz + 1
//   2-D  double g[6][nj][ni]       (metric terms, surface fields)
//   1-D  double c[nk]              (per-level constants)
// i is the fastest index so that a warp reads 32 consecutive i points.
// Index (t, i, j, k) uses the reference's storage indices (compute domain
// starts at i = j = halo).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/fv3core_b200.h"
#include "dims.h"

namespace fv3b {

// Box of storage indices [i0, i1) x [j0, j1) x [k0, k1), all six tiles.
struct Box {
  int i0, i1, j0, j1, k0, k1;
};

// Launch f(t, i, j, k) over a box: x covers i (warp-contiguous), y covers j,
// z covers (tile, k).
// Tile slot and level of grid z = t * nkb + (k - k0): the quotient taken
// as a float product with 1/nkb, which spares each thread an integer
// division.  It is exact: (z + 0.5) / nkb lies at least 0.5 / nkb from an
// integer, and for z < 2^16 the two roundings are off by less than
// 2^-22 * 2^16 / nkb = 0.016 / nkb (checked for every z < 2^16 and every
// nkb < 256).
__device__ __forceinline__ void box_tk(const Box& b, int& t, int& k) {
  const int nkb = b.k1 - b.k0;
  const int z = blockIdx.z;
  t = __float2int_rz((static_cast<float>(z) + 0.5f) * __frcp_rn(static_cast<float>(nkb)));
  k = b.k0 + z - t * nkb;
}

template <typename F>
__global__ void box_kernel(Box b, F f) {
  int i = b.i0 + blockIdx.x * blockDim.x + threadIdx.x;
  int j = b.j0 + blockIdx.y * blockDim.y + threadIdx.y;
  int t, k;
  box_tk(b, t, k);
  if (i < b.i1 && j < b.j1) f(t, i, j, k);
}

// Counts kernel launches of this library (host side, all threads); read
// through fv3b_launch_count().
void note_launch();

// Thread-block shapes of the box and column kernels: process-wide settings
// (fv3b_set_launch_shape), chosen by the autotuner; the shape changes no
// result, since every thread computes its own points.
struct LaunchShape {
  int box_x = 32, box_y = 4, col = 128;
};
const LaunchShape& launch_shape();

// Tile slots of the calling entry point's arrays (6, or 6 x members of a
// batched context), a per-host-thread setting that TileScope sets from the
// context for the duration of a call; the launch helpers size their grids
// by it, so one launch covers every member.
int& tile_slots();
struct TileScope {
  int saved;
  explicit TileScope(int nt) : saved(tile_slots()) { tile_slots() = nt; }
  ~TileScope() { tile_slots() = saved; }
  TileScope(const TileScope&) = delete;
  TileScope& operator=(const TileScope&) = delete;
};

template <typename F>
cudaError_t launch_box(const Box& b, cudaStream_t s, F f) {
  int ni = b.i1 - b.i0, nj = b.j1 - b.j0, nk = b.k1 - b.k0;
  if (ni <= 0 || nj <= 0 || nk <= 0) return cudaSuccess;
  const LaunchShape& ls = launch_shape();
  dim3 block(ls.box_x, ls.box_y, 1);
  dim3 grid((ni + ls.box_x - 1) / ls.box_x, (nj + ls.box_y - 1) / ls.box_y, tile_slots() * nk);
  box_kernel<<<grid, block, 0, s>>>(b, f);
  note_launch();
  return cudaGetLastError();
}

// A box launch whose thread order along i puts the columns [a0, a1) first,
// padded to a whole number of thread-block rows, and the box's other
// columns after them.  Stencils whose edge columns take a longer code path
// (the PPM boundary formulas, the cube-corner reads) then keep those
// columns out of the warps that run the interior path; every point still
// computes what it computes under launch_box.
template <typename F>
__global__ void box_kernel_split(Box b, int a0, int nint, int nint_pad, F f) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = b.j0 + blockIdx.y * blockDim.y + threadIdx.y;
  int t, k;
  box_tk(b, t, k);
  int i;
  if (x < nint_pad) {
    if (x >= nint) return;
    i = a0 + x;
  } else {
    const int e = x - nint_pad, nleft = a0 - b.i0;
    i = e < nleft ? b.i0 + e : a0 + nint + (e - nleft);
    if (i >= b.i1) return;
  }
  if (j < b.j1) f(t, i, j, k);
}

template <typename F>
cudaError_t launch_box_split(const Box& b, int a0, int a1, cudaStream_t s, F f) {
  int ni = b.i1 - b.i0, nj = b.j1 - b.j0, nk = b.k1 - b.k0;
  if (ni <= 0 || nj <= 0 || nk <= 0) return cudaSuccess;
  a0 = a0 < b.i0 ? b.i0 : a0;
  a1 = a1 > b.i1 ? b.i1 : a1;
  if (a1 <= a0) return launch_box(b, s, f);
  const LaunchShape& ls = launch_shape();
  const int nint = a1 - a0;
  const int nint_pad = (nint + ls.box_x - 1) / ls.box_x * ls.box_x;
  const int nx = nint_pad + (ni - nint);
  dim3 block(ls.box_x, ls.box_y, 1);
  dim3 grid((nx + ls.box_x - 1) / ls.box_x, (nj + ls.box_y - 1) / ls.box_y, tile_slots() * nk);
  box_kernel_split<<<grid, block, 0, s>>>(b, a0, nint, nint_pad, f);
  note_launch();
  return cudaGetLastError();
}

// Launch f(t, i, j) over the columns of a 2-D box (all six tiles).
template <typename F>
__global__ void column_kernel(int i0, int i1, int j0, int j1, F f) {
  int ncol_i = i1 - i0;
  int ncol = ncol_i * (j1 - j0);
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  int t = blockIdx.y;
  if (c >= ncol) return;
  int i = i0 + c % ncol_i;
  int j = j0 + c / ncol_i;
  f(t, i, j);
}

template <typename F>
cudaError_t launch_columns(int i0, int i1, int j0, int j1, cudaStream_t s, F f, int block = 0) {
  if (block <= 0) block = launch_shape().col;
  int ncol = (i1 - i0) * (j1 - j0);
  if (ncol <= 0) return cudaSuccess;
  dim3 grid((ncol + block - 1) / block, tile_slots(), 1);
  column_kernel<<<grid, block, 0, s>>>(i0, i1, j0, j1, f);
  note_launch();
  return cudaGetLastError();
}

void set_last_error(const char* where, cudaError_t e);
void set_last_error_msg(const char* msg);

}  // namespace fv3b

#define FV3B_CHECK(call)                                  \
  do {                                                    \
    cudaError_t _e = (call);                              \
    if (_e != cudaSuccess) {                              \
      fv3b::set_last_error(__func__, _e);                 \
      return FV3B_ERR_CUDA;                               \
    }                                                     \
  } while (0)

// every entry point that takes a context starts with this: its launches
// cover the context's tile slots
#define FV3B_TILES(ctx) const ::fv3b::TileScope _fv3b_tiles((ctx) ? (ctx)->d.nt : 6)

#define FV3B_REQUIRE(cond, msg)                           \
  do {                                                    \
    if (!(cond)) {                                        \
      fv3b::set_last_error_msg(msg);                      \
      return FV3B_ERR_ARGUMENT;                           \
    }                                                     \
  } while (0)

// fv3b_generate_grid: the cubed-sphere metric terms generated on the
// device (csrc/grid_gen.h holds the point functions).  One thread per
// (field, tile, j, i) output value, then one block for the four area
// extremes.  Nothing is allocated: the caller passes every output array.
#include <cuda_runtime.h>

#include "common.cuh"
#include "grid_gen.h"

namespace fv3b {
namespace {

struct GridOut {
  double* field[gg::GF_COUNT];
  double* edge[4];
  double* a2b;
};

__global__ void grid_fields_kernel(gg::Grid g, GridOut out) {
  const long long npt = 6LL * g.m * g.m;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int f = blockIdx.y;
  if (idx >= npt) return;
  const int t = (int)(idx / ((long long)g.m * g.m));
  const int r = (int)(idx - (long long)t * g.m * g.m);
  const int j = r / g.m, i = r - j * g.m;
  // device layout: i fastest
  out.field[f][idx] = gg::field_at(g, f, t, i, j);
}

__global__ void grid_edges_kernel(gg::Grid g, GridOut out) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  const int ne = 6 * (g.n + 1);
  if (idx < 4 * ne) {
    const int e = idx / ne, r = idx - e * ne;
    const int t = r / (g.n + 1), j = r - t * (g.n + 1);
    out.edge[e][r] = gg::edge_factor(g, e, t, j);
  } else if (idx < 4 * ne + 72) {
    const int r = idx - 4 * ne;  // [6][4][3]
    const int t = r / 12, q = (r / 3) % 4, m = r % 3;
    out.a2b[r] = gg::a2b_extrap_at(g, t, q, m);
  }
}

// min and max of the cell areas over the compute domains, and of the dual
// cell areas over the compute corners; one block
constexpr int EXT_THREADS = 512;
__global__ void grid_extremes_kernel(gg::Grid g, double* scalars) {
  __shared__ double s[4][EXT_THREADS];
  const int n = g.n, h = g.h;
  double amin = 1.0e300, amax = -1.0e300, cmin = 1.0e300, cmax = -1.0e300;
  const int na = 6 * n * n, nc = 6 * (n + 1) * (n + 1);
  for (int p = threadIdx.x; p < na; p += blockDim.x) {
    const int t = p / (n * n), r = p % (n * n);
    const double a = gg::area_at(g, t, h + r % n, h + r / n);
    amin = fmin(amin, a);
    amax = fmax(amax, a);
  }
  for (int p = threadIdx.x; p < nc; p += blockDim.x) {
    const int t = p / ((n + 1) * (n + 1)), r = p % ((n + 1) * (n + 1));
    const double a = gg::area_c_at(g, t, h + r % (n + 1), h + r / (n + 1));
    cmin = fmin(cmin, a);
    cmax = fmax(cmax, a);
  }
  s[0][threadIdx.x] = amin;
  s[1][threadIdx.x] = amax;
  s[2][threadIdx.x] = cmin;
  s[3][threadIdx.x] = cmax;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w /= 2) {
    if (threadIdx.x < w) {
      s[0][threadIdx.x] = fmin(s[0][threadIdx.x], s[0][threadIdx.x + w]);
      s[1][threadIdx.x] = fmax(s[1][threadIdx.x], s[1][threadIdx.x + w]);
      s[2][threadIdx.x] = fmin(s[2][threadIdx.x], s[2][threadIdx.x + w]);
      s[3][threadIdx.x] = fmax(s[3][threadIdx.x], s[3][threadIdx.x + w]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    scalars[0] = s[0][0];
    scalars[1] = s[1][0];
    scalars[2] = s[2][0];
    scalars[3] = s[3][0];
  }
}

}  // namespace
}  // namespace fv3b

// MetricTerms (fv3core/grid/generation.py:66) for one cube, on the device.
extern "C" int fv3b_generate_grid(int n, int halo, int lattice, double radius, double omega,
                                  const fv3b_grid_fields* out, void* stream) {
  using namespace fv3b;
  FV3B_REQUIRE(out != nullptr && out->a2b_extrap != nullptr && out->scalars != nullptr,
               "fv3b_generate_grid: null output");
  for (int f = 0; f < FV3B_GRID_NFIELDS; ++f) FV3B_REQUIRE(out->field[f] != nullptr, "fv3b_generate_grid: null field");
  for (int e = 0; e < 4; ++e) FV3B_REQUIRE(out->edge[e] != nullptr, "fv3b_generate_grid: null edge factors");
  FV3B_REQUIRE(halo >= 1 && halo <= 8 && n >= 2 * halo && n <= 4096,
               "fv3b_generate_grid: need 1 <= halo <= 8 and 2 * halo <= n <= 4096");
  FV3B_REQUIRE(radius > 0.0, "fv3b_generate_grid: radius must be positive");
  FV3B_REQUIRE(lattice == 0 || lattice == 1, "fv3b_generate_grid: lattice must be 0 (equiangular) or 1 (equidistant)");
  static_assert(FV3B_GRID_NFIELDS == gg::GF_COUNT, "field list of the header and of grid_gen.h differ");
  fv3b_grid_dims gd{n, halo, 1, 0};
  gg::Grid g;
  g.d = make_dims(&gd);
  g.n = n;
  g.h = halo;
  g.m = n + 2 * halo + 1;
  g.lattice = lattice;
  g.radius = radius;
  g.omega = omega;
  GridOut o;
  for (int f = 0; f < gg::GF_COUNT; ++f) o.field[f] = out->field[f];
  for (int e = 0; e < 4; ++e) o.edge[e] = out->edge[e];
  o.a2b = out->a2b_extrap;
  cudaStream_t st = (cudaStream_t)stream;
  const long long npt = 6LL * g.m * g.m;
  grid_fields_kernel<<<dim3((unsigned)((npt + 127) / 128), gg::GF_COUNT), 128, 0, st>>>(g, o);
  note_launch();
  FV3B_CHECK(cudaGetLastError());
  const int ne = 4 * 6 * (n + 1) + 72;
  grid_edges_kernel<<<(ne + 127) / 128, 128, 0, st>>>(g, o);
  note_launch();
  FV3B_CHECK(cudaGetLastError());
  grid_extremes_kernel<<<1, EXT_THREADS, 0, st>>>(g, out->scalars);
  note_launch();
  FV3B_CHECK(cudaGetLastError());
  return FV3B_OK;
}

// Device halo updates of the six-tile array (see halo.cuh for the
// geometry).  One thread per (tile, edge-halo point, level): the copies of
// all levels go out at once instead of one level after another (the copies
// are small, so their latency, not their bytes, sets a launch's time); up
// to four fields of the same staggering share a launch.
#include "ctx.cuh"
#include "halo.cuh"
#include "halo_ops.cuh"

namespace fv3b {

namespace {
constexpr int HALO_BLOCK = 128;

struct FieldSet {
  real* f[4];
  int n;
};

__global__ void halo_scalar_kernel(Dims d, FieldSet fs, int sx, int sy, int n_halo) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int t = blockIdx.y, k = blockIdx.z;
  if (p >= halo_candidates(d, n_halo)) return;
  int i, j;
  if (!halo_point(d, p, sx, sy, n_halo, i, j)) return;
  const int sxo[2] = {sx, sx}, syo[2] = {sy, sy};
  HaloSource src;
  if (!halo_source(d, t, i, j, 0, sxo, syo, n_halo, src)) return;
  const idx_t dst = idx3(d, t, i, j, k), from = idx3(d, src.t, src.i, src.j, k);
  for (int q = 0; q < fs.n; ++q) {
    real* f = fs.f[q];
    f[dst] = f[from];
  }
}

__global__ void halo_vector_kernel(Dims d, real* x, real* y, int cgrid) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int t = blockIdx.y >> 1, comp = blockIdx.y & 1, k = blockIdx.z;
  const int n_halo = d.h;
  if (p >= halo_candidates(d, n_halo)) return;
  // D grid: x (u) on (centre, interface), y (v) on (interface, centre);
  // C grid the other way round
  const int sxo[2] = {cgrid ? 0 : 1, cgrid ? 1 : 0};
  const int syo[2] = {cgrid ? 1 : 0, cgrid ? 0 : 1};
  int i, j;
  if (!halo_point(d, p, sxo[comp], syo[comp], n_halo, i, j)) return;
  HaloSource src;
  if (!halo_source(d, t, i, j, comp, sxo, syo, n_halo, src)) return;
  real* dstf = comp == 0 ? x : y;
  const real* srcf = src.comp == 0 ? x : y;
  const real sign = (real)src.sign;
  dstf[idx3(d, t, i, j, k)] = sign * srcf[idx3(d, src.t, src.i, src.j, k)];
}

__global__ void interface_sync_kernel(Dims d, real* u, real* v) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  const int t = blockIdx.y >> 1, comp = blockIdx.y & 1, k = blockIdx.z;
  if (a >= d.n) return;
  HaloSource dst;
  interface_sync_target(d, t, comp == 0 ? EDGE_S : EDGE_W, a, dst);
  const int si = comp == 0 ? d.h + a : d.h, sj = comp == 0 ? d.h : d.h + a;
  const real* srcf = comp == 0 ? u : v;
  real* dstf = dst.comp == 0 ? u : v;
  const real sign = (real)dst.sign;
  dstf[idx3(d, dst.t, dst.i, dst.j, k)] = sign * srcf[idx3(d, t, si, sj, k)];
}
}  // namespace

cudaError_t halo_scalars(const Dims& d, real* const* fields, int nfields, int stagger, int n_halo, int nlev,
                         cudaStream_t st) {
  const int nc = halo_candidates(d, n_halo);
  if (nlev <= 0) return cudaSuccess;
  dim3 grid((nc + HALO_BLOCK - 1) / HALO_BLOCK, d.nt, nlev);
  for (int f0 = 0; f0 < nfields; f0 += 4) {
    FieldSet fs;
    fs.n = nfields - f0 < 4 ? nfields - f0 : 4;
    for (int q = 0; q < fs.n; ++q) fs.f[q] = fields[f0 + q];
    halo_scalar_kernel<<<grid, HALO_BLOCK, 0, st>>>(d, fs, stagger, stagger, n_halo);
    note_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t halo_vector(const Dims& d, real* x, real* y, bool cgrid, int nlev, cudaStream_t st) {
  const int nc = halo_candidates(d, d.h);
  if (nlev <= 0) return cudaSuccess;
  dim3 grid((nc + HALO_BLOCK - 1) / HALO_BLOCK, 2 * d.nt, nlev);
  halo_vector_kernel<<<grid, HALO_BLOCK, 0, st>>>(d, x, y, cgrid ? 1 : 0);
  note_launch();
  return cudaGetLastError();
}

cudaError_t sync_vector_interfaces(const Dims& d, real* u, real* v, int nlev, cudaStream_t st) {
  if (nlev <= 0) return cudaSuccess;
  dim3 grid((d.n + HALO_BLOCK - 1) / HALO_BLOCK, 2 * d.nt, nlev);
  interface_sync_kernel<<<grid, HALO_BLOCK, 0, st>>>(d, u, v);
  note_launch();
  return cudaGetLastError();
}

}  // namespace fv3b

using namespace fv3b;

// HaloUpdater.update of one scalar field (fv3gfs-util, as the reference's
// AcousticDynamics uses it): stagger 1 = cell centres (X, Y), 0 = cell
// corners (X_INTERFACE, Y_INTERFACE); n_halo rows; nlev levels.
extern "C" int fv3b_halo_update_scalar(fv3b_ctx* ctx, real* field, int stagger, int n_halo, int nlev,
                                       void* stream) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && field, "fv3b_halo_update_scalar: null argument");
  FV3B_REQUIRE(stagger == 0 || stagger == 1, "fv3b_halo_update_scalar: stagger must be 0 or 1");
  FV3B_REQUIRE(n_halo >= 1 && n_halo <= ctx->d.h, "fv3b_halo_update_scalar: n_halo out of range");
  FV3B_REQUIRE(nlev >= 1 && nlev <= ctx->d.nk, "fv3b_halo_update_scalar: nlev out of range");
  FV3B_CHECK(halo_scalars(ctx->d, &field, 1, stagger, n_halo, nlev, (cudaStream_t)stream));
  return FV3B_OK;
}

// Vector HaloUpdater.update: grid 0 = D-grid winds (u, v), 1 = C-grid winds
// (uc, vc); full halo width.
extern "C" int fv3b_halo_update_vector(fv3b_ctx* ctx, real* x, real* y, int grid, int nlev, void* stream) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && x && y, "fv3b_halo_update_vector: null argument");
  FV3B_REQUIRE(grid == 0 || grid == 1, "fv3b_halo_update_vector: grid must be 0 (D) or 1 (C)");
  FV3B_REQUIRE(nlev >= 1 && nlev <= ctx->d.nk, "fv3b_halo_update_vector: nlev out of range");
  FV3B_CHECK(halo_vector(ctx->d, x, y, grid == 1, nlev, (cudaStream_t)stream));
  return FV3B_OK;
}

// CubedSphereCommunicator.synchronize_vector_interfaces for D-grid winds.
extern "C" int fv3b_synchronize_vector_interfaces(fv3b_ctx* ctx, real* u, real* v, int nlev, void* stream) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && u && v, "fv3b_synchronize_vector_interfaces: null argument");
  FV3B_REQUIRE(nlev >= 1 && nlev <= ctx->d.nk, "fv3b_synchronize_vector_interfaces: nlev out of range");
  FV3B_CHECK(sync_vector_interfaces(ctx->d, u, v, nlev, (cudaStream_t)stream));
  return FV3B_OK;
}

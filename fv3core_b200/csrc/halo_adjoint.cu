// Adjoints of the halo updates (halo_adjoint.h), in place on the
// cotangents: one launch adds every halo point's cotangent into its source
// (atomically: edge points can feed more than one halo point), a second
// zeroes the halo points, whose values the forward overwrote.
#include "ctx.cuh"
#include "halo_adjoint.h"

namespace fv3b {
namespace {
constexpr int HALO_ADJ_BLOCK = 128;

struct HaloAdjArgs {
  real *gx, *gy;
  int sx[2], sy[2];
  int ncomp, n_halo, nlev;
};

__global__ void halo_adjoint_kernel(Dims d, HaloAdjArgs a, int zero) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int t = blockIdx.y / a.ncomp, comp = blockIdx.y % a.ncomp;
  if (p >= halo_candidates(d, a.n_halo)) return;
  HaloCopy c;
  if (!halo_copy(d, t, p, comp, a.sx, a.sy, a.n_halo, c)) return;
  real* gd = comp == 0 ? a.gx : a.gy;
  real* gs = c.src_comp == 0 ? a.gx : a.gy;
  // scalars copy without the vector rotation's sign
  const real sign = a.ncomp == 2 ? (real)c.sign : RC(1.0);
  for (int k = 0; k < a.nlev; ++k) {
    if (zero) gd[c.dst + k * d.sk] = RC(0.0);
    else atomicAdd(gs + c.src + k * d.sk, sign * gd[c.dst + k * d.sk]);
  }
}

__global__ void interface_sync_adjoint_kernel(Dims d, real* gu, real* gv, int nlev, int zero) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  const int t = blockIdx.y >> 1, comp = blockIdx.y & 1;
  if (a >= d.n) return;
  int dst_comp;
  const HaloCopy c = interface_sync_copy(d, t, comp, a, dst_comp);
  real* gd = dst_comp == 0 ? gu : gv;
  real* gs = comp == 0 ? gu : gv;
  const real sign = (real)c.sign;
  for (int k = 0; k < nlev; ++k) {
    if (zero) gd[c.dst + k * d.sk] = RC(0.0);
    else atomicAdd(gs + c.src + k * d.sk, sign * gd[c.dst + k * d.sk]);
  }
}

cudaError_t halo_adjoint(const Dims& d, const HaloAdjArgs& a, cudaStream_t st) {
  dim3 grid((halo_candidates(d, a.n_halo) + HALO_ADJ_BLOCK - 1) / HALO_ADJ_BLOCK, d.nt * a.ncomp);
  for (int zero = 0; zero < 2; ++zero) {
    halo_adjoint_kernel<<<grid, HALO_ADJ_BLOCK, 0, st>>>(d, a, zero);
    note_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}
}  // namespace
}  // namespace fv3b

using namespace fv3b;

// Adjoint of fv3b_halo_update_scalar: g holds the cotangent of the updated
// field and is turned, in place, into that of the field before the update.
extern "C" int fv3b_halo_update_scalar_adjoint(fv3b_ctx* ctx, real* g, int stagger, int n_halo, int nlev,
                                               void* stream) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && g, "fv3b_halo_update_scalar_adjoint: null argument");
  FV3B_REQUIRE(stagger == 0 || stagger == 1, "fv3b_halo_update_scalar_adjoint: stagger must be 0 or 1");
  FV3B_REQUIRE(n_halo >= 1 && n_halo <= ctx->d.h, "fv3b_halo_update_scalar_adjoint: n_halo out of range");
  FV3B_REQUIRE(nlev >= 1 && nlev <= ctx->d.nk, "fv3b_halo_update_scalar_adjoint: nlev out of range");
  const HaloAdjArgs a{g, g, {stagger, stagger}, {stagger, stagger}, 1, n_halo, nlev};
  FV3B_CHECK(halo_adjoint(ctx->d, a, (cudaStream_t)stream));
  return FV3B_OK;
}

// Adjoint of fv3b_halo_update_vector (grid 0 = D, 1 = C), in place on gx, gy.
extern "C" int fv3b_halo_update_vector_adjoint(fv3b_ctx* ctx, real* gx, real* gy, int grid, int nlev,
                                               void* stream) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && gx && gy, "fv3b_halo_update_vector_adjoint: null argument");
  FV3B_REQUIRE(grid == 0 || grid == 1, "fv3b_halo_update_vector_adjoint: grid must be 0 (D) or 1 (C)");
  FV3B_REQUIRE(nlev >= 1 && nlev <= ctx->d.nk, "fv3b_halo_update_vector_adjoint: nlev out of range");
  const int c = grid == 1;
  const HaloAdjArgs a{gx, gy, {c ? 0 : 1, c ? 1 : 0}, {c ? 1 : 0, c ? 0 : 1}, 2, ctx->d.h, nlev};
  FV3B_CHECK(halo_adjoint(ctx->d, a, (cudaStream_t)stream));
  return FV3B_OK;
}

// Adjoint of fv3b_synchronize_vector_interfaces, in place on gu, gv.
extern "C" int fv3b_synchronize_vector_interfaces_adjoint(fv3b_ctx* ctx, real* gu, real* gv, int nlev,
                                                          void* stream) {
  FV3B_TILES(ctx);
  FV3B_REQUIRE(ctx && gu && gv, "fv3b_synchronize_vector_interfaces_adjoint: null argument");
  FV3B_REQUIRE(nlev >= 1 && nlev <= ctx->d.nk, "fv3b_synchronize_vector_interfaces_adjoint: nlev out of range");
  const Dims d = ctx->d;
  dim3 grid((d.n + HALO_ADJ_BLOCK - 1) / HALO_ADJ_BLOCK, 2 * d.nt);
  for (int zero = 0; zero < 2; ++zero) {
    interface_sync_adjoint_kernel<<<grid, HALO_ADJ_BLOCK, 0, (cudaStream_t)stream>>>(d, gu, gv, nlev, zero);
    note_launch();
    FV3B_CHECK(cudaGetLastError());
  }
  return FV3B_OK;
}

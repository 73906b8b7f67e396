// Context: grid sizes, metric pointers, device workspace.
#include <new>

#include "ctx.cuh"

using namespace fv3b;

extern "C" int fv3b_ctx_create_batched(const fv3b_grid_dims* dims, const fv3b_metrics* metrics, int members,
                                       fv3b_ctx** out) {
  FV3B_REQUIRE(dims && metrics && out, "fv3b_ctx_create: null argument");
  FV3B_REQUIRE(dims->npx >= 4 && dims->n_halo == 3 && dims->npz >= 2 && dims->npz < 127,
               "fv3b_ctx_create: need npx >= 4, n_halo == 3, 2 <= npz < 127");
  FV3B_REQUIRE(members >= 1 && members <= 10000, "fv3b_ctx_create_batched: members must be in 1..10000");
  FV3B_REQUIRE(dims_fit(dims), "fv3b_ctx_create: a 3-D field of the six tiles must hold fewer than 2^31 elements");
  {
    const long long ni = (long long)dims->npx + 2LL * dims->n_halo + 1;
    FV3B_REQUIRE(6LL * members * ni * ni * (dims->npz + 1LL) < (1LL << 31),
                 "fv3b_ctx_create_batched: a 3-D field of all members must hold fewer than 2^31 elements");
  }
  fv3b_ctx* c = new (std::nothrow) fv3b_ctx();
  FV3B_REQUIRE(c != nullptr, "fv3b_ctx_create: out of host memory");
  c->d = make_dims(dims);
  c->d.nt = 6 * members;
  c->m = *metrics;
  size_t n3 = (size_t)c->d.st * c->d.nt;
  cudaError_t e = cudaMalloc((void**)&c->ws_base, n3 * sizeof(real) * NWS);
  if (e != cudaSuccess) {
    delete c;
    set_last_error("fv3b_ctx_create", e);
    return FV3B_ERR_CUDA;
  }
  for (int i = 0; i < NWS; ++i) c->ws[i] = c->ws_base + n3 * i;
  e = cudaMalloc((void**)&c->col, sizeof(real) * NCOL * MAXLEV);
  if (e != cudaSuccess) {
    cudaFree(c->ws_base);
    delete c;
    set_last_error("fv3b_ctx_create", e);
    return FV3B_ERR_CUDA;
  }
  e = cudaMemset(c->ws_base, 0, n3 * sizeof(real) * NWS);
  if (e != cudaSuccess) {
    cudaFree(c->ws_base);
    delete c;
    set_last_error("fv3b_ctx_create", e);
    return FV3B_ERR_CUDA;
  }
  *out = c;
  return FV3B_OK;
}

extern "C" int fv3b_ctx_create(const fv3b_grid_dims* dims, const fv3b_metrics* metrics, fv3b_ctx** out) {
  return fv3b_ctx_create_batched(dims, metrics, 1, out);
}

extern "C" int fv3b_ctx_destroy(fv3b_ctx* ctx) {
  FV3B_TILES(ctx);
  if (!ctx) return FV3B_OK;
  fv3b_acoustics_release(ctx);
  cudaError_t e = cudaFree(ctx->ws_base);
  cudaError_t e2 = cudaFree(ctx->col);
  cudaError_t e3 = cudaFree(ctx->remap_akbk);
  cudaError_t e4 = cudaFree(ctx->sat_tables);
  delete ctx;
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = e3;
  if (e == cudaSuccess) e = e4;
  FV3B_CHECK(e);
  return FV3B_OK;
}

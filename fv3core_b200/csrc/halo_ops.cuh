// Host launchers of the device halo updates (halo.cu).
#pragma once
#include "common.cuh"

namespace fv3b {
// scalars with staggering 1 (cell centres) or 0 (cell corners) on both axes
cudaError_t halo_scalars(const Dims& d, real* const* fields, int nfields, int stagger, int n_halo, int nlev,
                         cudaStream_t st);
// D-grid (u, v) or C-grid (uc, vc) winds, full halo width
cudaError_t halo_vector(const Dims& d, real* x, real* y, bool cgrid, int nlev, cudaStream_t st);
cudaError_t sync_vector_interfaces(const Dims& d, real* u, real* v, int nlev, cudaStream_t st);
}  // namespace fv3b

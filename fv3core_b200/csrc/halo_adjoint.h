// Transposes of the halo updates (halo.cuh): the forward copies, for every
// edge-halo point dst, sign * f[src] into f[dst] (sources never being
// destinations of the same update), so its adjoint adds sign * g[dst] into
// g[src] for every dst, then zeroes g[dst].  The same holds for
// synchronize_vector_interfaces.  Host+device, so that a host test can check
// the transposes against the package's gather tables by the dot-product
// identity.
#pragma once
#include "halo.cuh"

namespace fv3b {

// One halo copy of candidate p of tile t for component comp of a field with
// staggering (sx_of, sy_of): destination and source offsets (level 0), the
// source component and the sign (which scalar copies ignore).  False when p
// is not a halo point.
struct HaloCopy {
  idx_t dst, src;
  int src_comp, sign;
};

__host__ __device__ inline bool halo_copy(const Dims& d, int t, int p, int comp, const int sx_of[2],
                                          const int sy_of[2], int n_halo, HaloCopy& c) {
  int i, j;
  if (!halo_point(d, p, sx_of[comp], sy_of[comp], n_halo, i, j)) return false;
  HaloSource s;
  if (!halo_source(d, t, i, j, comp, sx_of, sy_of, n_halo, s)) return false;
  c.dst = idx3(d, t, i, j, 0);
  c.src = idx3(d, s.t, s.i, s.j, 0);
  c.src_comp = s.comp;
  c.sign = s.sign;
  return true;
}

// The copy of synchronize_vector_interfaces from position a of tile t's
// south edge line (comp 0, u) or west edge line (comp 1, v).
__host__ __device__ inline HaloCopy interface_sync_copy(const Dims& d, int t, int comp, int a, int& dst_comp) {
  HaloSource dst;
  interface_sync_target(d, t, comp == 0 ? EDGE_S : EDGE_W, a, dst);
  const int si = comp == 0 ? d.h + a : d.h, sj = comp == 0 ? d.h : d.h + a;
  HaloCopy c;
  c.dst = idx3(d, dst.t, dst.i, dst.j, 0);
  c.src = idx3(d, t, si, sj, 0);
  c.src_comp = comp;
  c.sign = dst.sign;
  dst_comp = dst.comp;
  return c;
}

}  // namespace fv3b

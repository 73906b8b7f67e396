// Host-side check of the fused del-n chain (deln_window_ok in
// fv3core_b200/csrc/transport.cuh) for a range of grids, printed as
// "n halo nmax ok" lines for a CPU test.
#include <cstdio>

#include "../../fv3core_b200/csrc/transport.cuh"

int main() {
  for (int h = 2; h <= 3; ++h)
    for (int n = 4; n <= 200; ++n)
      for (int nmax = 1; nmax <= 2; ++nmax) {
        fv3b_grid_dims g{n, h, 1, 0};
        const fv3b::Dims d = fv3b::make_dims(&g);
        std::printf("%d %d %d %d\n", n, h, nmax, fv3b::deln_window_ok(d, nmax) ? 1 : 0);
      }
  return 0;
}

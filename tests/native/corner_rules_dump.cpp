// Host build of the device corner-rule functions, for a CPU test that
// compares them with the oracle's rule tables.
#include <cstdio>
#include "../../fv3core_b200/csrc/corners.cuh"

int main(int argc, char** argv) {
  fv3b_grid_dims g{12, 3, 8, 0};
  fv3b::Dims d = fv3b::make_dims(&g);
  for (int i = 0; i < d.ni; ++i)
    for (int j = 0; j < d.nj; ++j) {
      int si, sj;
      if (fv3b::copy_corner_x(d, i, j, si, sj)) printf("cx %d %d %d %d\n", i, j, si, sj);
      if (fv3b::copy_corner_y(d, i, j, si, sj)) printf("cy %d %d %d %d\n", i, j, si, sj);
      if (fv3b::bgrid_corner_x(d, i, j, si, sj)) printf("bx %d %d %d %d\n", i, j, si, sj);
      if (fv3b::bgrid_corner_y(d, i, j, si, sj)) printf("by %d %d %d %d\n", i, j, si, sj);
    }
  return 0;
}

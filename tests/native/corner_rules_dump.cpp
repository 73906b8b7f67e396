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
      fv3b::CornerRule r;
      if (fv3b::corner_x(d, i, j, true, 1.0, 1.0, 1.0, 1.0, r)) printf("x3 %d %d %d %d\n", i, j, i + r.di, j + r.dj);
      if (fv3b::corner_x(d, i, j, false, 1.0, 1.0, 1.0, 1.0, r)) printf("x2 %d %d %d %d\n", i, j, i + r.di, j + r.dj);
      if (fv3b::corner_y(d, i, j, true, 1.0, 1.0, 1.0, 1.0, r)) printf("y3 %d %d %d %d\n", i, j, i + r.di, j + r.dj);
      if (fv3b::corner_y(d, i, j, false, 1.0, 1.0, 1.0, 1.0, r)) printf("y2 %d %d %d %d\n", i, j, i + r.di, j + r.dj);
    }
  return 0;
}

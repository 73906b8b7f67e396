// Host build of the device halo-source functions, for a CPU test that
// compares them with the Python gather tables (fv3core_b200/halo_map.py).
// Output lines: kind comp t i j src_t src_i src_j src_comp sign
#include <cstdio>
#include <cstdlib>
#include "../../fv3core_b200/csrc/halo.cuh"

static void dump(const fv3b::Dims& d, const char* kind, const int sx[2], const int sy[2], int ncomp, int n_halo) {
  for (int comp = 0; comp < ncomp; ++comp)
    for (int t = 0; t < 6; ++t)
      for (int p = 0; p < fv3b::halo_candidates(d, n_halo); ++p) {
        int i, j;
        if (!fv3b::halo_point(d, p, sx[comp], sy[comp], n_halo, i, j)) continue;
        fv3b::HaloSource s;
        if (!fv3b::halo_source(d, t, i, j, comp, sx, sy, n_halo, s)) {
          printf("miss %s %d %d %d %d\n", kind, comp, t, i, j);
          continue;
        }
        printf("%s %d %d %d %d %d %d %d %d %d\n", kind, comp, t, i, j, s.t, s.i, s.j, s.comp, s.sign);
      }
}

int main(int argc, char** argv) {
  int n = argc > 1 ? atoi(argv[1]) : 12;
  if (argc > 2) {  // "edges": the tile connectivity of 24 tile slots (four batched cubes)
    for (int t = 0; t < 24; ++t)
      for (int edge = 0; edge < 4; ++edge) {
        int t2, e2;
        bool rev;
        fv3b::edge_neighbor(t, edge, t2, e2, rev);
        printf("edge %d %d %d %d %d\n", t, edge, t2, e2, rev ? 1 : 0);
      }
    return 0;
  }
  fv3b_grid_dims g{n, 3, 8, 0};
  fv3b::Dims d = fv3b::make_dims(&g);
  const int centre[2] = {1, 1}, corner[2] = {0, 0};
  dump(d, "scalar3", centre, centre, 1, 3);
  dump(d, "scalar2", centre, centre, 1, 2);
  dump(d, "corner3", corner, corner, 1, 3);
  const int dsx[2] = {1, 0}, dsy[2] = {0, 1};  // D grid: u (x centre, y interface), v
  dump(d, "dgrid", dsx, dsy, 2, 3);
  const int csx[2] = {0, 1}, csy[2] = {1, 0};  // C grid: uc (x interface, y centre), vc
  dump(d, "cgrid", csx, csy, 2, 3);
  for (int t = 0; t < 6; ++t)
    for (int comp = 0; comp < 2; ++comp)
      for (int a = 0; a < n; ++a) {
        fv3b::HaloSource s;
        fv3b::interface_sync_target(d, t, comp == 0 ? fv3b::EDGE_S : fv3b::EDGE_W, a, s);
        int si = comp == 0 ? d.h + a : d.h, sj = comp == 0 ? d.h : d.h + a;
        printf("sync %d %d %d %d %d %d %d %d %d\n", s.comp, s.t, s.i, s.j, t, si, sj, comp, s.sign);
      }
  return 0;
}

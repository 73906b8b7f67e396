// Context layout shared by the stage sources.
#pragma once
#include "common.cuh"

namespace fv3b {
constexpr int NWS = 40;   // 3-D scratch fields in the workspace
constexpr int NCOL = 16;  // per-level column arrays
constexpr int MAXLEV = 128;

// indices of the per-level columns in ctx->col
enum ColumnId {
  COL_NORD = 0, COL_NORD_V, COL_NORD_W, COL_NORD_T, COL_DAMP_VT, COL_DAMP_W, COL_DAMP_T, COL_D2_DIVG,
  COL_D_CON, COL_KE_BG, COL_DAMP4_VT_C, COL_DAMP4_W_C, COL_DAMP4_VT, COL_DAMP4_T, COL_SPARE0, COL_SPARE1
};

// workspace slots (3-D scratch fields); a stage owns them only while it runs,
// except the D-grid contravariant winds, which keep their halo rows between
// calls like the reference's instance storages
enum WorkspaceId {
  WS_UC_CONTRA = 30, WS_VC_CONTRA = 31
};

struct DswSetup {
  bool ready = false;
  fv3b_dsw_config cfg;
  int nonzero_nord_k = 0, nonzero_nord = 0;
  int nmax_v = 0, nmax_w = 0, nmax_t = 0;
  double dd8 = 0.0;
};
}  // namespace fv3b

struct fv3b_ctx {
  fv3b::Dims d;
  fv3b_metrics m;
  double* ws_base = nullptr;
  double* ws[fv3b::NWS];
  double* col = nullptr;  // [NCOL][MAXLEV] device columns
  fv3b::DswSetup dsw;
};
